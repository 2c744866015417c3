// Launch-shape autotuner: per batch size, a grid scale for each tunable
// launch (the default grid x-extent times 2^scale), found by timing each
// kernel alone with the kernel probe at every scale and keeping the fastest
// (coordinate descent, kernel by kernel: the kernels of the chain run one
// after another, so each one's time depends on its own shape only).  The
// table lives in the context; a text cache keeps it per device and batch
// size.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "runtime.h"

namespace pixgpu {

const char* const kTuneNames[kNumTune] = {
    "kRawToDigi",      "kModuleBoundaries", "kFindClustersBig", "kGetHitsBig",       "kPhiCount",
    "kPhiFill",        "kPhiRec",           "kDoubletCount",    "kDoubletWrite",     "kOuterHitFill",
    "kOhRec",          "kConnect",          "kEdgeScatter",     "kNbrPool",          "kFishbone",
    "kNtupletCount",   "kNtupletWrite",     "kTrackCount",      "kTrackFill",        "kTrackPool",
    "kEarlyDup",       "kTupleDet",         "kClassify",        "kFastDupInDegree",
    "kHitToTupleCount", "kHitToTupleFill",  "kTripletCleaner",  "kFitZero",          "kBLFit",
    "kFedCopy"};

namespace {

int tuneIndex(const char* name) {
  if (!name) return -1;
  for (uint32_t i = 0; i < kNumTune; ++i)
    if (std::strcmp(name, kTuneNames[i]) == 0) return int(i);
  if (std::strcmp(name, "kRiemannFit") == 0 || std::strcmp(name, "kBLFitMixed") == 0 ||
      std::strcmp(name, "kRiemannFitMixed") == 0)
    return int(kTuneFit);
  return -1;
}

// the name the probe sees for a tunable launch
const char* launchedName(const pg_ctx* c, uint32_t id) {
  if (id == kTuneFit && c->cfg.riemann_fit) return c->cfg.mixed_fit ? "kRiemannFitMixed" : "kRiemannFit";
  if (id == kTuneFit && c->cfg.mixed_fit) return "kBLFitMixed";
  return kTuneNames[id];
}

void dropGraphs(pg_ctx* c) {
  for (auto& s : c->slots) {
    cudaStreamSynchronize(s.stream);
    for (auto& g : s.graphs) cudaGraphExecDestroy(g.second);
    s.graphs.clear();
    s.probeUsed.clear();
  }
}

std::string deviceName(const pg_ctx* c) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, c->cfg.device) != cudaSuccess) return "unknown";
  std::string n = p.name;
  for (auto& ch : n)
    if (ch == '|' || ch == '\n') ch = ' ';
  return n;
}

}  // namespace

LaunchTuning tuningFor(const pg_ctx* c, uint32_t n) {
  LaunchTuning t;
  std::memset(&t, 0, sizeof(t));
  // the table of this batch size, else of the largest tuned size below it
  auto it = c->tuning.upper_bound(n);
  if (it != c->tuning.begin()) t = std::prev(it)->second;
  return t;
}

}  // namespace pixgpu

using namespace pixgpu;

extern "C" {

const char* pg_tune_kernel_name(uint32_t i) { return i < kNumTune ? kTuneNames[i] : nullptr; }

int pg_tune_set(pg_ctx* c, uint32_t nEvents, const char* kernel, int scale) {
  if (!c || nEvents == 0) return PG_ERR_ARG;
  const int id = tuneIndex(kernel);
  if (id < 0) return fail(c, PG_ERR_NOTFOUND, "not a tunable kernel");
  if (scale < kTuneMinScale || scale > kTuneMaxScale) return fail(c, PG_ERR_ARG, "scale outside -3..3");
  std::lock_guard<std::mutex> lk(c->mu);
  for (auto& s : c->slots)
    if (s.state != SlotState::kFree) return fail(c, PG_ERR_BUSY, "pg_tune_set needs every slot free");
  cudaSetDevice(c->cfg.device);
  auto it = c->tuning.find(nEvents);
  if (it == c->tuning.end()) it = c->tuning.emplace(nEvents, tuningFor(c, nEvents)).first;
  it->second.scale[id] = int8_t(scale);
  dropGraphs(c);
  return PG_OK;
}

int pg_tune_get(const pg_ctx* c, uint32_t nEvents, const char* kernel, int* scale) {
  if (!c || !scale) return PG_ERR_ARG;
  const int id = tuneIndex(kernel);
  if (id < 0) return PG_ERR_NOTFOUND;
  *scale = tuningFor(c, nEvents).scale[id];
  return PG_OK;
}

int pg_tune_save(const pg_ctx* c, const char* path) {
  if (!c || !path) return PG_ERR_ARG;
  std::ofstream f(path);
  if (!f) return PG_ERR_ARG;
  const std::string dev = deviceName(c);
  f << "# launch tuning: <device>|<events per batch> <kernel> <grid scale (default x 2^scale)>\n";
  for (const auto& kv : c->tuning)
    for (uint32_t i = 0; i < kNumTune; ++i)  // every kernel, so that a tuned size never falls back to another
      f << dev << "|" << kv.first << " " << kTuneNames[i] << " " << int(kv.second.scale[i]) << "\n";
  return f ? PG_OK : PG_ERR_ARG;
}

// Applies the entries of this context's device; returns their number (>= 0)
// or a status.  Lines of other devices, unknown kernels or scales outside
// -3..3 are skipped.
int pg_tune_load(pg_ctx* c, const char* path) {
  if (!c || !path) return PG_ERR_ARG;
  std::ifstream f(path);
  if (!f) return fail(c, PG_ERR_NOTFOUND, "tuning cache not found");
  std::lock_guard<std::mutex> lk(c->mu);
  for (auto& s : c->slots)
    if (s.state != SlotState::kFree) return fail(c, PG_ERR_BUSY, "pg_tune_load needs every slot free");
  cudaSetDevice(c->cfg.device);
  const std::string dev = deviceName(c);
  std::string line;
  int applied = 0;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    const size_t bar = line.rfind('|');
    if (bar == std::string::npos || line.substr(0, bar) != dev) continue;
    std::istringstream in(line.substr(bar + 1));
    uint32_t n = 0;
    std::string name;
    int scale = 0;
    if (!(in >> n >> name >> scale) || n == 0) continue;
    const int id = tuneIndex(name.c_str());
    if (id < 0 || scale < kTuneMinScale || scale > kTuneMaxScale) continue;
    auto it = c->tuning.find(n);
    if (it == c->tuning.end()) {
      LaunchTuning z;
      std::memset(&z, 0, sizeof(z));
      it = c->tuning.emplace(n, z).first;
    }
    it->second.scale[id] = int8_t(scale);
    ++applied;
  }
  dropGraphs(c);
  return applied;
}

// Tunes the launches for batches of n events on the given raw records (the
// first n are used): for each tunable kernel, every scale in -2..2 is timed
// over `repeats` batches (after one to capture the graph) and the fastest is
// kept when it beats the current one by 2%.  *gain_ms (may be null) receives
// the summed saving per batch.  Every slot must be free; the probe setting is
// restored afterwards.
int pg_autotune(pg_ctx* c, uint32_t n, const uint8_t* const* raws, const size_t* sizes, uint32_t repeats,
                double* gain_ms) {
  if (!c || !raws || !sizes || n == 0 || n > c->cfg.max_events) return PG_ERR_ARG;
  if (repeats == 0) repeats = 3;
  const std::string probe0 = c->probeName;
  double gain = 0;
  int rc = PG_OK;
  auto timeBatches = [&](double* ms) -> int {
    std::vector<double> per;
    for (uint32_t r = 0; r <= repeats; ++r) {
      uint32_t slot = 0;
      int e = pg_submit(c, n, raws, sizes, &slot);
      if (e != PG_OK) return e;
      e = pg_wait(c, slot);
      pg_probe_entry buf[16];
      uint32_t got = 0;
      if (e == PG_OK) e = pg_probe_read(c, slot, 16, buf, &got);
      const int e2 = pg_release(c, slot);
      if (e != PG_OK) return e;
      if (e2 != PG_OK) return e2;
      double sum = 0;
      for (uint32_t i = 0; i < got; ++i) sum += buf[i].ms;
      if (r > 0) per.push_back(sum);  // the first batch captures the graph
    }
    std::sort(per.begin(), per.end());
    *ms = per[per.size() / 2];
    return PG_OK;
  };
  for (uint32_t id = 0; id < kNumTune && rc == PG_OK; ++id) {
    if (id == kTuneFedCopy && !c->cfg.fed_scan) continue;
    if ((rc = pg_set_probe(c, launchedName(c, id))) != PG_OK) break;
    const int start = tuningFor(c, n).scale[id];
    double best = 0;
    if ((rc = pg_tune_set(c, n, kTuneNames[id], start)) != PG_OK || (rc = timeBatches(&best)) != PG_OK) break;
    const double base = best;
    int bestScale = start;
    for (int s = -2; s <= 2 && rc == PG_OK; ++s) {
      if (s == start) continue;
      double ms = 0;
      if ((rc = pg_tune_set(c, n, kTuneNames[id], s)) != PG_OK || (rc = timeBatches(&ms)) != PG_OK) break;
      if (ms < 0.98 * best) {
        best = ms;
        bestScale = s;
      }
    }
    if (rc == PG_OK) rc = pg_tune_set(c, n, kTuneNames[id], bestScale);
    gain += base - best;
  }
  const int rp = pg_set_probe(c, probe0.empty() ? nullptr : probe0.c_str());
  if (rc == PG_OK) rc = rp;
  if (gain_ms) *gain_ms = gain;
  return rc;
}

}  // extern "C"
