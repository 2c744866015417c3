// C ABI of the B200 pixel chain (include/pixgpu.h): context, ES upload,
// host FED scan, batch slots, captured graphs, asynchronous batches and
// product access.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "runtime.h"

namespace pixgpu {
cudaError_t fitDirect(int N, uint32_t n, const double* hits, const float* ge, double B, float* state, float* cov,
                      float* pt, float* eta, float* chi2, cudaStream_t stream);
cudaError_t fitDirectMixed(int N, uint32_t n, const double* hits, const float* ge, double B, float* state, float* cov,
                           float* pt, float* eta, float* chi2, cudaStream_t stream);
cudaError_t fitDirectRiemann(int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                             float* cov, float* pt, float* eta, float* chi2, bool mixed, cudaStream_t stream);

int fail(pg_ctx* c, int code, const std::string& msg) {
  if (c) {
    std::lock_guard<std::mutex> lk(c->errMu);
    c->err = msg;
  }
  return code;
}
bool resolveCaps(const pg_config& cfg, Caps* out) {
  const Caps r = referenceCaps();
  Caps c = r;
  auto pick = [](uint32_t v, uint32_t def) { return v ? v : def; };
  c.fedWords = pick(cfg.cap_fed_words, r.fedWords);
  c.hits = pick(cfg.cap_hits, r.hits);
  c.cells = pick(cfg.cap_doublets, r.cells);
  c.lists = pick(cfg.cap_lists, r.lists);
  c.tuples = pick(cfg.cap_tuples, r.tuples);
  c.multiplicity = pick(cfg.cap_multiplicity, r.multiplicity);
  c.h2t = pick(cfg.cap_hit_to_tuple, r.h2t);
  if (c.fedWords < r.fedWords || c.hits < r.hits || c.cells < r.cells || c.lists < r.lists || c.tuples < r.tuples ||
      c.multiplicity < r.multiplicity || c.h2t < r.h2t)
    return false;
  // the doublet search packs hit indices into 21 bits; the multiplicity fill
  // counts each bin in a 20-bit field
  if (c.hits > kMaxHitCapLimit || c.tuples >= (1u << 20) || c.multiplicity > c.tuples) return false;
  if (uint64_t(c.cells) * 2 > 0xffffffffull || uint64_t(c.hits) * 6 > 0xffffffffull) return false;
  c.jCap = 6 * c.hits;
  // CA links kept: the reference's 2 x 458752, or one per doublet beyond it
  c.edges = std::max(r.edges, c.cells);
  // scratchA/scratchB: CA link staging, two duplicate-round worklists of
  // cells, the doublet staging (one entry per inner-hit slot in B) and the
  // vertex finder's per-track arrays
  c.scratch = std::max<uint32_t>(std::max(std::max(c.edges, 2 * c.cells), c.jCap), uint32_t(kVtxScratchAWords));
  *out = c;
  return true;
}

std::string lastError(pg_ctx* c) {
  std::lock_guard<std::mutex> lk(c->errMu);
  return c->err;
}
int cudaFail(pg_ctx* c, cudaError_t e, const char* where) {
  return fail(c, PG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
}  // namespace pixgpu

using namespace pixgpu;

namespace {

struct Rd {
  const uint8_t* p;
  size_t n, off = 0;
  bool ok = true;
  void bytes(void* d, size_t k) {
    if (off + k > n) {
      ok = false;
      return;
    }
    std::memcpy(d, p + off, k);
    off += k;
  }
  template <typename T>
  T get() {
    T x{};
    bytes(&x, sizeof(T));
    return x;
  }
};

}  // namespace

// FED scan: Source record -> (words, fed index per word pair); follows
// SiPixelRawToClusterCUDA.cc:78-138 with ErrorChecker.cc:36-91 semantics.
namespace {

// the record's FED directory (Source.cc:9-21): data pointer and byte size of
// each FED id; PG_ERR_FORMAT for a truncated record or an id >= 4096
int fedDirectory(const uint8_t* raw, size_t n, const uint8_t** fedPtr, uint32_t* fedSize) {
  std::memset(fedSize, 0, 4096 * sizeof(uint32_t));
  Rd r{raw, n};
  uint32_t nfeds = r.get<uint32_t>();
  if (!r.ok) return PG_ERR_FORMAT;
  for (uint32_t i = 0; i < nfeds; ++i) {
    uint32_t id = r.get<uint32_t>(), size = r.get<uint32_t>();
    if (!r.ok || id >= 4096 || r.off + size > n) return PG_ERR_FORMAT;
    fedPtr[id] = raw + r.off;
    fedSize[id] = size;
    r.off += size;
  }
  return PG_OK;
}

}  // namespace

int pixgpu::unpackRaw(const std::vector<uint32_t>& fedIds, const uint8_t* raw, size_t n, uint32_t* words, uint8_t* fed,
              uint32_t cap, uint32_t* nWordsOut, std::vector<PfFormatterError>* fmt) {
  const uint8_t* fedPtr[4096];
  uint32_t fedSize[4096];
  if (fedDirectory(raw, n, fedPtr, fedSize) != PG_OK) return PG_ERR_FORMAT;
  uint32_t wc = 0;
  for (uint32_t fedId : fedIds) {
    if (fedId == 40 || fedId >= 4096) continue;
    uint32_t size = fedSize[fedId];
    int n64 = int(size / 8);
    if (n64 == 0) continue;
    const uint8_t* d = fedPtr[fedId];
    auto w64 = [&](int k) {
      uint64_t v;
      std::memcpy(&v, d + 8 * size_t(k), 8);
      return v;
    };
    auto record = [&](uint64_t v, uint32_t type) {
      if (fmt) fmt->push_back(PfFormatterError{v, type, fedId});
    };
    // checkCRC: the CRC-modified bit of the last word drops the FED
    if ((w64(n64 - 1) >> 2) & 1) {
      record(w64(n64 - 1), 39);
      continue;
    }
    // checkHeader: start marker 0x5 (else the headers end, unrecorded),
    // source id, more-headers bit; bounded by the FED (the reference is not)
    int h = -1;
    bool more = true;
    while (more && h + 1 < n64) {
      ++h;
      uint64_t v = w64(h);
      if (((uint32_t(v >> 32) >> 28) & 0xf) != 0x5) break;
      if (((uint32_t(v) >> 8) & 0xfff) != fedId) record(v, 32);
      more = (uint32_t(v) >> 3) & 1;
    }
    // checkTrailer: end marker 0xa (else type 33 and the trailers end),
    // fragment length against the FED's 64-bit words (type 34), more-trailers bit
    int t = n64;
    more = true;
    while (more && t > 0) {
      --t;
      uint64_t v = w64(t);
      if (((uint32_t(v >> 32) >> 28) & 0xf) != 0xa) {
        record(v, 33);
        break;
      }
      if ((uint32_t(v >> 32) & 0x00ffffffu) != uint32_t(n64)) record(v, 34);
      more = (uint32_t(v) >> 3) & 1;
    }
    if (t < h + 1) continue;  // header and trailer overlap (undefined in the reference): no payload
    uint32_t len = uint32_t(t - (h + 1)) * 2;
    if (wc + len > cap) return PG_ERR_CAPACITY;
    std::memcpy(words + wc, d + 8 * size_t(h + 1), 4 * size_t(len));
    std::memset(fed + wc / 2, int(fedId - 1200), len / 2);
    wc += len;
  }
  *nWordsOut = wc;
  return PG_OK;
}

namespace {

int uploadES(pg_ctx* c, const pg_es_images* es) {
  Rd cpe{es->cpe, es->cpe_size}, bs{es->beamspot, es->beamspot_size}, fi{es->fedids, es->fedids_size};
  // sizes
  if (es->cabling_size < sizeof(PfCablingMap) + 4) return fail(c, PG_ERR_FORMAT, "cabling image too short");
  uint32_t nUnp;
  std::memcpy(&nUnp, es->cabling + sizeof(PfCablingMap), 4);
  if (es->cabling_size < sizeof(PfCablingMap) + 4 + nUnp || nUnp < PF_MAX_SIZE)
    return fail(c, PG_ERR_FORMAT, "cabling image: modToUnp size");
  if (es->gain_size < sizeof(PfGainHeader) + 4) return fail(c, PG_ERR_FORMAT, "gain image too short");
  uint32_t nGain;
  std::memcpy(&nGain, es->gain + sizeof(PfGainHeader), 4);
  if (es->gain_size < sizeof(PfGainHeader) + 4 + nGain) return fail(c, PG_ERR_FORMAT, "gain payload truncated");
  PfGainHeader gh;
  std::memcpy(&gh, es->gain, sizeof(gh));
  for (int i = 0; i < PF_MAX_MODULES; ++i) {
    if (gh.rangeAndCols[i].nCols <= 0 || gh.rangeAndCols[i].second > nGain)
      return fail(c, PG_ERR_FORMAT, "gain ranges outside the payload");
  }
  PfCommonParams common = cpe.get<PfCommonParams>();
  uint32_t nDet = cpe.get<uint32_t>();
  if (!cpe.ok || nDet < PF_N_MODULES || nDet > 4096) return fail(c, PG_ERR_FORMAT, "cpe image: detector count");
  std::vector<PfDetParams> det(nDet);
  cpe.bytes(det.data(), nDet * sizeof(PfDetParams));
  PfAverageGeometry ag = cpe.get<PfAverageGeometry>();
  PfLayerGeometry lg = cpe.get<PfLayerGeometry>();
  if (!cpe.ok) return fail(c, PG_ERR_FORMAT, "cpe image truncated");
  PfBeamSpot b = bs.get<PfBeamSpot>();
  if (!bs.ok) return fail(c, PG_ERR_FORMAT, "beamspot image truncated");
  uint32_t nf = fi.get<uint32_t>();
  if (!fi.ok || nf > 4096) return fail(c, PG_ERR_FORMAT, "fedIds image");
  c->hes.fedIds.resize(nf);
  fi.bytes(c->hes.fedIds.data(), nf * 4);
  if (!fi.ok) return fail(c, PG_ERR_FORMAT, "fedIds image truncated");
  c->hes.scanFeds.clear();
  for (uint32_t id : c->hes.fedIds)
    if (id != 40 && id < 4096) c->hes.scanFeds.push_back(id);
  // one device allocation for the resident conditions
  size_t off = 0;
  auto place = [&](size_t bytes) {
    off = (off + 255) & ~size_t(255);
    size_t o = off;
    off += bytes;
    return o;
  };
  size_t oCab = place(sizeof(PfCablingMap)), oUnp = place(PF_MAX_SIZE), oGh = place(sizeof(PfGainHeader)),
         oGp = place(nGain), oCom = place(sizeof(PfCommonParams)), oDet = place(nDet * sizeof(PfDetParams)),
         oAg = place(sizeof(PfAverageGeometry)), oLg = place(sizeof(PfLayerGeometry)), oBs = place(sizeof(PfBeamSpot));
  cudaError_t e = cudaMalloc(&c->esMem, off);
  if (e != cudaSuccess) return cudaFail(c, e, "cudaMalloc(ES)");
  char* base = static_cast<char*>(c->esMem);
  struct Cp {
    size_t o;
    const void* src;
    size_t n;
  } cps[] = {{oCab, es->cabling, sizeof(PfCablingMap)},
             {oUnp, es->cabling + sizeof(PfCablingMap) + 4, PF_MAX_SIZE},
             {oGh, es->gain, sizeof(PfGainHeader)},
             {oGp, es->gain + sizeof(PfGainHeader) + 4, nGain},
             {oCom, &common, sizeof(common)},
             {oDet, det.data(), nDet * sizeof(PfDetParams)},
             {oAg, &ag, sizeof(ag)},
             {oLg, &lg, sizeof(lg)},
             {oBs, &b, sizeof(b)}};
  for (auto& cp : cps) {
    e = cudaMemcpy(base + cp.o, cp.src, cp.n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cudaFail(c, e, "cudaMemcpy(ES)");
  }
  c->des.cab = reinterpret_cast<const PfCablingMap*>(base + oCab);
  c->des.modToUnp = reinterpret_cast<const uint8_t*>(base + oUnp);
  c->des.gainHdr = reinterpret_cast<const PfGainHeader*>(base + oGh);
  c->des.gainPayload = reinterpret_cast<const uint8_t*>(base + oGp);
  c->des.common = reinterpret_cast<const PfCommonParams*>(base + oCom);
  c->des.det = reinterpret_cast<const PfDetParams*>(base + oDet);
  c->des.ag = reinterpret_cast<const PfAverageGeometry*>(base + oAg);
  c->des.lg = reinterpret_cast<const PfLayerGeometry*>(base + oLg);
  c->des.bs = reinterpret_cast<const PfBeamSpot*>(base + oBs);
  c->des.nDet = nDet;
  c->des.gainPayloadSize = nGain;
  return PG_OK;
}

// Device FED scan: copies every FED block of the ES list, header to trailer,
// to the pinned raw buffer and writes the per-event FED table; the payload
// words are bounded by two per 64-bit word between one header and one trailer
// (the exact count for well-formed FEDs), which must fit the event and batch
// capacities.
int stageRawBlocks(pg_ctx* c, Slot& s, uint32_t nEvents, const uint8_t* const* raws, const size_t* sizes) {
  const FedScanBuffers& fs = s.ws.scan;
  const uint32_t F = fs.nFeds;
  const uint32_t* ids = c->hes.scanFeds.data();
  const uint8_t* fedPtr[4096];
  uint32_t fedSize[4096];
  uint64_t cursor = 0, batchBound = 0;
  for (uint32_t k = 0; k < nEvents; ++k) {
    if (fedDirectory(raws[k], sizes[k], fedPtr, fedSize) != PG_OK) return fail(c, PG_ERR_FORMAT, "malformed raw record");
    uint64_t bound = 0;
    uint2* tab = s.hTab + size_t(k) * F;
    for (uint32_t j = 0; j < F; ++j) {
      const uint32_t n64 = fedSize[ids[j]] / 8;
      if (cursor + n64 > fs.rawCap64) return fail(c, PG_ERR_CAPACITY, "raw records larger than the staging buffer");
      tab[j] = make_uint2(uint32_t(cursor), n64);
      if (n64) std::memcpy(s.hRaw + cursor, fedPtr[ids[j]], size_t(n64) * 8);
      cursor += n64;
      bound += n64 >= 2 ? 2 * uint64_t(n64 - 2) : 0;
    }
    if (bound > c->caps.fedWords) return fail(c, PG_ERR_CAPACITY, "event or batch too large");
    batchBound += bound;
  }
  if (batchBound > c->cfg.max_words_per_batch) return fail(c, PG_ERR_CAPACITY, "event or batch too large");
  cudaError_t e;
  if (cursor && (e = cudaMemcpyAsync(fs.raw64, s.hRaw, size_t(cursor) * 8, cudaMemcpyHostToDevice, s.stream)) !=
                    cudaSuccess)
    return cudaFail(c, e, "H2D FED blocks");
  if ((e = cudaMemcpyAsync(fs.tab, s.hTab, size_t(nEvents) * F * sizeof(uint2), cudaMemcpyHostToDevice,
                           s.stream)) != cudaSuccess)
    return cudaFail(c, e, "H2D FED table");
  s.fmtErrors.clear();
  s.fmtOff.clear();
  s.nEvents = nEvents;
  s.staged = true;
  return PG_OK;
}

int stage(pg_ctx* c, Slot& s, uint32_t nEvents, const uint8_t* const* raws, const size_t* sizes) {
  if (nEvents == 0 || nEvents > c->cfg.max_events) return fail(c, PG_ERR_CAPACITY, "batch size");
  if (s.ws.scan.on) return stageRawBlocks(c, s, nEvents, raws, sizes);
  uint32_t off = 0;
  const bool fmt = c->cfg.formatter_errors != 0;
  s.fmtErrors.clear();
  s.fmtOff.assign(1, 0);
  for (uint32_t k = 0; k < nEvents; ++k) {
    s.hOffsets[k] = off;
    uint32_t nw = 0;
    uint32_t room = c->cfg.max_words_per_batch - off;
    room = room > c->caps.fedWords ? c->caps.fedWords : room;
    int rc = unpackRaw(c->hes.fedIds, raws[k], sizes[k], s.hWords + off, s.hFed + off / 2, room, &nw,
                       fmt ? &s.fmtErrors : nullptr);
    s.fmtOff.push_back(uint32_t(s.fmtErrors.size()));
    if (rc != PG_OK) return fail(c, rc, rc == PG_ERR_CAPACITY ? "event or batch too large" : "malformed raw record");
    off += nw;
  }
  s.hOffsets[nEvents] = off;
  cudaError_t e;
  if (off) {
    if ((e = cudaMemcpyAsync(s.ws.words, s.hWords, size_t(off) * 4, cudaMemcpyHostToDevice, s.stream)) != cudaSuccess)
      return cudaFail(c, e, "H2D words");
    if ((e = cudaMemcpyAsync(s.ws.fedIds, s.hFed, size_t(off) / 2 + 1, cudaMemcpyHostToDevice, s.stream)) !=
        cudaSuccess)
      return cudaFail(c, e, "H2D fedIds");
  }
  if ((e = cudaMemcpyAsync(s.ws.wordOffsets, s.hOffsets, size_t(nEvents + 1) * 4, cudaMemcpyHostToDevice,
                           s.stream)) != cudaSuccess)
    return cudaFail(c, e, "H2D offsets");
  s.nEvents = nEvents;
  s.staged = true;
  return PG_OK;
}

// Captures runChain + result packing for `n` events on the slot's stream.
int captureGraph(pg_ctx* c, Slot& s, uint32_t n, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cudaFail(c, e, "begin capture");
  KernelProbe* pr = c->probeName.empty() ? nullptr : s.probe;
  if (pr) pr->used = 0;
  tProbe = pr;
  s.ws.tune = tuningFor(c, n);
  cudaError_t le = runChain(c->des, s.ws, n, s.stream, c->cfg.riemann_fit != 0, int(c->cfg.vertex_algo));
  if (le == cudaSuccess) {
    launchPack(s.ws, n, s.dRes, s.stream);
    le = cudaGetLastError();
  }
  tProbe = nullptr;
  s.probeUsed[n] = pr ? pr->used : 0;
  e = cudaStreamEndCapture(s.stream, &g);
  if (le != cudaSuccess || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cudaFail(c, le != cudaSuccess ? le : e, "graph capture");
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cudaFail(c, e, "graph instantiate");
  return PG_OK;
}

template <typename T>
int copyOut(pg_ctx* c, Slot& s, const T* src, size_t n, void* dst, size_t cap, size_t* count, int* elem) {
  *elem = int(sizeof(T));
  *count = n;
  if (!dst) return PG_OK;
  if (n * sizeof(T) > cap) return fail(c, PG_ERR_CAPACITY, "product larger than the destination");
  if (n == 0) return PG_OK;
  cudaError_t e = cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, s.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) return cudaFail(c, e, "D2H product");
  return PG_OK;
}

}  // namespace

int pixgpu::captureGraphFor(pg_ctx* c, Slot& s, uint32_t n) {
  if (s.graphs.count(n)) return PG_OK;
  cudaGraphExec_t g = nullptr;
  int rc = captureGraph(c, s, n, &g);
  if (rc != PG_OK) return rc;
  s.graphs.emplace(n, g);
  return PG_OK;
}

int pixgpu::launchBatch(pg_ctx* c, Slot& s) {
  cudaError_t e;
  if (c->cfg.use_graphs) {
    int rc = captureGraphFor(c, s, s.nEvents);
    if (rc != PG_OK) return rc;
    s.lastProbeUsed = s.probeUsed[s.nEvents];
    e = cudaGraphLaunch(s.graphs[s.nEvents], s.stream);
    if (e != cudaSuccess) return cudaFail(c, e, "graph launch");
  } else {
    KernelProbe* pr = c->probeName.empty() ? nullptr : s.probe;
    if (pr) pr->used = 0;
    tProbe = pr;
    s.ws.tune = tuningFor(c, s.nEvents);
    e = runChain(c->des, s.ws, s.nEvents, s.stream, c->cfg.riemann_fit != 0, int(c->cfg.vertex_algo));
    if (e == cudaSuccess) launchPack(s.ws, s.nEvents, s.dRes, s.stream);
    tProbe = nullptr;
    s.lastProbeUsed = pr ? pr->used : 0;
    if (e != cudaSuccess) return cudaFail(c, e, "chain launch");
  }
  e = cudaEventRecord(s.done, s.stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cudaFail(c, e, "chain launch");
  return PG_OK;
}

int pixgpu::findFreeSlot(pg_ctx* c) {
  for (size_t i = 0; i < c->slots.size(); ++i)
    if (c->slots[i].state == SlotState::kFree) return int(i);
  return -1;
}

extern "C" {

void pg_default_config(pg_config* cfg) {
  cfg->device = 0;
  cfg->max_events = 64;
  cfg->max_words_per_batch = 64u * 160000u;
  cfg->slots = 1;
  cfg->use_graphs = 1;
  cfg->pool_words = 0;
  cfg->hbm_fraction = 0.5;
  cfg->riemann_fit = 0;
  cfg->vertex_algo = 0;
  // CAHitNtupletGeneratorOnGPU.cc:45-66
  cfg->min_hits_per_ntuplet = 3;
  cfg->include_jumping_forward_doublets = 1;
  cfg->early_fishbone = 1;
  cfg->late_fishbone = 0;
  cfg->ideal_conditions = 1;
  cfg->do_cluster_cut = 1;
  cfg->do_z0_cut = 1;
  cfg->do_pt_cut = 1;
  cfg->formatter_errors = 0;
  cfg->fed_scan = 0;
  cfg->mixed_fit = 0;
  // the reference's container capacities
  cfg->cap_fed_words = cfg->cap_hits = cfg->cap_doublets = cfg->cap_lists = 0;
  cfg->cap_tuples = cfg->cap_multiplicity = cfg->cap_hit_to_tuple = 0;
}

namespace {

int createSlot(pg_ctx* c, Slot& s, size_t bytes) {
  const uint32_t E = c->cfg.max_events;
  if (cudaMalloc(&s.dmem, bytes) != cudaSuccess) return fail(c, PG_ERR_NOMEM, "slot workspace");
  workspaceCarve(s.ws, s.dmem, E, c->cfg.max_words_per_batch, c->caps);
  // scan state words and batch epochs start at zero (no tile published)
  if (cudaMemset(s.ws.scanState, 0, size_t(E) * kScanCalls * s.ws.scanTiles * sizeof(uint64_t)) != cudaSuccess ||
      cudaMemset(s.ws.scanEpoch, 0, size_t(E) * sizeof(uint32_t)) != cudaSuccess)
    return fail(c, PG_ERR_CUDA, "slot scan state");
  // layer pairs of CAHitNtupletGeneratorKernels.cc:52-57
  s.ws.ca.nPairs = c->cfg.min_hits_per_ntuplet > 3 ? 13u : (c->cfg.include_jumping_forward_doublets ? 19u : 15u);
  s.ws.ca.minHits = c->cfg.min_hits_per_ntuplet;
  s.ws.ca.idealConditions = c->cfg.ideal_conditions != 0;
  s.ws.ca.doClusterCut = c->cfg.do_cluster_cut != 0;
  s.ws.ca.doZ0Cut = c->cfg.do_z0_cut != 0;
  s.ws.ca.doPtCut = c->cfg.do_pt_cut != 0;
  s.ws.ca.earlyFishbone = c->cfg.early_fishbone != 0;
  s.ws.ca.lateFishbone = c->cfg.late_fishbone != 0;
  s.ws.ca.mixedFit = c->cfg.mixed_fit != 0;
  if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s.gathered, cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost(&s.hWords, size_t(c->cfg.max_words_per_batch) * 4) != cudaSuccess ||
      cudaMallocHost(&s.hFed, size_t(c->cfg.max_words_per_batch) / 2 + 16) != cudaSuccess ||
      cudaMallocHost(&s.hOffsets, size_t(E + 1) * 4) != cudaSuccess ||
      cudaMallocHost(&s.hRefs, size_t(E) * sizeof(PoolRef)) != cudaSuccess ||
      cudaMalloc(&s.dRefs, size_t(E) * sizeof(PoolRef)) != cudaSuccess ||
      cudaHostAlloc(&s.hRes, size_t(E) * kResultStride, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void**>(&s.dRes), s.hRes, 0) != cudaSuccess)
    return fail(c, PG_ERR_NOMEM, "slot stream, events or pinned buffers");
  if (c->cfg.fed_scan) {
    // device FED scan buffers (fedscan.cu)
    FedScanBuffers& fs = s.ws.scan;
    const uint32_t F = uint32_t(c->hes.scanFeds.size());
    fs.on = 1;
    fs.recordErrors = c->cfg.formatter_errors != 0;
    fs.nFeds = F;
    // payload plus up to four framing words per FED
    fs.rawCap64 = c->cfg.max_words_per_batch / 2 + 4 * E * F + 16;
    const size_t EF = size_t(E) * F;
    size_t off = 0;
    auto take = [&](size_t bytes) {
      size_t o = off;
      off = (off + bytes + 255) & ~size_t(255);
      return o;
    };
    const size_t oIds = take(F * 4), oRaw = take(size_t(fs.rawCap64) * 8), oTab = take(EF * sizeof(uint2)),
                 oLen = take(EF * 4), oSrc = take(EF * 4), oDst = take(EF * 4), oEv = take(size_t(E) * 4),
                 oFmt = take(size_t(E) * kFmtErrCap * sizeof(PfFormatterError)), oCnt = take(size_t(E) * 4);
    if (cudaMalloc(&s.dScan, off) != cudaSuccess ||
        cudaMallocHost(&s.hRaw, size_t(fs.rawCap64) * 8) != cudaSuccess ||
        cudaMallocHost(&s.hTab, EF * sizeof(uint2) + 8) != cudaSuccess)
      return fail(c, PG_ERR_NOMEM, "FED scan buffers");
    char* b = static_cast<char*>(s.dScan);
    fs.fedIds = reinterpret_cast<const uint32_t*>(b + oIds);
    fs.raw64 = reinterpret_cast<uint64_t*>(b + oRaw);
    fs.tab = reinterpret_cast<uint2*>(b + oTab);
    fs.len = reinterpret_cast<uint32_t*>(b + oLen);
    fs.src = reinterpret_cast<uint32_t*>(b + oSrc);
    fs.dst = reinterpret_cast<uint32_t*>(b + oDst);
    fs.evWords = reinterpret_cast<uint32_t*>(b + oEv);
    fs.fmt = reinterpret_cast<PfFormatterError*>(b + oFmt);
    fs.fmtCount = reinterpret_cast<uint32_t*>(b + oCnt);
    if (F && cudaMemcpyAsync(b + oIds, c->hes.scanFeds.data(), F * 4, cudaMemcpyHostToDevice, s.stream) !=
                 cudaSuccess)
      return fail(c, PG_ERR_CUDA, "FED id list");
  }
  // the kernels read the batch input through this descriptor
  launchSetInput(s.ws, s.ws.words, s.ws.fedIds, s.stream);
  cudaError_t e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) return cudaFail(c, e, "slot set-up");
  return PG_OK;
}

void destroySlot(Slot& s) {
  if (s.stream) cudaStreamSynchronize(s.stream);
  for (auto& g : s.graphs) cudaGraphExecDestroy(g.second);
  s.graphs.clear();
  if (s.probe) {
    for (auto& ev : s.probe->ev)
      if (ev) cudaEventDestroy(ev);
    delete s.probe;
    s.probe = nullptr;
  }
  if (s.dmem) cudaFree(s.dmem);
  if (s.dScan) cudaFree(s.dScan);
  if (s.hRaw) cudaFreeHost(s.hRaw);
  if (s.hTab) cudaFreeHost(s.hTab);
  if (s.dRefs) cudaFree(s.dRefs);
  if (s.done) cudaEventDestroy(s.done);
  if (s.gathered) cudaEventDestroy(s.gathered);
  if (s.stream) cudaStreamDestroy(s.stream);
  if (s.hWords) cudaFreeHost(s.hWords);
  if (s.hFed) cudaFreeHost(s.hFed);
  if (s.hOffsets) cudaFreeHost(s.hOffsets);
  if (s.hRefs) cudaFreeHost(s.hRefs);
  if (s.hRes) cudaFreeHost(s.hRes);
}

}  // namespace

int pg_create(const pg_es_images* es, const pg_config* cfgIn, pg_ctx** out) {
  if (!es || !out) return PG_ERR_ARG;
  *out = nullptr;
  auto c = std::make_unique<pg_ctx>();
  if (cfgIn)
    c->cfg = *cfgIn;
  else
    pg_default_config(&c->cfg);
  if (c->cfg.max_events == 0 || c->cfg.max_events > kFlatMaxEvents || c->cfg.max_words_per_batch == 0 || c->cfg.max_words_per_batch > (1u << 30) ||
      c->cfg.vertex_algo > 2 || c->cfg.min_hits_per_ntuplet < 3 || c->cfg.min_hits_per_ntuplet > 4 ||
      c->cfg.fed_scan > 1 || (c->cfg.fed_scan && c->cfg.pool_words) ||  // the pool stages on the host
      c->cfg.mixed_fit > 1)
    return PG_ERR_ARG;
  if (!resolveCaps(c->cfg, &c->caps)) return PG_ERR_ARG;
  c->device = c->cfg.device;
  cudaError_t e = cudaSetDevice(c->cfg.device);
  if (e != cudaSuccess) return PG_ERR_CUDA;
  int rc = uploadES(c.get(), es);
  if (rc != PG_OK) {
    if (c->esMem) cudaFree(c->esMem);
    return rc;
  }
  if (c->cfg.pool_words) {
    rc = poolCreate(c.get(), c->cfg.pool_words);
    if (rc != PG_OK) {
      pg_destroy(c.release());
      return rc;
    }
  }
  size_t bytes = workspaceBytes(c->cfg.max_events, c->cfg.max_words_per_batch, c->caps);
  uint32_t nSlots = c->cfg.slots;
  if (nSlots == 0) {
    // admission by free HBM: as many slots as fit in the given share of the free memory
    size_t freeB = 0, totalB = 0;
    if ((e = cudaMemGetInfo(&freeB, &totalB)) != cudaSuccess) {
      pg_destroy(c.release());
      return PG_ERR_CUDA;
    }
    double frac = c->cfg.hbm_fraction > 0 && c->cfg.hbm_fraction <= 0.95 ? c->cfg.hbm_fraction : 0.5;
    size_t fit = size_t(double(freeB) * frac) / bytes;
    nSlots = uint32_t(std::min<size_t>(std::max<size_t>(fit, 1), 16));
    c->cfg.slots = nSlots;
  }
  c->slots.resize(nSlots);
  for (auto& s : c->slots) {
    if ((rc = createSlot(c.get(), s, bytes)) != PG_OK) {
      std::string msg = c->err;
      pg_destroy(c.release());
      return rc;
    }
  }
  *out = c.release();
  return PG_OK;
}

void pg_destroy(pg_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->cfg.device);
  for (auto& s : c->slots) destroySlot(s);
  poolDestroy(c);
  if (c->esMem) cudaFree(c->esMem);
  delete c;
}

int pg_get_config(const pg_ctx* c, pg_config* out) {
  if (!c || !out) return PG_ERR_ARG;
  *out = c->cfg;
  return PG_OK;
}

const char* pg_last_error(const pg_ctx* c) { return c ? c->err.c_str() : "null context"; }

size_t pg_slot_bytes(const pg_ctx* c) {
  return c ? workspaceBytes(c->cfg.max_events, c->cfg.max_words_per_batch, c->caps) : 0;
}

int pg_unpack_raw(const pg_ctx* c, const uint8_t* raw, size_t n, uint32_t* words, uint8_t* fedIds, uint32_t cap,
                  uint32_t* nWords) {
  if (!c || !raw || !words || !fedIds || !nWords) return PG_ERR_ARG;
  return unpackRaw(c->hes.fedIds, raw, n, words, fedIds, cap, nWords);
}

int pg_cluster_digis(pg_ctx* c, uint32_t n, const uint16_t* moduleInd, const uint16_t* xx, const uint16_t* yy,
                     const uint16_t* adc, uint16_t* moduleIndOut, int32_t* clus, uint32_t* clusInModule,
                     uint32_t* moduleId, uint32_t* moduleStart, uint32_t* nModules, uint32_t* flags) {
  if (!c || !moduleInd || !xx || !yy || !adc || !moduleIndOut || !clus || !clusInModule || !moduleId ||
      !moduleStart || !nModules)
    return PG_ERR_ARG;
  Slot& s = c->slots[0];
  if (s.state != SlotState::kFree) return fail(c, PG_ERR_BUSY, "slot 0 holds an asynchronous batch");
  if (n > c->cfg.max_words_per_batch || n > c->caps.fedWords)
    return fail(c, PG_ERR_CAPACITY, "more digis than a batch or an event holds");
  cudaSetDevice(c->cfg.device);
  Workspace& ws = s.ws;
  std::vector<int32_t> iota(n);
  for (uint32_t i = 0; i < n; ++i) iota[i] = int32_t(i);
  const uint32_t off[2] = {0, n};
  cudaError_t e = cudaSuccess;
  auto h2d = [&](void* dst, const void* src, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s.stream);
  };
  h2d(ws.moduleInd, moduleInd, size_t(n) * 2);
  h2d(ws.xx, xx, size_t(n) * 2);
  h2d(ws.yy, yy, size_t(n) * 2);
  h2d(ws.adc, adc, size_t(n) * 2);
  h2d(ws.clus, iota.data(), size_t(n) * 4);
  h2d(ws.wordOffsets, off, sizeof(off));
  if (e == cudaSuccess) e = runClusters(ws, 1, s.stream);
  EventCounters ec{};
  auto d2h = [&](void* dst, const void* src, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s.stream);
  };
  d2h(moduleIndOut, ws.moduleInd, size_t(n) * 2);
  d2h(clus, ws.clus, size_t(n) * 4);
  d2h(clusInModule, ws.clusInModule, size_t(kMaxModules) * 4);
  d2h(moduleId, ws.moduleId, size_t(kMaxModules) * 4);
  d2h(moduleStart, ws.moduleStart, size_t(kMaxModules + 1) * 4);
  d2h(&ec, ws.ev, sizeof(ec));
  if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) return cudaFail(c, e, "clustering");
  s.nEvents = 0;  // the slot's products no longer describe a batch
  *nModules = std::min(ec.nModules, kMaxModules);
  if (flags) *flags = ec.flags;
  return PG_OK;
}

int pg_stage_batch(pg_ctx* c, uint32_t slot, uint32_t nEvents, const uint8_t* const* raws, const size_t* sizes) {
  if (!c || slot >= c->slots.size() || !raws || !sizes) return PG_ERR_ARG;
  if (c->slots[slot].state != SlotState::kFree) return fail(c, PG_ERR_BUSY, "slot holds an asynchronous batch");
  cudaSetDevice(c->cfg.device);
  return stage(c, c->slots[slot], nEvents, raws, sizes);
}

int pg_run_staged(pg_ctx* c, uint32_t slot) {
  if (!c || slot >= c->slots.size() || !c->slots[slot].staged) return PG_ERR_ARG;
  return launchBatch(c, c->slots[slot]);
}

int pg_sync(pg_ctx* c, uint32_t slot) {
  if (!c || slot >= c->slots.size()) return PG_ERR_ARG;
  cudaError_t e = cudaStreamSynchronize(c->slots[slot].stream);
  if (e != cudaSuccess) return cudaFail(c, e, "chain");
  return PG_OK;
}

void* pg_slot_stream(pg_ctx* c, uint32_t slot) {
  if (!c || slot >= c->slots.size()) return nullptr;
  return c->slots[slot].stream;
}

int pg_process_batch(pg_ctx* c, uint32_t nEvents, const uint8_t* const* raws, const size_t* sizes) {
  int rc = pg_stage_batch(c, 0, nEvents, raws, sizes);
  if (rc != PG_OK) return rc;
  rc = pg_run_staged(c, 0);
  if (rc != PG_OK) return rc;
  return pg_sync(c, 0);
}

int pg_event_counts_get(pg_ctx* c, uint32_t k, pg_event_counts* out) {
  if (!c || !out || k >= c->slots[0].nEvents) return PG_ERR_ARG;
  Slot& s = c->slots[0];
  EventCounters ec;
  cudaError_t e = cudaMemcpy(&ec, s.ws.ev + k, sizeof(ec), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cudaFail(c, e, "D2H counters");
  out->n_words = ec.nWords;
  out->n_modules = ec.nModules;
  out->n_digi_errors = ec.nErrors;
  out->n_hits = ec.nHits;
  out->n_cells = ec.nCells;
  out->n_tuples = ec.nTuples;
  out->n_loose = ec.nLoose;
  out->n_vertices = ec.nVertices;
  out->n_cut_margin_doublets = ec.nearDoublet;
  out->n_cut_margin_ca = ec.nearCA;
  out->n_cut_margin_quality = ec.nearQuality;
  out->flags = ec.flags;
  return PG_OK;
}

namespace {
int slotProduct(pg_ctx* c, Slot& s, uint32_t k, const char* name, void* dst, size_t cap, size_t* count, int* elem);
}  // namespace

int pg_get_product(pg_ctx* c, uint32_t k, const char* name, void* dst, size_t cap, size_t* count, int* elem) {
  if (!c || !name || !count || !elem || k >= c->slots[0].nEvents) return PG_ERR_ARG;
  return slotProduct(c, c->slots[0], k, name, dst, cap, count, elem);
}

int pg_slot_product(pg_ctx* c, uint32_t slot, uint32_t k, const char* name, void* dst, size_t cap, size_t* count,
                    int* elem) {
  if (!c || !name || !count || !elem || slot >= c->slots.size()) return PG_ERR_ARG;
  Slot& s = c->slots[slot];
  if (s.state != SlotState::kBusy || k >= s.nEvents) return fail(c, PG_ERR_ARG, "slot holds no such event");
  const cudaError_t q = cudaEventQuery(s.done);
  if (q == cudaErrorNotReady) return PG_ERR_BUSY;
  if (q != cudaSuccess) return cudaFail(c, q, "batch");
  return slotProduct(c, s, k, name, dst, cap, count, elem);
}

namespace {
int slotProduct(pg_ctx* c, Slot& s, uint32_t k, const char* name, void* dst, size_t cap, size_t* count, int* elem) {
  const Workspace& ws = s.ws;
  EventCounters ec;
  cudaError_t e = cudaMemcpy(&ec, ws.ev + k, sizeof(ec), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cudaFail(c, e, "D2H counters");
  std::string n(name);
  const size_t w0 = ec.wordStart, nw = ec.nWords;
  const uint32_t kHitCap = ws.cap.hits, kCellCap = ws.cap.cells, kTupleBins = ws.cap.tuples;
  const uint32_t kTupleHitCap = ws.cap.tupleHits(), kTupleCellCap = ws.cap.tupleCells(), kEdgeCap = ws.cap.edges;
  const size_t hb = size_t(k) * kHitCap, mb = size_t(k) * kModStride, cb = size_t(k) * kCellCap,
               tb = size_t(k) * kTupleBins, vb = size_t(k) * kMaxVtx;
  const uint32_t nh = ec.nHits, nc = ec.nCells;
  if (n == "nDigis" || n == "nModules" || n == "nClusters" || n == "nHits" || n == "nCells" || n == "nTuples" ||
      n == "nVertices" || n == "nNbrLists" || n == "nTrkLists" || n == "nCutMarginDoublets" || n == "nCutMarginCA" ||
      n == "nCutMarginQuality") {
    uint32_t v = n == "nCutMarginDoublets" ? ec.nearDoublet
                 : n == "nCutMarginCA" ? ec.nearCA
                 : n == "nCutMarginQuality" ? ec.nearQuality
                 : n == "nDigis" ? ec.nWords
                 : n == "nModules" ? ec.nModules
                 : (n == "nClusters" || n == "nHits") ? ec.nHits
                 : n == "nCells" ? ec.nCells
                 : n == "nTuples" ? 0u
                 : n == "nVertices" ? ec.nVertices
                 : n == "nNbrLists" ? ec.nNbrLists
                                    : ec.nTrkLists;
    if (n == "nTuples") {
      // number of tuples before the first empty one (the serial loops' guard)
      uint32_t g = ec.nTuples;
      if (ec.apcM >= kTupleBins) g = kTupleBins - 1;
      v = g;
    }
    *elem = 4;
    *count = 1;
    if (dst) {
      if (cap < 4) return PG_ERR_CAPACITY;
      std::memcpy(dst, &v, 4);
    }
    return PG_OK;
  }
  uint32_t nTup = ec.apcM >= kTupleBins ? kTupleBins - 1 : ec.nTuples;
  if (n == "xx") return copyOut(c, s, ws.xx + w0, nw, dst, cap, count, elem);
  if (n == "yy") return copyOut(c, s, ws.yy + w0, nw, dst, cap, count, elem);
  if (n == "adc") return copyOut(c, s, ws.adc + w0, nw, dst, cap, count, elem);
  if (n == "moduleInd") return copyOut(c, s, ws.moduleInd + w0, nw, dst, cap, count, elem);
  if (n == "clus") return copyOut(c, s, ws.clus + w0, nw, dst, cap, count, elem);
  if (n == "pdigi") return copyOut(c, s, ws.pdigi + w0, nw, dst, cap, count, elem);
  if (n == "rawIdArr") return copyOut(c, s, ws.rawIdArr + w0, nw, dst, cap, count, elem);
  if (n == "errors") return copyOut(c, s, ws.errors + size_t(k) * kErrCap, std::min<size_t>(ec.nErrors, kErrCap), dst, cap, count, elem);
  if (n == "formatterErrors" && ws.scan.on) {
    uint32_t cnt = 0;
    e = cudaMemcpy(&cnt, ws.scan.fmtCount + k, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cudaFail(c, e, "D2H formatter error count");
    return copyOut(c, s, ws.scan.fmt + size_t(k) * kFmtErrCap, std::min<size_t>(cnt, kFmtErrCap), dst, cap, count,
                   elem);
  }
  if (n == "formatterErrors") {
    *elem = int(sizeof(PfFormatterError));
    const bool have = k + 1 < s.fmtOff.size();
    const size_t b = have ? s.fmtOff[k] : 0, m = have ? s.fmtOff[k + 1] - s.fmtOff[k] : 0;
    *count = m;
    if (!dst || m == 0) return PG_OK;
    if (m * sizeof(PfFormatterError) > cap) return fail(c, PG_ERR_CAPACITY, "product larger than the destination");
    std::memcpy(dst, s.fmtErrors.data() + b, m * sizeof(PfFormatterError));
    return PG_OK;
  }
  if (n == "moduleStart") return copyOut(c, s, ws.moduleStart + mb, kMaxModules + 1, dst, cap, count, elem);
  if (n == "clusInModule") return copyOut(c, s, ws.clusInModule + mb, kMaxModules, dst, cap, count, elem);
  if (n == "moduleId") return copyOut(c, s, ws.moduleId + mb, kMaxModules, dst, cap, count, elem);
  if (n == "clusModuleStart") return copyOut(c, s, ws.clusModuleStart + mb, kMaxModules + 1, dst, cap, count, elem);
  if (n == "xl") return copyOut(c, s, ws.xl + hb, nh, dst, cap, count, elem);
  if (n == "yl") return copyOut(c, s, ws.yl + hb, nh, dst, cap, count, elem);
  if (n == "xerr") return copyOut(c, s, ws.xerr + hb, nh, dst, cap, count, elem);
  if (n == "yerr") return copyOut(c, s, ws.yerr + hb, nh, dst, cap, count, elem);
  if (n == "xg") return copyOut(c, s, ws.xg + hb, nh, dst, cap, count, elem);
  if (n == "yg") return copyOut(c, s, ws.yg + hb, nh, dst, cap, count, elem);
  if (n == "zg") return copyOut(c, s, ws.zg + hb, nh, dst, cap, count, elem);
  if (n == "rg") return copyOut(c, s, ws.rg + hb, nh, dst, cap, count, elem);
  if (n == "charge") return copyOut(c, s, ws.charge + hb, nh, dst, cap, count, elem);
  if (n == "iphi") return copyOut(c, s, ws.iphi + hb, nh, dst, cap, count, elem);
  if (n == "xsize") return copyOut(c, s, ws.xsize + hb, nh, dst, cap, count, elem);
  if (n == "ysize") return copyOut(c, s, ws.ysize + hb, nh, dst, cap, count, elem);
  if (n == "detInd") return copyOut(c, s, ws.detInd + hb, nh, dst, cap, count, elem);
  if (n == "hitsLayerStart") return copyOut(c, s, &ws.ev[k].layerStart[0], 11, dst, cap, count, elem);
  if (n == "phiOff") return copyOut(c, s, ws.phiOff + size_t(k) * kPhiStride, kPhiTot, dst, cap, count, elem);
  if (n == "phiBins") return copyOut(c, s, ws.phiBins + hb, nh, dst, cap, count, elem);
  if (n == "cellInner") return copyOut(c, s, ws.cellInner + cb, nc, dst, cap, count, elem);
  if (n == "cellOuter") return copyOut(c, s, ws.cellOuter + cb, nc, dst, cap, count, elem);
  if (n == "cellUsed") return copyOut(c, s, ws.cellUsed + cb, nc, dst, cap, count, elem);
  if (n == "cellDoubletId") return copyOut(c, s, ws.cellDoubletId + cb, nc, dst, cap, count, elem);
  if (n == "cellLayerPair") return copyOut(c, s, ws.cellPair + cb, nc, dst, cap, count, elem);
  if (n == "outerHitOffRaw") return copyOut(c, s, ws.ohOff + size_t(k) * (kHitCap + 1), nh + 1, dst, cap, count, elem);
  if (n == "outerHitCellsRaw") {
    // the device orders only lists longer than the 128 the CA reads; the
    // product gives every list in ascending order, as the serial fill does
    int rc = copyOut(c, s, ws.ohCells + cb, nc, dst, cap, count, elem);
    if (rc != PG_OK || !dst || nc == 0) return rc;
    std::vector<uint32_t> off(size_t(nh) + 1);
    cudaError_t e2 = cudaMemcpy(off.data(), ws.ohOff + size_t(k) * (kHitCap + 1), off.size() * 4,
                                cudaMemcpyDeviceToHost);
    if (e2 != cudaSuccess) return cudaFail(c, e2, "D2H outer-hit offsets");
    uint32_t* cells = static_cast<uint32_t*>(dst);
    for (uint32_t h = 0; h < nh; ++h)
      std::sort(cells + std::min<size_t>(off[h], nc), cells + std::min<size_t>(off[h + 1], nc));
    return PG_OK;
  }
  if (n == "cellNbrOffRaw") return copyOut(c, s, ws.nbrOff + size_t(k) * (kCellCap + 1), nc + 1, dst, cap, count, elem);
  if (n == "cellNbrRaw") return copyOut(c, s, ws.nbr + size_t(k) * kEdgeCap, std::min(ec.nEdges, kEdgeCap), dst, cap, count, elem);
  if (n == "cellTrkOffRaw") return copyOut(c, s, ws.trkOff + size_t(k) * (kCellCap + 1), nc + 1, dst, cap, count, elem);
  if (n == "cellTrkRaw") {
    uint32_t tot = 0;
    cudaMemcpy(&tot, ws.trkOff + size_t(k) * (kCellCap + 1) + nc, 4, cudaMemcpyDeviceToHost);
    return copyOut(c, s, ws.trk + size_t(k) * kTupleCellCap, tot, dst, cap, count, elem);
  }
  if (n == "tupleOff") return copyOut(c, s, ws.tupleOff + size_t(k) * (kTupleBins + 1), nTup + 1, dst, cap, count, elem);
  if (n == "tupleHits" || n == "tupleDet") {
    uint32_t tot = 0;
    cudaMemcpy(&tot, ws.tupleOff + size_t(k) * (kTupleBins + 1) + nTup, 4, cudaMemcpyDeviceToHost);
    if (n == "tupleHits") return copyOut(c, s, ws.tupleHits + size_t(k) * kTupleHitCap, tot, dst, cap, count, elem);
    return copyOut(c, s, ws.tupleDet + size_t(k) * kTupleHitCap, tot, dst, cap, count, elem);
  }
  if (n == "quality") return copyOut(c, s, ws.quality + tb, nTup, dst, cap, count, elem);
  if (n == "state") return copyOut(c, s, ws.state + tb * 5, size_t(nTup) * 5, dst, cap, count, elem);
  if (n == "cov") return copyOut(c, s, ws.cov + tb * 15, size_t(nTup) * 15, dst, cap, count, elem);
  if (n == "pt") return copyOut(c, s, ws.pt + tb, nTup, dst, cap, count, elem);
  if (n == "eta") return copyOut(c, s, ws.eta + tb, nTup, dst, cap, count, elem);
  if (n == "chi2") return copyOut(c, s, ws.chi2 + tb, nTup, dst, cap, count, elem);
  if (n == "zv") return copyOut(c, s, ws.zv + vb, ec.nVertices, dst, cap, count, elem);
  if (n == "wv") return copyOut(c, s, ws.wv + vb, ec.nVertices, dst, cap, count, elem);
  if (n == "vchi2") return copyOut(c, s, ws.vchi2 + vb, ec.nVertices, dst, cap, count, elem);
  if (n == "ptv2") return copyOut(c, s, ws.ptv2 + vb, ec.nVertices, dst, cap, count, elem);
  if (n == "ndof") return copyOut(c, s, ws.ndof + vb, ec.nVertices, dst, cap, count, elem);
  if (n == "sortInd") return copyOut(c, s, ws.sortInd + vb, ec.nVertices, dst, cap, count, elem);
  if (n == "idv") return copyOut(c, s, ws.idv + tb, nTup, dst, cap, count, elem);
  return fail(c, PG_ERR_NOTFOUND, "unknown product " + n);
}
}  // namespace

int pg_submit(pg_ctx* c, uint32_t nEvents, const uint8_t* const* raws, const size_t* sizes, uint32_t* slotOut) {
  if (!c || !raws || !sizes || !slotOut) return PG_ERR_ARG;
  cudaSetDevice(c->cfg.device);
  int k;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    k = findFreeSlot(c);
    if (k < 0) return fail(c, PG_ERR_BUSY, "no free slot");
    c->slots[k].state = SlotState::kBusy;
  }
  Slot& s = c->slots[k];
  int rc = stage(c, s, nEvents, raws, sizes);
  if (rc == PG_OK) rc = launchBatch(c, s);
  if (rc != PG_OK) {
    cudaStreamSynchronize(s.stream);
    s.state = SlotState::kFree;
    return rc;
  }
  *slotOut = uint32_t(k);
  return PG_OK;
}

int pg_query(pg_ctx* c, uint32_t slot) {
  if (!c || slot >= c->slots.size() || c->slots[slot].state != SlotState::kBusy) return PG_ERR_ARG;
  cudaError_t e = cudaEventQuery(c->slots[slot].done);
  if (e == cudaErrorNotReady) return PG_ERR_BUSY;
  if (e != cudaSuccess) return cudaFail(c, e, "batch");
  return PG_OK;
}

int pg_wait(pg_ctx* c, uint32_t slot) {
  if (!c || slot >= c->slots.size() || c->slots[slot].state != SlotState::kBusy) return PG_ERR_ARG;
  cudaError_t e = cudaEventSynchronize(c->slots[slot].done);
  if (e != cudaSuccess) return cudaFail(c, e, "batch");
  return PG_OK;
}

int pg_result(pg_ctx* c, uint32_t slot, uint32_t k, pg_result_view* v) {
  if (!c || !v || slot >= c->slots.size()) return PG_ERR_ARG;
  Slot& s = c->slots[slot];
  if (s.state != SlotState::kBusy || k >= s.nEvents) return PG_ERR_ARG;
  if (cudaEventQuery(s.done) != cudaSuccess) return fail(c, PG_ERR_BUSY, "batch not finished");
  uint8_t* base = s.hRes + size_t(k) * kResultStride;
  const ResultHeader* h = reinterpret_cast<const ResultHeader*>(base);
  ResultTracks t = resultTracks(base);
  ResultVertices vx = resultVertices(base);
  v->n_tracks = h->nTracks;
  v->n_loose_all = h->nLooseAll;
  v->n_vertices = h->nVertices;
  v->n_hits = h->nHits;
  v->n_tuples = h->nTuples;
  v->n_digis = h->nDigis;
  v->n_cells = h->nCells;
  v->flags = h->flags;
  v->tuple_index = t.tupleIndex;
  v->track_n_hits = t.nHits;
  v->quality = t.quality;
  v->state = t.state;
  v->cov = t.cov;
  v->pt = t.pt;
  v->eta = t.eta;
  v->chi2 = t.chi2;
  v->hits = t.hits;
  v->vertex = t.vertex;
  v->zv = vx.zv;
  v->wv = vx.wv;
  v->vchi2 = vx.chi2;
  v->ptv2 = vx.ptv2;
  v->ndof = vx.ndof;
  v->sort_ind = vx.sortInd;
  return PG_OK;
}

int pg_batch_summary_get(pg_ctx* c, uint32_t slot, pg_batch_summary* out) {
  if (!c || !out || slot >= c->slots.size()) return PG_ERR_ARG;
  Slot& s = c->slots[slot];
  if (s.state != SlotState::kBusy) return PG_ERR_ARG;
  if (cudaEventQuery(s.done) != cudaSuccess) return fail(c, PG_ERR_BUSY, "batch not finished");
  *out = pg_batch_summary{};
  out->n_events = s.nEvents;
  for (uint32_t k = 0; k < s.nEvents; ++k) {
    const ResultHeader* h = reinterpret_cast<const ResultHeader*>(s.hRes + size_t(k) * kResultStride);
    out->flags |= h->flags;
    out->n_tracks += h->nTracks;
    out->n_vertices += h->nVertices;
    out->result_bytes += sizeof(ResultHeader) + h->nTracks * kResultTrackBytes + h->nVertices * kResultVertexBytes;
    out->n_digis += h->nDigis;
    out->n_modules += h->nModules;
    out->n_hits += h->nHits;
    out->n_cells += h->nCells;
    out->n_edges += h->nEdges;
    out->n_tuples += h->nTuples;
    out->n_tuple_hits += h->nTupleHits;
    out->n_cut_margin += uint64_t(h->nearDoublet) + h->nearCA + h->nearQuality;
    out->n_flagged_events += (h->flags & ~kFlagResultOverflow) ? 1 : 0;
  }
  return PG_OK;
}

int pg_release(pg_ctx* c, uint32_t slot) {
  if (!c || slot >= c->slots.size()) return PG_ERR_ARG;
  Slot& s = c->slots[slot];
  if (s.state != SlotState::kBusy) return PG_ERR_ARG;
  cudaError_t e = cudaEventSynchronize(s.done);
  poolReclaimSlot(c, s);
  std::lock_guard<std::mutex> lk(c->mu);
  s.state = SlotState::kFree;
  if (e != cudaSuccess) return cudaFail(c, e, "batch");
  return PG_OK;
}

int pg_set_probe(pg_ctx* c, const char* kernel) {
  if (!c) return PG_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  for (auto& s : c->slots)
    if (s.state != SlotState::kFree) return fail(c, PG_ERR_BUSY, "pg_set_probe needs every slot free");
  std::string name = kernel ? kernel : "";
  if (name.size() >= sizeof(KernelProbe::name)) return fail(c, PG_ERR_ARG, "kernel name too long");
  cudaSetDevice(c->cfg.device);
  for (auto& s : c->slots) {
    cudaStreamSynchronize(s.stream);
    for (auto& g : s.graphs) cudaGraphExecDestroy(g.second);
    s.graphs.clear();
    s.probeUsed.clear();
    s.lastProbeUsed = 0;
    if (!name.empty() && !s.probe) {
      s.probe = new KernelProbe();
      std::memset(s.probe, 0, sizeof(KernelProbe));
      for (auto& ev : s.probe->ev)
        if (cudaEventCreate(&ev) != cudaSuccess) return fail(c, PG_ERR_CUDA, "probe events");
    }
    if (s.probe) std::snprintf(s.probe->name, sizeof(s.probe->name), "%s", name.c_str());
  }
  c->probeName = name;
  return PG_OK;
}

int pg_probe_read(pg_ctx* c, uint32_t slot, uint32_t max, pg_probe_entry* out, uint32_t* n) {
  if (!c || !n || slot >= c->slots.size()) return PG_ERR_ARG;
  Slot& s = c->slots[slot];
  *n = 0;
  if (c->probeName.empty() || !s.probe) return PG_OK;
  cudaError_t e = cudaEventQuery(s.done);
  if (e == cudaErrorNotReady) return fail(c, PG_ERR_BUSY, "batch not finished");
  if (e != cudaSuccess) return cudaFail(c, e, "batch");
  uint32_t k = std::min(s.lastProbeUsed, max);
  for (uint32_t i = 0; i < k; ++i) {
    float ms = 0;
    e = cudaEventElapsedTime(&ms, s.probe->ev[2 * i], s.probe->ev[2 * i + 1]);
    if (e != cudaSuccess) return cudaFail(c, e, "probe elapsed time");
    if (out) {
      out[i].kernel = s.probe->launched[i];
      out[i].ms = ms;
    }
  }
  *n = k;
  return PG_OK;
}

int pg_fit_broken_line(pg_ctx* c, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                       float* cov, float* pt, float* eta, float* chi2, void* stream) {
  if (!c || (N != 3 && N != 4)) return PG_ERR_ARG;
  cudaError_t e = fitDirect(N, n, hits, ge, B, state, cov, pt, eta, chi2, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cudaFail(c, e, "fit launch");
  return PG_OK;
}

int pg_fit_broken_line_mixed(pg_ctx* c, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                       float* cov, float* pt, float* eta, float* chi2, void* stream) {
  if (!c || (N != 3 && N != 4)) return PG_ERR_ARG;
  cudaError_t e = fitDirectMixed(N, n, hits, ge, B, state, cov, pt, eta, chi2, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cudaFail(c, e, "fit launch");
  return PG_OK;
}

int pg_fit_riemann(pg_ctx* c, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                   float* cov, float* pt, float* eta, float* chi2, void* stream) {
  if (!c || (N != 3 && N != 4)) return PG_ERR_ARG;
  cudaError_t e =
      fitDirectRiemann(N, n, hits, ge, B, state, cov, pt, eta, chi2, false, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cudaFail(c, e, "fit launch");
  return PG_OK;
}

int pg_fit_riemann_mixed(pg_ctx* c, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                         float* cov, float* pt, float* eta, float* chi2, void* stream) {
  if (!c || (N != 3 && N != 4)) return PG_ERR_ARG;
  cudaError_t e =
      fitDirectRiemann(N, n, hits, ge, B, state, cov, pt, eta, chi2, true, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cudaFail(c, e, "fit launch");
  return PG_OK;
}

}  // extern "C"
