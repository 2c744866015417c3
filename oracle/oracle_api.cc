// C entry points of the oracle library (checker only; see oracle.h).
// Products are exposed by name with the same names the checker build of the
// reference (oracle/ref/ref_driver.cc) uses, so tests compare them directly.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

struct Blob {
  std::vector<uint8_t> bytes;
  int elem = 1;
};

struct Handle {
  oracle::ES es;
  oracle::Event ev;
  std::map<std::string, Blob> out;
  double lastSeconds = 0;
  oracle::Options opts;
  std::string error;

  template <typename T>
  void put(const std::string& name, const T* p, size_t n) {
    Blob b;
    b.elem = sizeof(T);
    b.bytes.resize(n * sizeof(T));
    if (n) std::memcpy(b.bytes.data(), p, n * sizeof(T));
    out[name] = std::move(b);
  }
  template <typename T>
  void put1(const std::string& name, T v) {
    put(name, &v, 1);
  }
};

void record(Handle& h) {
  auto& d = h.ev.digis;
  auto& c = h.ev.clusters;
  auto& hi = h.ev.hits;
  auto& ca = h.ev.ca;
  auto& v = h.ev.vtx;
  h.out.clear();
  // the FED loop's word stream (WordFedAppender): words and one FED index per word pair
  h.put("fedWords", h.ev.words.word.data(), h.ev.words.nWords);
  h.put("fedWordFedIds", h.ev.words.fedId.data(), (h.ev.words.nWords + 1) / 2);
  h.put1<uint32_t>("nDigis", d.nDigis);
  h.put1<uint32_t>("nModules", d.nModules);
  h.put("xx", d.xx.data(), d.nDigis);
  h.put("yy", d.yy.data(), d.nDigis);
  h.put("adc", d.adc.data(), d.nDigis);
  h.put("moduleInd", d.moduleInd.data(), d.nDigis);
  h.put("clus", d.clus.data(), d.nDigis);
  h.put("pdigi", d.pdigi.data(), d.nDigis);
  h.put("rawIdArr", d.rawIdArr.data(), d.nDigis);
  h.put("errors", d.errors.data(), d.errors.size());
  h.put("formatterErrors", h.ev.words.formatterErrors.data(), h.ev.words.formatterErrors.size());
  h.put1<uint32_t>("nClusters", c.nClusters);
  h.put("moduleStart", c.moduleStart.data(), c.moduleStart.size());
  h.put("clusInModule", c.clusInModule.data(), c.clusInModule.size());
  h.put("moduleId", c.moduleId.data(), c.moduleId.size());
  h.put("clusModuleStart", c.clusModuleStart.data(), c.clusModuleStart.size());
  uint32_t nh = hi.nHits;
  h.put1<uint32_t>("nHits", nh);
  h.put("xl", hi.xl.data(), nh);
  h.put("yl", hi.yl.data(), nh);
  h.put("xerr", hi.xerr.data(), nh);
  h.put("yerr", hi.yerr.data(), nh);
  h.put("xg", hi.xg.data(), nh);
  h.put("yg", hi.yg.data(), nh);
  h.put("zg", hi.zg.data(), nh);
  h.put("rg", hi.rg.data(), nh);
  h.put("charge", hi.charge.data(), nh);
  h.put("iphi", hi.iphi.data(), nh);
  h.put("xsize", hi.xsize.data(), nh);
  h.put("ysize", hi.ysize.data(), nh);
  h.put("detInd", hi.detInd.data(), nh);
  if (nh) {
    h.put("hitsLayerStart", hi.layerStart, 11);
    h.put("phiOff", hi.phiOff.data(), hi.phiOff.size());
    h.put("phiBins", hi.phiBins.data(), nh);
  }
  h.put("agcLadderR", hi.agc.ladderR, PF_N_LADDERS_BARREL);
  // CA internals
  h.put1<uint32_t>("nCells", ca.nCells);
  h.put("cellInner", ca.inner.data(), ca.nCells);
  h.put("cellOuter", ca.outer.data(), ca.nCells);
  h.put("cellLayerPair", ca.layerPair.data(), ca.nCells);
  h.put("cellDoubletId", ca.doubletId.data(), ca.nCells);
  h.put("cellUsed", ca.used.data(), ca.nCells);
  {
    std::vector<uint32_t> off(1, 0), val, toff(1, 0);
    std::vector<uint32_t> tval;
    for (uint32_t c2 = 0; c2 < ca.nCells; ++c2) {
      for (auto x : ca.nbr[c2]) val.push_back(x);
      off.push_back(uint32_t(val.size()));
      for (auto x : ca.trk[c2]) tval.push_back(x);
      toff.push_back(uint32_t(tval.size()));
    }
    h.put("cellNbrOff", off.data(), off.size());
    h.put("cellNbr", val.data(), val.size());
    h.put("cellTrkOff", toff.data(), toff.size());
    h.put("cellTrk", tval.data(), tval.size());
    std::vector<uint32_t> ooff(1, 0), oval;
    if (nh)
      for (uint32_t i = 0; i < nh; ++i) {
        for (auto x : ca.outerHitCells[i]) oval.push_back(x);
        ooff.push_back(uint32_t(oval.size()));
      }
    h.put("outerHitOff", ooff.data(), ooff.size());
    h.put("outerHitCells", oval.data(), oval.size());
    h.put1<int32_t>("nNbrLists", ca.nbrPool);
    h.put1<int32_t>("nTrkLists", ca.trkPool);
  }
  uint32_t nt = 0;
  while (nt < ca.tupleBins && ca.size(nt) > 0) ++nt;
  h.put1<uint32_t>("nTuples", nt);
  h.put("tupleOff", ca.tupleOff.data(), nt + 1);
  h.put("tupleHits", ca.tupleHits.data(), ca.tupleOff[nt]);
  h.put("tupleDet", ca.tupleDet.data(), ca.tupleOff[nt]);
  h.put("quality", ca.quality.data(), nt);
  h.put("state", ca.state.data(), size_t(nt) * 5);
  h.put("cov", ca.cov.data(), size_t(nt) * 15);
  h.put("pt", ca.pt.data(), nt);
  h.put("eta", ca.eta.data(), nt);
  h.put("chi2", ca.chi2.data(), nt);
  h.put1<uint32_t>("nCutMarginDoublets", ca.nearDoublet);
  h.put1<uint32_t>("nCutMarginCA", ca.nearCA);
  h.put1<uint32_t>("nCutMarginQuality", ca.nearQuality);
  h.put1<uint32_t>("nVertices", v.nvFinal);
  h.put("zv", v.zv.data(), v.nvFinal);
  h.put("wv", v.wv.data(), v.nvFinal);
  h.put("vchi2", v.chi2.data(), v.nvFinal);
  h.put("ptv2", v.ptv2.data(), v.nvFinal);
  h.put("ndof", v.ndof.data(), v.nvFinal);
  h.put("sortInd", v.sortInd.data(), v.nvFinal);
  h.put("idv", v.idv.data(), nt);
}

}  // namespace

namespace oracle {
void processEvent(const ES& es, const uint8_t* raw, size_t n, Event& ev, const Options& o) {
  fedLoop(es, raw, n, ev.words, o.formatterErrors, o.ca.caps);
  makeClusters(es, ev.words, ev.digis, ev.clusters, o.ca.caps);
  makeHits(es, ev.digis, ev.clusters, ev.hits, o.ca.caps);
  makeTuples(es, ev.hits, ev.ca, o.ca);
  makeVertices(ev.ca, ev.vtx, o.vertexAlgo);
}
}  // namespace oracle

extern "C" {

// ES records are the file images of cablingMap.bin, gain.bin, cpefast.bin,
// beamspot.bin and fedIds.bin.  Returns nullptr on malformed input.
void* or_create(const uint8_t* cabling, size_t ncab, const uint8_t* gain, size_t ngain, const uint8_t* cpe,
                size_t ncpe, const uint8_t* bs, size_t nbs, const uint8_t* fedids, size_t nfed) {
  auto h = new Handle();
  try {
    oracle::loadES(h->es, cabling, ncab, gain, ngain, cpe, ncpe, bs, nbs, fedids, nfed);
  } catch (std::exception&) {
    delete h;
    return nullptr;
  }
  return h;
}

void or_destroy(void* p) { delete static_cast<Handle*>(p); }

// useRiemannFit of the CA module configuration (off by default, as in the reference)
void or_set_riemann(void* p, int on) { static_cast<Handle*>(p)->opts.ca.useRiemannFit = on != 0; }

// the CA module's switches (CAHitNtupletGeneratorOnGPU.cc:46-58); -1 when
// minHitsPerNtuplet is outside 3..4
int or_set_ca_params(void* p, int minHitsPerNtuplet, int includeJumpingForwardDoublets, int earlyFishbone,
                     int lateFishbone, int idealConditions, int doClusterCut, int doZ0Cut, int doPtCut) {
  if (minHitsPerNtuplet < 3 || minHitsPerNtuplet > 4) return -1;
  auto& c = static_cast<Handle*>(p)->opts.ca;
  c.minHitsPerNtuplet = uint32_t(minHitsPerNtuplet);
  c.includeJumpingForwardDoublets = includeJumpingForwardDoublets != 0;
  c.earlyFishbone = earlyFishbone != 0;
  c.lateFishbone = lateFishbone != 0;
  c.idealConditions = idealConditions != 0;
  c.doClusterCut = doClusterCut != 0;
  c.doZ0Cut = doZ0Cut != 0;
  c.doPtCut = doPtCut != 0;
  return 0;
}

// container capacities (oracle::Caps; the reference's values by default).
// Zero leaves a field unchanged; -1 when a capacity is below the reference's
// (smaller containers would change results the reference defines).
int or_set_caps(void* p, uint32_t fedWords, uint32_t hits, uint32_t doublets, uint32_t lists, uint32_t tuples,
                uint32_t multiplicity, uint32_t hitToTuple) {
  oracle::Caps c = static_cast<Handle*>(p)->opts.ca.caps;
  if (fedWords) c.fedWords = fedWords;
  if (hits) c.hits = hits;
  if (doublets) c.doublets = doublets;
  if (lists) c.lists = lists;
  if (tuples) c.tuples = tuples;
  if (multiplicity) c.multiplicity = multiplicity;
  if (hitToTuple) c.hitToTuple = hitToTuple;
  const oracle::Caps d;
  if (c.fedWords < d.fedWords || c.hits < d.hits || c.doublets < d.doublets || c.lists < d.lists ||
      c.tuples < d.tuples || c.multiplicity < d.multiplicity || c.hitToTuple < d.hitToTuple)
    return -1;
  static_cast<Handle*>(p)->opts.ca.caps = c;
  return 0;
}

// vertex clustering of PixelVertexProducerCUDA: 0 density (default), 1 DBSCAN, 2 iterative
int or_set_vertex_algo(void* p, int algo) {
  if (algo < 0 || algo > 2) return -1;
  static_cast<Handle*>(p)->opts.vertexAlgo = algo;
  return 0;
}

// the ErrorChecker's includeErrors: record the FED loop's framing errors
// (off in the reference, ErrorChecker.cc:36)
void or_set_formatter_errors(void* p, int on) { static_cast<Handle*>(p)->opts.formatterErrors = on != 0; }

// Runs the chain on one raw.bin event record; 0 on success.
int or_process(void* p, const uint8_t* raw, size_t n) {
  Handle& h = *static_cast<Handle*>(p);
  try {
    auto t0 = std::chrono::steady_clock::now();
    oracle::processEvent(h.es, raw, n, h.ev, h.opts);
    auto t1 = std::chrono::steady_clock::now();
    h.lastSeconds = std::chrono::duration<double>(t1 - t0).count();
    record(h);
  } catch (std::exception& e) {
    h.error = e.what();
    return -1;
  }
  return 0;
}

int or_get(void* p, const char* name, const void** data, size_t* count, int* elem) {
  Handle& h = *static_cast<Handle*>(p);
  auto it = h.out.find(name);
  if (it == h.out.end()) return -1;
  *data = it->second.bytes.data();
  *elem = it->second.elem;
  *count = it->second.bytes.size() / size_t(it->second.elem);
  return 0;
}

double or_last_seconds(void* p) { return static_cast<Handle*>(p)->lastSeconds; }

// Times the chain (FED loop to vertices) over n event records on `threads`
// host threads, one event per thread at a time (the reference's event-level
// parallelism).  Writes per-event seconds into lat[n] (may be null) and
// returns the wall time in seconds, or a negative value on error.
double or_time_events(void* p, const uint8_t* const* raws, const size_t* sizes, int n, int threads, double* lat) {
  Handle& h = *static_cast<Handle*>(p);
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  std::atomic<int> next{0};
  std::atomic<int> failed{0};
  auto t0 = std::chrono::steady_clock::now();
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&]() {
      oracle::Event ev;
      for (;;) {
        int k = next.fetch_add(1);
        if (k >= n) break;
        auto a = std::chrono::steady_clock::now();
        try {
          oracle::processEvent(h.es, raws[k], sizes[k], ev, h.opts);
        } catch (std::exception&) {
          failed++;
        }
        auto b = std::chrono::steady_clock::now();
        if (lat) lat[k] = std::chrono::duration<double>(b - a).count();
      }
    });
  }
  for (auto& th : pool) th.join();
  auto t1 = std::chrono::steady_clock::now();
  if (failed) return -1.0;
  return std::chrono::duration<double>(t1 - t0).count();
}

// Broken-line fit of n tuples of N (3 or 4) hits: hits[(t*N+i)*3+k] (x,y,z),
// ge[(t*N+i)*6+k]; outputs state[t*5+k], cov[t*15+k], pt/eta/chi2[t].
int or_fit(int N, uint32_t n, const double* hits, const float* ge, double B, float* state, float* cov, float* pt,
           float* eta, float* chi2) {
  if (N != 3 && N != 4) return -1;
  for (uint32_t t = 0; t < n; ++t)
    oracle::brokenLineFit(N, hits + size_t(t) * N * 3, ge + size_t(t) * N * 6, B, state + size_t(t) * 5,
                          cov + size_t(t) * 15, pt + t, eta + t, chi2 + t);
  return 0;
}

// Riemann fit of n tuples, same layout as or_fit.
int or_fit_riemann(int N, uint32_t n, const double* hits, const float* ge, double B, float* state, float* cov,
                   float* pt, float* eta, float* chi2) {
  if (N != 3 && N != 4) return -1;
  for (uint32_t t = 0; t < n; ++t)
    oracle::riemannFit(N, hits + size_t(t) * N * 3, ge + size_t(t) * N * 6, B, state + size_t(t) * 5,
                       cov + size_t(t) * 15, pt + t, eta + t, chi2 + t);
  return 0;
}

// Clustering of given digis (module index, row, column, calibrated charge):
// moduleIndOut/clus per digi, clusInModule/moduleId per module (2000),
// moduleStart (2001), the module-run count; -1 where the reference's result
// is undefined (a module's digis in two runs).
int or_cluster_digis(uint32_t n, const uint16_t* moduleInd, const uint16_t* xx, const uint16_t* yy,
                     const uint16_t* adc, uint16_t* moduleIndOut, int32_t* clus, uint32_t* clusInModule,
                     uint32_t* moduleId, uint32_t* moduleStart, uint32_t* nModules) {
  oracle::Digis d;
  oracle::Clusters c;
  d.nDigis = n;
  d.xx.assign(xx, xx + n);
  d.yy.assign(yy, yy + n);
  d.adc.assign(adc, adc + n);
  d.moduleInd.assign(moduleInd, moduleInd + n);
  d.clus.assign(n, 0);
  try {
    oracle::clusterDigis(d, c);
  } catch (std::exception&) {
    return -1;
  }
  std::copy(d.moduleInd.begin(), d.moduleInd.end(), moduleIndOut);
  std::copy(d.clus.begin(), d.clus.end(), clus);
  std::copy(c.clusInModule.begin(), c.clusInModule.end(), clusInModule);
  std::copy(c.moduleId.begin(), c.moduleId.end(), moduleId);
  std::copy(c.moduleStart.begin(), c.moduleStart.end(), moduleStart);
  *nModules = d.nModules;
  return 0;
}

// Vertexing of a given track SoA (n tuples): tuple_off[n+1], quality[n],
// pt[n], state[n*5], cov[n*15]; outputs idv[n], zv/wv/chi2/ptv2/ndof/sortInd
// (1024 each) and the vertex count.  Test infrastructure for the vertex
// finder run on tracks that do not come from an event.
int or_vertices(uint32_t n, const uint32_t* tupleOff, const uint8_t* quality, const float* pt, const float* state,
                const float* cov, int16_t* idv, float* zv, float* wv, float* chi2, float* ptv2, int32_t* ndof,
                uint16_t* sortInd, uint32_t* nVertices) {
  if (n >= PF_TRACK_STRIDE) return -1;
  oracle::CA ca;
  ca.tupleOff.assign(PF_TRACK_STRIDE + 1, tupleOff[n]);
  std::copy(tupleOff, tupleOff + n + 1, ca.tupleOff.begin());
  ca.quality.assign(PF_TRACK_STRIDE, 0);
  std::copy(quality, quality + n, ca.quality.begin());
  ca.pt.assign(PF_TRACK_STRIDE, 0.f);
  std::copy(pt, pt + n, ca.pt.begin());
  ca.state.assign(size_t(PF_TRACK_STRIDE) * 5, 0.f);
  std::copy(state, state + size_t(n) * 5, ca.state.begin());
  ca.cov.assign(size_t(PF_TRACK_STRIDE) * 15, 0.f);
  std::copy(cov, cov + size_t(n) * 15, ca.cov.begin());
  oracle::Vertices v;
  try {
    oracle::makeVertices(ca, v);
  } catch (std::exception&) {
    return -1;
  }
  std::copy(v.idv.begin(), v.idv.begin() + n, idv);
  std::copy(v.zv.begin(), v.zv.begin() + 1024, zv);
  std::copy(v.wv.begin(), v.wv.begin() + 1024, wv);
  std::copy(v.chi2.begin(), v.chi2.begin() + 1024, chi2);
  std::copy(v.ptv2.begin(), v.ptv2.begin() + 1024, ptv2);
  std::copy(v.ndof.begin(), v.ndof.begin() + 1024, ndof);
  std::copy(v.sortInd.begin(), v.sortInd.begin() + 1024, sortInd);
  *nVertices = v.nvFinal;
  return 0;
}

}  // extern "C"
