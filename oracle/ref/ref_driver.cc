// Checker-only driver that runs the reference's own serial pixel chain (the
// unmodified src/serial sources, compiled in place) on one raw.bin event and
// exposes every product and CA internal by name.  It replaces the TBB
// framework (EventProcessor/Worker) with a plain per-event call sequence:
//   SiPixelRawToClusterCUDA::produce   (plugin-SiPixelClusterizer/SiPixelRawToClusterCUDA.cc:60-158)
//   SiPixelRecHitCUDA::produce         (plugin-SiPixelRecHits/SiPixelRecHitCUDA.cc:37-50)
//   CAHitNtupletCUDA::produce          (plugin-PixelTriplets/CAHitNtupletCUDA.cc:30-36,
//                                       body of CAHitNtupletGeneratorOnGPU::makeTuples :96-126)
//   PixelVertexProducerCUDA::produce   (plugin-PixelVertexFinding/PixelVertexProducerCUDA.cc:42-62)
// with the module configuration of those constructors.  ES records are read
// exactly as the ESProducers read them.  This file is test infrastructure:
// it is linked only into oracle/_ref and never into the product.
#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <set>
#include <sstream>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>
#include <bitset>
#include <typeindex>
#include <stdexcept>
#include <iomanip>
#include <chrono>
#include <thread>

#include "Eigen/Core"

// CA internals (cells, neighbour and track lists) are private members of the
// reference's kernel classes; the checker reads them for the doublet/ntuplet
// parity fixtures.
#define private public
#define protected public
#include "plugin-PixelTriplets/CAHitNtupletGeneratorOnGPU.h"
#include "plugin-PixelTriplets/CAHitNtupletGeneratorKernels.h"
#include "plugin-PixelTriplets/GPUCACell.h"
// and the ErrorChecker's includeErrors switch
#include "plugin-SiPixelClusterizer/ErrorChecker.h"
#undef private
#undef protected

#include "CUDADataFormats/SiPixelClustersSoA.h"
#include "CUDADataFormats/SiPixelDigisSoA.h"
#include "CUDADataFormats/SiPixelDigiErrorsSoA.h"
#include "CUDADataFormats/TrackingRecHit2DHeterogeneous.h"
#include "CUDADataFormats/PixelTrackHeterogeneous.h"
#include "CUDADataFormats/ZVertexHeterogeneous.h"
#include "CondFormats/SiPixelGainCalibrationForHLTGPU.h"
#include "CondFormats/SiPixelGainForHLTonGPU.h"
#include "CondFormats/SiPixelFedCablingMapGPUWrapper.h"
#include "CondFormats/SiPixelFedIds.h"
#include "CondFormats/PixelCPEFast.h"
#include "DataFormats/BeamSpotPOD.h"
#include "DataFormats/FEDRawData.h"
#include "DataFormats/FEDRawDataCollection.h"
#include "DataFormats/PixelErrors.h"
#include "Framework/ProductRegistry.h"
#include "plugin-SiPixelClusterizer/SiPixelRawToClusterGPUKernel.h"
#include "plugin-SiPixelRecHits/PixelRecHits.h"
#include "plugin-PixelVertexFinding/gpuVertexFinder.h"
#include "plugin-PixelTriplets/RiemannFit.h"

namespace {

struct Blob {
  std::vector<uint8_t> bytes;
  int elem = 1;
};

struct RefChain {
  std::vector<unsigned int> fedIds;
  std::unique_ptr<SiPixelFedCablingMapGPUWrapper> cabling;
  std::unique_ptr<SiPixelGainCalibrationForHLTGPU> gains;
  std::unique_ptr<PixelCPEFast> cpe;
  BeamSpotPOD bs;
  edm::ProductRegistry reg;
  std::unique_ptr<CAHitNtupletGeneratorOnGPU> caGen;
  std::unique_ptr<gpuVertexFinder::Producer> vtx;
  std::unique_ptr<pixelgpudetails::SiPixelRawToClusterGPUKernel::WordFedAppender> appender;
  std::map<std::string, Blob> out;
  double lastSeconds = 0;
  // the fit choice of a configuration with useRiemannFit=true; the
  // reference's own configuration fixes it to false
  // (CAHitNtupletGeneratorOnGPU.cc:49)
  bool useRiemannFit = false;
  // the ErrorChecker's includeErrors (false in ErrorChecker.cc:36)
  bool formatterErrors = false;
  // the CA module's switches when set through pr_set_ca_params; otherwise
  // the reference's own configuration (caGen->m_params)
  std::unique_ptr<cAHitNtupletGenerator::Params> caParams;
  const cAHitNtupletGenerator::Params& params() const { return caParams ? *caParams : caGen->m_params; }

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

template <typename T>
void readPod(std::ifstream& in, T& x) {
  in.read(reinterpret_cast<char*>(&x), sizeof(T));
}

}  // namespace

extern "C" {

void* pr_create(const char* datadir) {
  namespace fs = std::filesystem;
  auto h = std::make_unique<RefChain>();
  fs::path dir(datadir);
  {
    // SiPixelFedCablingMapGPUWrapperESProducer::produce (:20-41)
    std::ifstream in(dir / "fedIds.bin", std::ios::binary);
    in.exceptions(std::ifstream::badbit | std::ifstream::failbit | std::ifstream::eofbit);
    unsigned int nfeds;
    readPod(in, nfeds);
    h->fedIds.resize(nfeds);
    in.read(reinterpret_cast<char*>(h->fedIds.data()), sizeof(unsigned int) * nfeds);
  }
  {
    std::ifstream in(dir / "cablingMap.bin", std::ios::binary);
    in.exceptions(std::ifstream::badbit | std::ifstream::failbit | std::ifstream::eofbit);
    auto obj = std::make_unique<SiPixelFedCablingMapGPU>();
    in.read(reinterpret_cast<char*>(obj.get()), sizeof(SiPixelFedCablingMapGPU));
    unsigned int n;
    readPod(in, n);
    std::vector<unsigned char> modToUnp(n);
    in.read(reinterpret_cast<char*>(modToUnp.data()), n);
    h->cabling = std::make_unique<SiPixelFedCablingMapGPUWrapper>(*obj, std::move(modToUnp));
  }
  {
    // SiPixelGainCalibrationForHLTGPUESProducer::produce (:20-30)
    std::ifstream in(dir / "gain.bin", std::ios::binary);
    in.exceptions(std::ifstream::badbit | std::ifstream::failbit | std::ifstream::eofbit);
    SiPixelGainForHLTonGPU gain;
    in.read(reinterpret_cast<char*>(&gain), sizeof(SiPixelGainForHLTonGPU));
    unsigned int nbytes;
    readPod(in, nbytes);
    std::vector<char> data(nbytes);
    in.read(data.data(), nbytes);
    h->gains = std::make_unique<SiPixelGainCalibrationForHLTGPU>(gain, std::move(data));
  }
  h->cpe = std::make_unique<PixelCPEFast>((dir / "cpefast.bin").string());
  {
    std::ifstream in(dir / "beamspot.bin", std::ios::binary);
    in.exceptions(std::ifstream::badbit | std::ifstream::failbit | std::ifstream::eofbit);
    readPod(in, h->bs);
  }
  h->caGen = std::make_unique<CAHitNtupletGeneratorOnGPU>(h->reg);
  // PixelVertexProducerCUDA ctor (:16-26)
  h->vtx = std::make_unique<gpuVertexFinder::Producer>(true, true, false, false, 2, 0.07, 0.01, 9);
  h->appender = std::make_unique<pixelgpudetails::SiPixelRawToClusterGPUKernel::WordFedAppender>();
  return h.release();
}

void pr_destroy(void* p) { delete static_cast<RefChain*>(p); }

// Runs the chain on one raw.bin event record.  dump != 0 also records
// the CA internals.  Returns 0 on success.
int pr_process(void* p, const uint8_t* raw, size_t nraw, int dump) {
  RefChain& h = *static_cast<RefChain*>(p);
  h.out.clear();
  // Source::readRaw (bin/Source.cc:9-21)
  FEDRawDataCollection buffers;
  {
    size_t off = 0;
    auto rd = [&](void* dst, size_t n) {
      if (off + n > nraw) throw std::runtime_error("truncated raw record");
      std::memcpy(dst, raw + off, n);
      off += n;
    };
    unsigned int nfeds;
    rd(&nfeds, 4);
    for (unsigned i = 0; i < nfeds; ++i) {
      unsigned int fedId, size;
      rd(&fedId, 4);
      rd(&size, 4);
      FEDRawData& d = buffers.FEDData(fedId);
      d.resize(size);
      rd(d.data(), size);
    }
  }
  auto t0 = std::chrono::steady_clock::now();

  // ---- SiPixelRawToClusterCUDA::produce, host part (:60-138)
  const bool isRun2 = true, includeErrors = true, useQuality = true;
  const auto* gpuMap = h.cabling->getCPUProduct();
  const unsigned char* modToUnp = h.cabling->getModToUnpAll();
  const auto* gpuGains = h.gains->getCPUProduct();
  PixelFormatterErrors errors;
  unsigned int wordCounterGPU = 0, fedCounter = 0;
  bool errorsInEvent = false;
  ErrorChecker errorcheck;
  errorcheck.includeErrors = h.formatterErrors;
  for (int fedId : h.fedIds) {
    if (fedId == 40) continue;
    assert(fedId >= 1200);
    fedCounter++;
    const FEDRawData& rawData = buffers.FEDData(fedId);
    int nWords = rawData.size() / sizeof(uint64_t);
    if (nWords == 0) continue;
    const uint64_t* trailer = reinterpret_cast<const uint64_t*>(rawData.data()) + (nWords - 1);
    if (not errorcheck.checkCRC(errorsInEvent, fedId, trailer, errors)) continue;
    const uint64_t* header = reinterpret_cast<const uint64_t*>(rawData.data());
    header--;
    bool moreHeaders = true;
    while (moreHeaders) {
      header++;
      moreHeaders = errorcheck.checkHeader(errorsInEvent, fedId, header, errors);
    }
    bool moreTrailers = true;
    trailer++;
    while (moreTrailers) {
      trailer--;
      moreTrailers = errorcheck.checkTrailer(errorsInEvent, fedId, nWords, trailer, errors);
    }
    const uint32_t* bw = (const uint32_t*)(header + 1);
    const uint32_t* ew = (const uint32_t*)(trailer);
    assert(0 == (ew - bw) % 2);
    h.appender->initializeWordFed(fedId, wordCounterGPU, bw, (ew - bw));
    wordCounterGPU += (ew - bw);
  }
  pixelgpudetails::SiPixelRawToClusterGPUKernel gpuAlgo;
  gpuAlgo.makeClusters(isRun2, gpuMap, modToUnp, gpuGains, *h.appender, std::move(errors), wordCounterGPU,
                       fedCounter, useQuality, includeErrors, false);
  auto dc = gpuAlgo.getResults();
  SiPixelDigisSoA digis = std::move(dc.first);
  SiPixelClustersSoA clusters = std::move(dc.second);
  SiPixelDigiErrorsSoA digiErrors = gpuAlgo.getErrors();

  // ---- SiPixelRecHitCUDA::produce
  pixelgpudetails::PixelRecHitGPUKernel rh;
  TrackingRecHit2DCPU hits = rh.makeHits(digis, clusters, h.bs, &h.cpe->getCPUProduct());

  // ---- CAHitNtupletCUDA::produce -> CAHitNtupletGeneratorOnGPU::makeTuples (:96-126)
  auto bf = 0.0114256972711507;
  float bfield = bf;
  PixelTrackHeterogeneous tracks(std::make_unique<pixelTrack::TrackSoA>());
  auto* soa = tracks.get();
  CAHitNtupletGeneratorKernelsCPU kernels(h.params());
  kernels.counters_ = h.caGen->m_counters;
  kernels.allocateOnGPU(nullptr);
  kernels.buildDoublets(hits, nullptr);
  kernels.launchKernels(hits, soa, nullptr);
  kernels.fillHitDetIndices(hits.view(), soa, nullptr);
  if (0 != hits.nHits()) {
    HelixFitOnGPU fitter(bfield, h.params().fit5as4_);
    fitter.allocateOnGPU(&(soa->hitIndices), kernels.tupleMultiplicity(), soa);
    if (h.params().useRiemannFit_ || h.useRiemannFit)
      fitter.launchRiemannKernelsOnCPU(hits.view(), hits.nHits(), CAConstants::maxNumberOfQuadruplets());
    else
      fitter.launchBrokenLineKernelsOnCPU(hits.view(), hits.nHits(), CAConstants::maxNumberOfQuadruplets());
    kernels.classifyTuples(hits, soa, nullptr);
  }

  // ---- PixelVertexProducerCUDA::produce
  ZVertexHeterogeneous vertices = h.vtx->make(tracks.get(), 0.5f);
  auto t1 = std::chrono::steady_clock::now();
  h.lastSeconds = std::chrono::duration<double>(t1 - t0).count();
  if (dump < 0) return 0;  // timing only: no product copies

  // ---- record products
  uint32_t nDigis = digis.nDigis();
  h.put1<uint32_t>("nDigis", nDigis);
  h.put1<uint32_t>("nModules", digis.nModules());
  h.put("xx", digis.xx(), nDigis);
  h.put("yy", digis.yy(), nDigis);
  h.put("adc", digis.adc(), nDigis);
  h.put("moduleInd", digis.moduleInd(), nDigis);
  h.put("clus", digis.clus(), nDigis);
  h.put("pdigi", digis.pdigi(), nDigis);
  h.put("rawIdArr", digis.rawIdArr(), nDigis);
  {
    auto const* ev = digiErrors.error();
    int ne = ev ? ev->size() : 0;
    h.put("errors", ev ? ev->data() : (const PixelErrorCompact*)nullptr, size_t(ne));
    // PixelFormatterErrors, flattened in map order (the product's 16-byte records)
    struct FormatterErrorRecord {
      uint64_t word64;
      uint32_t errorType, fedId;
    };
    std::vector<FormatterErrorRecord> fe;
    for (auto const& kv : digiErrors.formatterErrors())
      for (auto const& er : kv.second)
        fe.push_back({er.getWord64(), uint32_t(er.getType()), uint32_t(er.getFedId())});
    h.put("formatterErrors", fe.data(), fe.size());
  }
  h.put1<uint32_t>("nClusters", clusters.nClusters());
  h.put("moduleStart", clusters.moduleStart(), gpuClustering::MaxNumModules + 1);
  h.put("clusInModule", clusters.clusInModule(), gpuClustering::MaxNumModules);
  h.put("moduleId", clusters.moduleId(), gpuClustering::MaxNumModules);
  h.put("clusModuleStart", clusters.clusModuleStart(), gpuClustering::MaxNumModules + 1);

  uint32_t nHits = hits.nHits();
  h.put1<uint32_t>("nHits", nHits);
  {
    auto const& v = *hits.view();
    std::vector<float> xl(nHits), yl(nHits), xe(nHits), ye(nHits), xg(nHits), yg(nHits), zg(nHits), rg(nHits);
    std::vector<int32_t> ch(nHits);
    std::vector<int16_t> iphi(nHits), sx(nHits), sy(nHits);
    std::vector<uint16_t> det(nHits);
    for (uint32_t i = 0; i < nHits; ++i) {
      xl[i] = v.xLocal(i);
      yl[i] = v.yLocal(i);
      xe[i] = v.xerrLocal(i);
      ye[i] = v.yerrLocal(i);
      xg[i] = v.xGlobal(i);
      yg[i] = v.yGlobal(i);
      zg[i] = v.zGlobal(i);
      rg[i] = v.rGlobal(i);
      ch[i] = v.charge(i);
      iphi[i] = v.iphi(i);
      sx[i] = v.clusterSizeX(i);
      sy[i] = v.clusterSizeY(i);
      det[i] = v.detectorIndex(i);
    }
    h.put("xl", xl.data(), nHits);
    h.put("yl", yl.data(), nHits);
    h.put("xerr", xe.data(), nHits);
    h.put("yerr", ye.data(), nHits);
    h.put("xg", xg.data(), nHits);
    h.put("yg", yg.data(), nHits);
    h.put("zg", zg.data(), nHits);
    h.put("rg", rg.data(), nHits);
    h.put("charge", ch.data(), nHits);
    h.put("iphi", iphi.data(), nHits);
    h.put("xsize", sx.data(), nHits);
    h.put("ysize", sy.data(), nHits);
    h.put("detInd", det.data(), nHits);
    if (nHits) {
      h.put("hitsLayerStart", v.hitsLayerStart(), 11);
      auto const& hist = v.phiBinner();
      h.put("phiOff", hist.off, TrackingRecHit2DSOAView::Hist::totbins());
      h.put("phiBins", hist.bins, nHits);
    }
    auto const& agc = v.averageGeometry();
    h.put("agcLadderR", agc.ladderR, phase1PixelTopology::numberOfLaddersInBarrel);
  }

  if (dump) {
    uint32_t nCells = *kernels.device_nCells_;
    h.put1<uint32_t>("nCells", nCells);
    std::vector<uint16_t> ci(nCells), co(nCells), cu(nCells);
    std::vector<int16_t> cl(nCells);
    std::vector<int32_t> cd(nCells);
    std::vector<uint32_t> nOff(1, 0), nVal, tOff(1, 0), tVal;
    GPUCACell const* cells = kernels.device_theCells_.get();
    for (uint32_t c = 0; c < nCells; ++c) {
      ci[c] = cells[c].theInnerHitId;
      co[c] = cells[c].theOuterHitId;
      cl[c] = cells[c].theLayerPairId;
      cd[c] = cells[c].theDoubletId;
      cu[c] = cells[c].theUsed;
      for (auto x : cells[c].outerNeighbors()) nVal.push_back(x);
      nOff.push_back(uint32_t(nVal.size()));
      for (auto x : cells[c].tracks()) tVal.push_back(x);
      tOff.push_back(uint32_t(tVal.size()));
    }
    h.put("cellInner", ci.data(), nCells);
    h.put("cellOuter", co.data(), nCells);
    h.put("cellLayerPair", cl.data(), nCells);
    h.put("cellDoubletId", cd.data(), nCells);
    h.put("cellUsed", cu.data(), nCells);
    h.put("cellNbrOff", nOff.data(), nOff.size());
    h.put("cellNbr", nVal.data(), nVal.size());
    h.put("cellTrkOff", tOff.data(), tOff.size());
    h.put("cellTrk", tVal.data(), tVal.size());
    std::vector<uint32_t> oOff(1, 0), oVal;
    if (nHits) {
      auto const* ohc = kernels.device_isOuterHitOfCell_.get();
      for (uint32_t i = 0; i < nHits; ++i) {
        for (auto x : ohc[i]) oVal.push_back(x);
        oOff.push_back(uint32_t(oVal.size()));
      }
    }
    h.put("outerHitOff", oOff.data(), oOff.size());
    h.put("outerHitCells", oVal.data(), oVal.size());
    h.put1<int32_t>("nNbrLists", kernels.device_theCellNeighbors_->size());
    h.put1<int32_t>("nTrkLists", kernels.device_theCellTracks_->size());
  }

  // tracks: only the filled prefix (the serial loops stop at the first empty tuple)
  {
    auto const& t = *soa;
    auto const& hc = t.hitIndices;
    uint32_t nt = 0;
    while (nt < uint32_t(pixelTrack::TrackSoA::stride()) && hc.size(nt) > 0) ++nt;
    h.put1<uint32_t>("nTuples", nt);
    h.put("tupleOff", hc.off, nt + 1);
    h.put("tupleHits", hc.bins, hc.off[nt]);
    h.put("tupleDet", t.detIndices.bins, hc.off[nt]);
    h.put("quality", t.m_quality.data(), nt);
    std::vector<float> st(size_t(nt) * 5), cv(size_t(nt) * 15), pt(nt), eta(nt), chi2(nt);
    for (uint32_t i = 0; i < nt; ++i) {
      for (int k = 0; k < 5; ++k) st[i * 5 + k] = t.stateAtBS.state(i)(k);
      for (int k = 0; k < 15; ++k) cv[i * 15 + k] = t.stateAtBS.covariance(i)(k);
      pt[i] = t.pt(i);
      eta[i] = t.eta(i);
      chi2[i] = t.chi2(i);
    }
    h.put("state", st.data(), st.size());
    h.put("cov", cv.data(), cv.size());
    h.put("pt", pt.data(), nt);
    h.put("eta", eta.data(), nt);
    h.put("chi2", chi2.data(), nt);
  }
  {
    auto const& v = *vertices.get();
    uint32_t nv = v.nvFinal;
    h.put1<uint32_t>("nVertices", nv);
    h.put("zv", v.zv, nv);
    h.put("wv", v.wv, nv);
    h.put("vchi2", v.chi2, nv);
    h.put("ptv2", v.ptv2, nv);
    h.put("ndof", v.ndof, nv);
    h.put("sortInd", v.sortInd, nv);
    uint32_t nt = *reinterpret_cast<const uint32_t*>(h.out["nTuples"].bytes.data());
    h.put("idv", v.idv, nt);
  }
  return 0;
}

// Pointer to a named product recorded by the last pr_process call.
int pr_get(void* p, const char* name, const void** data, size_t* count, int* elem) {
  RefChain& h = *static_cast<RefChain*>(p);
  auto it = h.out.find(name);
  if (it == h.out.end()) return -1;
  *data = it->second.bytes.data();
  *elem = it->second.elem;
  *count = it->second.bytes.size() / size_t(it->second.elem);
  return 0;
}

// Names of all recorded products, separated by ','.
int pr_names(void* p, char* buf, size_t n) {
  RefChain& h = *static_cast<RefChain*>(p);
  std::string s;
  for (auto& kv : h.out) {
    if (!s.empty()) s += ',';
    s += kv.first;
  }
  if (s.size() + 1 > n) return -1;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return 0;
}

// Seconds spent in the chain (excluding input parsing and product recording)
// during the last pr_process call.
double pr_last_seconds(void* p) { return static_cast<RefChain*>(p)->lastSeconds; }

void pr_set_formatter_errors(void* p, int on) { static_cast<RefChain*>(p)->formatterErrors = on != 0; }

void pr_set_riemann(void* p, int on) { static_cast<RefChain*>(p)->useRiemannFit = on != 0; }

// A CA module configuration that differs from the reference's own in its
// switches (CAHitNtupletGeneratorOnGPU.cc:46-58); every cut value is kept.
int pr_set_ca_params(void* p, int minHitsPerNtuplet, int includeJumpingForwardDoublets, int earlyFishbone,
                     int lateFishbone, int idealConditions, int doClusterCut, int doZ0Cut, int doPtCut) {
  if (minHitsPerNtuplet < 3 || minHitsPerNtuplet > 4) return -1;
  auto& h = *static_cast<RefChain*>(p);
  const auto& d = h.caGen->m_params;
  h.caParams = std::make_unique<cAHitNtupletGenerator::Params>(
      d.onGPU_, uint32_t(minHitsPerNtuplet), d.maxNumberOfDoublets_, d.useRiemannFit_, d.fit5as4_,
      includeJumpingForwardDoublets != 0, earlyFishbone != 0, lateFishbone != 0, idealConditions != 0, d.doStats_,
      doClusterCut != 0, doZ0Cut != 0, doPtCut != 0, d.ptmin_, d.CAThetaCutBarrel_, d.CAThetaCutForward_,
      d.hardCurvCut_, d.dcaCutInnerTriplet_, d.dcaCutOuterTriplet_, d.cuts_);
  return 0;
}

// The vertex finder of a PixelVertexProducerCUDA configured with useDensity
// (0, the reference's own configuration), useDBSCAN (1) or useIterative (2);
// the other parameters as in PixelVertexProducerCUDA.cc:26-35.
int pr_set_vertex_algo(void* p, int algo) {
  if (algo < 0 || algo > 2) return -1;
  static_cast<RefChain*>(p)->vtx =
      std::make_unique<gpuVertexFinder::Producer>(true, algo == 0, algo == 1, algo == 2, 2, 0.07, 0.01, 9);
  return 0;
}

// Event-level parallel timing, the reference's own concurrency model (one
// chain instance per stream, README.md:222-226): `threads` host threads, each
// with its own instance, take events from a shared counter.  Returns the wall
// seconds over all events (instances created beforehand), or < 0 on failure;
// lat[k] receives event k's chain seconds.
double pr_time_events(const char* datadir, const uint8_t* const* raws, const size_t* sizes, int n, int threads,
                      double* lat) {
  if (threads < 1) threads = 1;
  std::vector<void*> chains;
  try {
    for (int t = 0; t < threads; ++t) chains.push_back(pr_create(datadir));
  } catch (std::exception&) {
    for (void* c : chains) pr_destroy(c);
    return -1.0;
  }
  std::atomic<int> next{0}, failed{0};
  std::vector<std::thread> pool;
  auto t0 = std::chrono::steady_clock::now();
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t]() {
      for (;;) {
        int k = next.fetch_add(1);
        if (k >= n) break;
        try {
          if (pr_process(chains[t], raws[k], sizes[k], -1) != 0) failed++;
        } catch (std::exception&) {
          failed++;
        }
        if (lat) lat[k] = static_cast<RefChain*>(chains[t])->lastSeconds;
      }
    });
  }
  for (auto& th : pool) th.join();
  auto t1 = std::chrono::steady_clock::now();
  for (void* c : chains) pr_destroy(c);
  if (failed) return -1.0;
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"

// Riemann fit of n standalone tuples of N (3 or 4) hits through the
// reference's own Rfit functions, in the order of kernelFastFit,
// kernelCircleFit and kernelLineFit (RiemannFitOnGPU.h:20-162), with the
// result packing of kernelLineFit (:156-162).  Layout as the oracle's or_fit:
// hits[(t*N+i)*3+k], ge[(t*N+i)*6+k]; outputs state[t*5], cov[t*15],
// pt/eta/chi2[t].
template <int N>
static void refRiemann(uint32_t n, const double* hits, const float* ge, double B, float* state, float* cov, float* pt,
                       float* eta, float* chi2) {
  auto soa = std::make_unique<pixelTrack::TrackSoA>();
  for (uint32_t t = 0; t < n; ++t) {
    Rfit::Matrix3xNd<N> h;
    Eigen::Matrix<float, 6, N> g;
    for (int i = 0; i < N; ++i) {
      for (int k = 0; k < 3; ++k) h(k, i) = hits[(size_t(t) * N + i) * 3 + k];
      for (int k = 0; k < 6; ++k) g(k, i) = ge[(size_t(t) * N + i) * 6 + k];
    }
    Rfit::Vector4d fast_fit;
    Rfit::Fast_fit(h, fast_fit);
    Rfit::VectorNd<N> rad = (h.block(0, 0, 2, N).colwise().norm());
    Rfit::Matrix2Nd<N> hits_cov = Rfit::Matrix2Nd<N>::Zero();
    Rfit::loadCovariance2D(g, hits_cov);
    Rfit::circle_fit circle = Rfit::Circle_fit(h.block(0, 0, 2, N), hits_cov, fast_fit, rad, B, true);
    auto const& line = Rfit::Line_fit(h, g, circle, fast_fit, B, true);
    Rfit::fromCircleToPerigee(circle);
    soa->stateAtBS.copyFromCircle(circle.par, circle.cov, line.par, line.cov, 1.f / float(B), 0);
    for (int k = 0; k < 5; ++k) state[size_t(t) * 5 + k] = soa->stateAtBS.state(0)(k);
    for (int k = 0; k < 15; ++k) cov[size_t(t) * 15 + k] = soa->stateAtBS.covariance(0)(k);
    pt[t] = B / std::abs(circle.par(2));
    eta[t] = asinhf(line.par(0));
    chi2[t] = (circle.chi2 + line.chi2) / (2 * N - 5);
  }
}

extern "C" int pr_fit_riemann(int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                              float* cov, float* pt, float* eta, float* chi2) {
  if (N == 3)
    refRiemann<3>(n, hits, ge, B, state, cov, pt, eta, chi2);
  else if (N == 4)
    refRiemann<4>(n, hits, ge, B, state, cov, pt, eta, chi2);
  else
    return -1;
  return 0;
}
