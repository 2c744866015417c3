// CPU oracle: a sequential restatement of the reference's serial pixel chain,
// used only as the checker by tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py.  Nothing in the product links or calls it.
//
// Each function states the reference file:line it follows (paths relative to
// the reference's src/serial tree).  Integer outputs and all orderings are
// those of the serial backend; floating-point expressions keep the reference's
// evaluation order and types (including where an unqualified call such as
// fabs(float) resolves to the double overload in the serial build).
#ifndef PIXORACLE_H
#define PIXORACLE_H

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "pixfmt.h"

namespace oracle {

// Container capacities.  The defaults are the reference's compile-time
// constants and module parameters, whose overflow behaviour parity covers:
// MAX_FED_WORDS (SiPixelRawToClusterGPUKernel.cc:34), maxNumberOfHits
// (gpuClusteringConstants.h:10,27), maxNumberOfDoublets (the module parameter,
// CAHitNtupletGeneratorOnGPU.cc:48), maxNumOfActiveDoublets (CAConstants.h:40,
// the CellNeighbors and CellTracks pools), the HitContainer bins = TrackSoA
// stride (PixelTrackHeterogeneous.h:20,62; also the vertex finder's track
// stride, ZVertexSoA.h:11), maxNumberOfTuples (CAConstants.h:22: the
// TupleMultiplicity content and the fits' concurrency) and the HitToTuple
// content (4 x maxNumberOfTuples, CAConstants.h:64).  The reference changes
// them only by recompiling (CAConstants.h:18-40 selects smaller sets with
// GPU_SMALL_EVENTS); a larger set runs the same algorithm on events whose
// containers would overflow, with indices held in 32 bits throughout.
struct Caps {
  uint32_t fedWords = PF_MAX_FED_WORDS;
  uint32_t hits = PF_MAX_HITS;
  uint32_t doublets = PF_MAX_DOUBLETS_PARAM;
  uint32_t lists = PF_MAX_ACTIVE_DOUBLETS;
  uint32_t tuples = PF_TRACK_STRIDE;
  uint32_t multiplicity = PF_MAX_TUPLES;
  uint32_t hitToTuple = 4 * PF_MAX_TUPLES;
  bool isDefault() const {
    return fedWords == PF_MAX_FED_WORDS && hits == PF_MAX_HITS && doublets == PF_MAX_DOUBLETS_PARAM &&
           lists == PF_MAX_ACTIVE_DOUBLETS && tuples == PF_TRACK_STRIDE && multiplicity == PF_MAX_TUPLES &&
           hitToTuple == 4 * PF_MAX_TUPLES;
  }
};

struct ES {
  std::unique_ptr<PfCablingMap> cab;
  std::vector<uint8_t> modToUnp;
  PfGainHeader gain;
  std::vector<uint8_t> gainPayload;
  PfCommonParams common;
  std::vector<PfDetParams> det;
  PfAverageGeometry ag;
  PfLayerGeometry lg;
  PfBeamSpot bs;
  std::vector<uint32_t> fedIds;
};

// parse the ES file images (pixfmt.h); throws std::runtime_error on malformed input
void loadES(ES& es, const uint8_t* cabling, size_t ncab, const uint8_t* gain, size_t ngain, const uint8_t* cpe,
            size_t ncpe, const uint8_t* bs, size_t nbs, const uint8_t* fedids, size_t nfed);

struct Words {
  std::vector<uint32_t> word;
  std::vector<uint8_t> fedId;  // one per word pair, fedId - 1200
  uint32_t nWords = 0;
  std::vector<PfFormatterError> formatterErrors;  // with includeErrors in the ErrorChecker
};

struct Digis {
  uint32_t nDigis = 0, nModules = 0;
  std::vector<uint16_t> xx, yy, adc, moduleInd;
  std::vector<int32_t> clus;
  std::vector<uint32_t> pdigi, rawIdArr;
  std::vector<PfPixelError> errors;
};

struct Clusters {
  uint32_t nClusters = 0;
  std::vector<uint32_t> moduleStart, clusInModule, moduleId, clusModuleStart;
};

struct Hits {
  uint32_t nHits = 0;
  std::vector<float> xl, yl, xerr, yerr, xg, yg, zg, rg;
  std::vector<int32_t> charge;
  std::vector<int16_t> iphi, xsize, ysize;
  std::vector<uint16_t> detInd;
  uint32_t layerStart[11] = {};
  std::vector<uint32_t> phiOff;    // 10*128+1
  std::vector<uint32_t> phiBins;   // nHits
  PfAverageGeometry agc;           // beam-spot corrected average geometry
};

struct CA {
  uint32_t nCells = 0;
  uint32_t tupleBins = PF_TRACK_STRIDE;              // HitContainer bins (Caps::tuples)
  std::vector<uint32_t> inner, outer;
  std::vector<uint16_t> used;
  std::vector<int16_t> layerPair;
  std::vector<int32_t> doubletId;
  std::vector<float> innerZ, innerR;
  std::vector<std::vector<uint32_t>> outerHitCells;  // per hit, capped at 128
  std::vector<std::vector<uint32_t>> nbr;            // per cell, capped at 36
  std::vector<std::vector<uint32_t>> trk;            // per cell, capped at 48
  int32_t nbrPool = 1, trkPool = 1;                  // SimpleVector sizes (slot 0 = empty list)
  // tuples
  uint32_t apcM = 0, apcN = 0;                       // AtomicPairCounter {m, n}
  std::vector<uint32_t> tupleOff;                    // tupleBins + 1
  std::vector<uint32_t> tupleHits;                   // 5 * tupleBins
  std::vector<uint16_t> tupleDet;
  std::vector<uint8_t> quality;                      // tupleBins
  std::vector<uint32_t> tmOff;                       // TupleMultiplicity off[9]
  std::vector<uint32_t> tmBins;
  // fit results
  std::vector<float> state, cov, pt, eta, chi2;      // state[i*5+k], cov[i*15+k]
  // cut decisions whose two sides lie within kCutMarginRel of each other
  // (cutNear): doublet cuts, CA cuts (RZ alignment, curvature, dca),
  // classification cuts; the decisions that can flip when the operands are
  // computed in another precision
  uint32_t nearDoublet = 0, nearCA = 0, nearQuality = 0;
  uint32_t size(uint32_t t) const { return tupleOff[t + 1] - tupleOff[t]; }
};

struct Vertices {
  uint32_t nvFinal = 0;
  std::vector<float> zv, wv, chi2, ptv2;
  std::vector<int32_t> ndof;
  std::vector<uint16_t> sortInd;
  std::vector<int16_t> idv;
};

struct Event {
  Words words;
  Digis digis;
  Clusters clusters;
  Hits hits;
  CA ca;
  Vertices vtx;
};

// plugin-SiPixelClusterizer/SiPixelRawToClusterCUDA.cc:78-138 (FED loop, ErrorChecker, WordFedAppender);
// formatterErrors: the ErrorChecker's includeErrors (false in the reference's ErrorChecker.cc:36)
void fedLoop(const ES& es, const uint8_t* raw, size_t n, Words& w, bool formatterErrors = false,
             const Caps& caps = Caps());
// SiPixelRawToClusterGPUKernel::makeClusters (SiPixelRawToClusterGPUKernel.cc:509-600)
void makeClusters(const ES& es, const Words& w, Digis& d, Clusters& c, const Caps& caps = Caps());
// countModules, findClus, clusterChargeCut and fillHitsModuleStart on the
// digis d (xx, yy, calibrated adc, moduleInd; nDigis) -- the second half of
// makeClusters (gpuClustering.h:19-273, gpuClusterChargeCut.h:14-114,
// SiPixelRawToClusterGPUKernel.cc:464-506); sets d.clus and d.nModules
void clusterDigis(Digis& d, Clusters& c, const Caps& caps = Caps());
// PixelRecHitGPUKernel::makeHits (plugin-SiPixelRecHits/PixelRecHits.cc:33-53)
void makeHits(const ES& es, const Digis& d, const Clusters& c, Hits& h, const Caps& caps = Caps());
// the CA module's configurable switches (CAHitNtupletGeneratorOnGPU.cc:46-58,
// defaults as there; the cut values stay the reference's constants)
struct CAParams {
  uint32_t minHitsPerNtuplet = 3;              // 3 or 4
  bool includeJumpingForwardDoublets = true;   // pairs 15..18
  bool earlyFishbone = true, lateFishbone = false;
  bool idealConditions = true, doClusterCut = true, doZ0Cut = true, doPtCut = true;
  bool useRiemannFit = false;                  // Riemann fit in place of the broken-line fit
  Caps caps;                                   // container capacities
  // CAHitNtupletGeneratorKernels.cc:52-57: the layer pairs that are built
  int nPairs() const { return minHitsPerNtuplet > 3 ? 13 : (includeJumpingForwardDoublets ? 19 : 15); }
};

// CAHitNtupletGeneratorOnGPU::makeTuples (plugin-PixelTriplets/CAHitNtupletGeneratorOnGPU.cc:96-126)
void makeTuples(const ES& es, const Hits& h, CA& ca, const CAParams& p = CAParams());
// gpuVertexFinder::Producer::make (plugin-PixelVertexFinding/gpuVertexFinderImpl.h:84-111);
// algo: 0 clusterTracksByDensity (the PixelVertexProducerCUDA default),
// 1 clusterTracksDBSCAN, 2 clusterTracksIterative
void makeVertices(const CA& ca, Vertices& v, int algo = 0);
// the vertex finder's track stride is the TrackSoA stride (ca.tupleBins)

// broken-line fit of one tuple of N (3 or 4) hits; results in the TrackSoA layout
void brokenLineFit(int N, const double* hits /*3xN col-major*/, const float* hits_ge /*6xN*/, double B,
                   float* state5, float* cov15, float* pt, float* eta, float* chi2);

// Riemann fit of one tuple of N (3 or 4) hits; same I/O as brokenLineFit
void riemannFit(int N, const double* hits /*3xN col-major*/, const float* hits_ge /*6xN*/, double B, float* state5,
                float* cov15, float* pt, float* eta, float* chi2);

// Relative margin below which a cut decision counts as on its boundary: four
// single-precision ulps (2^-22) of the larger side.  Evaluated in double from
// the operands the cut compares, so that every implementation of the chain
// that computes those operands bit for bit counts the same decisions.
constexpr double kCutMarginRel = 1.0 / 4194304.0;
inline bool cutNear(double a, double b) {
  const double d = a > b ? a - b : b - a;
  const double m = (a < 0 ? -a : a) > (b < 0 ? -b : b) ? (a < 0 ? -a : a) : (b < 0 ? -b : b);
  return d <= kCutMarginRel * m;
}

// whole chain for one raw.bin event record
struct Options {
  CAParams ca;                   // ca.caps: the container capacities of the whole chain
  int vertexAlgo = 0;            // see makeVertices
  bool formatterErrors = false;  // see fedLoop
};
void processEvent(const ES& es, const uint8_t* raw, size_t n, Event& ev, const Options& o = Options());

}  // namespace oracle

#endif
