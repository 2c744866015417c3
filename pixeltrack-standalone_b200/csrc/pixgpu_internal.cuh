// Internal declarations of the B200 pixel chain: device ES tables, the batch
// workspace (per-event fixed strides, ragged FED words) and small device
// primitives shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pixfmt.h"
#include "pixgpu.h"

namespace pixgpu {

// ---------------------------------------------------------------- capacities
constexpr uint32_t kMaxModules = PF_MAX_MODULES;         // 2000
constexpr uint32_t kModStride = 2048;                    // per-event stride of module arrays
constexpr uint32_t kPhiTot = 10 * PF_PHI_BINS + 1;       // 1281
constexpr uint32_t kPhiStride = 1288;
constexpr uint32_t kMaxVtx = PF_MAX_VTX;
constexpr uint32_t kErrCap = 4096;                       // digi errors kept per event
constexpr uint32_t kBigSegCap = 8192;                    // long list segments queued per event and sort
// hit indices are packed with a module index into one 32-bit word of the
// doublet search's hit records (11 + 21 bits)
constexpr uint32_t kMaxHitCapLimit = 1u << 21;

// Per-event container capacities (a context's pg_config caps).  The
// defaults are the reference's compile-time constants and module parameters,
// whose truncation order parity covers; larger values run the same algorithm
// on events whose containers would overflow (indices are 32-bit throughout).
// Every per-event array is strided by these.
struct Caps {
  uint32_t fedWords;      // FED words per event (MAX_FED_WORDS)
  uint32_t hits;          // clusters kept per event (maxNumberOfHits)
  uint32_t cells;         // doublets (maxNumberOfDoublets, the module parameter)
  uint32_t edges;         // CA links kept (the neighbour lists' content)
  uint32_t lists;         // cells with a neighbour / a track list (maxNumOfActiveDoublets)
  uint32_t tuples;        // HitContainer bins = TrackSoA stride
  uint32_t multiplicity;  // TupleMultiplicity content = concurrent fits per multiplicity (maxNumberOfTuples)
  uint32_t h2t;           // HitToTuple content
  uint32_t jCap;          // doublet inner-hit slots (6 x hits covers every inner layer of the 19 pairs)
  uint32_t scratch;       // 32-bit words of scratchA/scratchB per event
  __host__ __device__ uint32_t tupleHits() const { return 5 * tuples; }
  __host__ __device__ uint32_t tupleCells() const { return 4 * tuples; }
};

// the reference's capacities
inline Caps referenceCaps() {
  Caps c;
  c.fedWords = PF_MAX_FED_WORDS;         // 300000
  c.hits = PF_MAX_HITS;                  // 49152
  c.cells = PF_MAX_DOUBLETS_PARAM;       // 458752
  c.edges = 2 * PF_MAX_DOUBLETS_PARAM;   // 917504
  c.lists = PF_MAX_ACTIVE_DOUBLETS;      // 65536
  c.tuples = PF_TRACK_STRIDE;            // 32768
  c.multiplicity = PF_MAX_TUPLES;        // 24576
  c.h2t = 4 * PF_MAX_TUPLES;             // 98304
  c.jCap = 6 * c.hits;
  c.scratch = c.edges;
  return c;
}

// The vertex finder's track cap (ZVertexSoA MAXTRACKS) and the per-event
// scratch it carves out of scratchA/scratchB for events above its
// shared-memory size (k_vertex.cu scratchOf): nine 32-bit arrays in A (the
// ninth the tracks' tuple indices); one 16-bit and two 8-bit arrays in B.
// noalloc.cu sizes its static array from the same numbers.
constexpr uint32_t kMaxVtxTracks = 32 * 1024;
constexpr size_t kVtxScratchAWords = size_t(9) * kMaxVtxTracks;
constexpr size_t kVtxScratchBWords = size_t(kMaxVtxTracks);

// flag bits in EventCounters::flags (capacity conditions where the result no
// longer follows the reference's truncation order exactly)
enum : uint32_t {
  kFlagModuleTooBig = 1u << 0,      // > 4000 pixels or > 1024 clusters in a module (truncated as the serial build)
  kFlagEdgeOverflow = 1u << 1,      // more CA links than cap.edges
  kFlagNbrPoolOverflow = 1u << 2,   // more cells with neighbours than the 65535-list pool
  kFlagTrkPoolOverflow = 1u << 3,   // more cells with tracks than the 65535-list pool
  kFlagFitBinOverflow = 1u << 4,    // more tuples of one multiplicity than concurrent fits
  kFlagTupleOverflow = 1u << 5,     // more tuples than HitContainer bins (reference drops the tail)
  kFlagCellOverflow = 1u << 6,      // doublet capacity reached (reference truncates; reproduced)
  kFlagHitOverflow = 1u << 7,       // more clusters than the hit capacity (reference truncates; reproduced)
  kFlagErrOverflow = 1u << 8,       // more digi errors than kErrCap
  kFlagTooManyWords = 1u << 9,      // event larger than cap.fedWords
  kFlagH2TOverflow = 1u << 10,      // hit-to-tuple capacity exceeded
  kFlagTmOverflow = 1u << 11,       // tuple multiplicity capacity exceeded
  kFlagVtxOverflow = 1u << 12,      // split vertex with >= 512 tracks or > 1024 vertices
  kFlagDeepTuple = 1u << 13,        // a CA path longer than 5 hits (reference aborts)
  kFlagJOverflow = 1u << 14,        // more doublet inner-hit slots than cap.jCap
  kFlagBadInput = 1u << 15,         // words/cabling entries outside the tables (ignored)
  kFlagSplitModule = 1u << 17,      // a module's digis in several runs (later runs read as padding)
  kFlagTooManyRuns = 1u << 18,      // more than 2000 module runs (the reference's counter wraps)
  kFlagScanStall = 1u << 19         // a scan tile waited past its bound for its predecessor (offsets invalid)
};

static_assert(uint32_t(kFlagBadInput) == uint32_t(PG_FLAG_BAD_INPUT) &&
                  uint32_t(kFlagJOverflow) == uint32_t(PG_FLAG_J_OVERFLOW) &&
                  uint32_t(kFlagTupleOverflow) == uint32_t(PG_FLAG_TUPLE_OVERFLOW) &&
                  uint32_t(kFlagModuleTooBig) == uint32_t(PG_FLAG_MODULE_TOO_BIG) &&
                  uint32_t(kFlagSplitModule) == uint32_t(PG_FLAG_SPLIT_MODULE) &&
                  uint32_t(kFlagTooManyRuns) == uint32_t(PG_FLAG_TOO_MANY_RUNS),
              "flag bits of the ABI");

struct EventCounters {
  uint32_t wordStart, nWords;   // input slice of the batch word buffer
  uint32_t nModules;            // module runs found (moduleStart[0])
  uint32_t nHits;               // clusModuleStart[2000]
  uint32_t layerStart[11];      // hitsLayerStart
  uint32_t ntot;                // doublet candidates (inner hits over all layer pairs)
  uint32_t pairCum[20];         // cumulative inner layer sizes per pair
  uint32_t nCellsRaw;           // doublets found before the capacity cut
  uint32_t nCells;              // doublets kept
  uint32_t nEdges;              // CA links
  uint32_t nNbrLists, nTrkLists;  // pool usage (including the reserved empty list)
  uint32_t apcM, apcN;          // tuples attempted and their hits
  uint32_t nTuples;             // tuples stored (min(apcM, 32768))
  uint32_t nTupleCells;         // entries of the tuple->cell table
  uint32_t nCandidates;         // cells with >= 2 tracks
  uint32_t nLoose;              // loose tuples
  uint32_t nVertices;
  uint32_t nErrors;
  uint32_t nVtxTracks;
  uint32_t flags;
  uint32_t nBig[4];             // long segments queued by each list ordering
  uint32_t nBigMod;             // modules queued for the block clusterizer
  uint32_t nSegList[4];         // list segments that received a second entry, per list ordering
  uint32_t nBigHitMod;          // modules queued for the block rechit kernel
  // cut decisions on their float boundary (cutNear): doublet, CA and quality cuts
  uint32_t nearDoublet, nearCA, nearQuality;
  uint32_t nStaged;             // tuples staged by the n-tuplet count pass
  uint32_t nFishHits;           // entries of the early fishbone's hit list
  uint32_t nLinked;             // cells with CA links (the n-tuplet search's start candidates)
};

// A cut decision counts as on its boundary when its two sides lie within
// four single-precision ulps (2^-22, relative) of the larger one, evaluated
// in double from the operands the cut compares: the decisions that can flip
// when those operands come from another precision.  The oracle counts the
// same decisions with the same test.
__device__ __forceinline__ uint32_t cutNear(double a, double b) {
  const double d = fabs(a - b);
  return d <= (1.0 / 4194304.0) * fmax(fabs(a), fabs(b)) ? 1u : 0u;
}
// The same test on single-precision operands, with a single-precision
// exclusion first: the rounded |a - b| is within 2^-24 of the exact one
// (exact for subnormal results), so a rounded difference above 2^-21 of the
// larger magnitude (a power-of-two scaling, exact for normal results) means
// the exact test fails.  NaN operands reach the exact test, which fails.
// The double-precision test is out of line: it is rarely reached, and
// inlined it cost the hot candidate loops registers and scheduling (measured:
// doublet count 601 -> 525 us per 64-event batch).
static __device__ __noinline__ uint32_t cutNearExact(float a, float b) { return cutNear(double(a), double(b)); }
__device__ __forceinline__ uint32_t cutNear(float a, float b) {
  if (fabsf(a - b) > 4.76837158203125e-7f * fmaxf(fabsf(a), fabsf(b))) return 0u;
  return cutNearExact(a, b);
}

// ---------------------------------------------------------------- ES on device
struct DeviceES {
  const PfCablingMap* cab;
  const uint8_t* modToUnp;
  const PfGainHeader* gainHdr;
  const uint8_t* gainPayload;
  const PfCommonParams* common;
  const PfDetParams* det;
  const PfAverageGeometry* ag;
  const PfLayerGeometry* lg;
  const PfBeamSpot* bs;
  uint32_t nDet;             // entries of det[]
  uint32_t gainPayloadSize;  // bytes of gainPayload
};

// ---------------------------------------------------------------- batch workspace
// where the batch's FED words live (the slot's staging buffer or a slice of
// the device-resident pool); read by the kernels so that a captured graph
// does not depend on it
struct BatchInput {
  const uint32_t* words;
  const uint8_t* fedIds;
};

// segmented scans of the chain: one state region each per event (scan.cu)
enum ScanCall : uint32_t {
  kScanPhi = 0,
  kScanDoubletSlots,
  kScanOuterHits,
  kScanNeighbours,
  kScanStartTuples,
  kScanStartHits,
  kScanCellTracks,
  kScanHitTuples,
  kScanCalls
};
constexpr uint32_t kScanTile = 4096;  // elements per tile of the single-pass scan
constexpr uint32_t kFlatMaxEvents = 1024;  // events per batch (kernels with one flat grid over the batch)

// CAHitNtupletGeneratorOnGPU parameters that select among the algorithm's
// variants (CAHitNtupletGeneratorOnGPU.cc:45-66; CAHitNtupletGeneratorKernels.cc:52-70)
struct CAConfig {
  uint32_t nPairs;           // layer pairs searched: 19; 15 without jumping forward doublets; 13 for quadruplets
  uint32_t minHits;          // minHitsPerNtuplet (3 or 4)
  uint32_t idealConditions;  // every ladder treated as outer in the cluster-size cut
  uint32_t doClusterCut, doZ0Cut, doPtCut;
  uint32_t earlyFishbone, lateFishbone;
  uint32_t mixedFit;         // the fits' mixed-precision variants (pg_config mixed_fit)
};

// FED scan on the device (fedscan.cu): the batch's whole FED blocks and the
// per-FED bookkeeping of the header/trailer walk
constexpr uint32_t kFmtErrCap = 1024;  // framing errors kept per event
struct FedScanBuffers {
  uint32_t on;               // 1: the chain starts from raw FED blocks (else from host-unpacked words)
  uint32_t recordErrors;     // record the framing errors (the ErrorChecker's includeErrors)
  uint32_t nFeds;            // FEDs of the ES list, in its order (fedId 40 and ids >= 4096 left out)
  uint32_t rawCap64;         // capacity of raw64, in 64-bit words
  const uint32_t* fedIds;    // [nFeds]
  uint64_t* raw64;           // the FED blocks, header to trailer, 8-byte aligned
  uint2* tab;                // [maxEvents][nFeds] {first 64-bit word in raw64, 64-bit length}
  uint32_t* len;             // [maxEvents][nFeds] payload words
  uint32_t* src;             // [maxEvents][nFeds] first payload 64-bit word in raw64
  uint32_t* dst;             // [maxEvents][nFeds] first payload word within the event
  uint32_t* evWords;         // [maxEvents]
  PfFormatterError* fmt;     // [maxEvents][kFmtErrCap]
  uint32_t* fmtCount;        // [maxEvents] (may exceed kFmtErrCap; the first kFmtErrCap are kept)
};

// Launch-shape tuning (tune.cu): the grid x-extent of each tunable launch is
// its default (a function of the batch size) times 2^scale.  Every tunable
// kernel loops grid-stride over its event's work, so the scale changes only
// the speed, never the results.
enum TuneId : uint32_t {
  kTuneRawToDigi, kTuneModuleBoundaries, kTuneFindClustersBig, kTuneGetHitsBig, kTunePhiCount, kTunePhiFill,
  kTunePhiRec, kTuneDoubletCount, kTuneDoubletWrite, kTuneOuterHitFill, kTuneOhRec, kTuneConnect, kTuneEdgeScatter,
  kTuneNbrPool, kTuneFishbone, kTuneNtupletCount, kTuneNtupletWrite, kTuneTrackCount, kTuneTrackFill,
  kTuneTrackPool, kTuneEarlyDup, kTuneTupleDet, kTuneClassify, kTuneFastDupInDegree,
  kTuneHitToTupleCount, kTuneHitToTupleFill, kTuneTripletCleaner, kTuneFitZero, kTuneFit, kTuneFedCopy, kNumTune
};
extern const char* const kTuneNames[kNumTune];
constexpr int kTuneMinScale = -3, kTuneMaxScale = 3;
struct LaunchTuning {
  int8_t scale[kNumTune];
};

struct Workspace {
  uint32_t maxEvents;
  uint32_t wordCap;          // words over the whole batch
  Caps cap;                  // per-event capacities (the strides of every per-event array)
  CAConfig ca;               // the context's CA configuration
  FedScanBuffers scan;       // device FED scan (scan.on == 0: not used)
  LaunchTuning tune;         // grid scales of the tunable launches (host side)
  // input
  uint32_t* words;
  uint8_t* fedIds;
  uint32_t* wordOffsets;     // [maxEvents + 1]
  BatchInput* input;         // device-resident descriptor of the batch input
  EventCounters* ev;         // [maxEvents]
  // digis (flat, batch word index)
  uint16_t *xx, *yy, *adc, *moduleInd;
  int32_t* clus;
  uint32_t *pdigi, *rawIdArr;
  PfPixelError* errors;      // [maxEvents][kErrCap]
  uint32_t* errWordIdx;      // [maxEvents][kErrCap]
  // clusters [maxEvents][kModStride]
  uint32_t *moduleStart, *clusInModule, *moduleId, *clusModuleStart;
  // hits [maxEvents][cap.hits]
  float *xl, *yl, *xerr, *yerr, *xg, *yg, *zg, *rg;
  int32_t* charge;
  int16_t *iphi, *xsize, *ysize;
  uint16_t* detInd;
  uint32_t* phiOff;          // [maxEvents][kPhiStride]
  uint32_t* phiBins;         // [maxEvents][cap.hits]
  uint4* phiRec;             // [maxEvents][cap.hits] hit records in phiBins order: z, r, iphi|ysize<<16,
                             // min(detInd, 2047)|hit<<11
  PfAverageGeometry* agc;    // [maxEvents]
  // doublets
  uint32_t* jCount;          // [maxEvents][cap.jCap + 1]
  uint32_t* jOffset;         // [maxEvents][cap.jCap + 1]
  uint32_t *cellInner, *cellOuter;   // [maxEvents][cap.cells]
  uint8_t* cellPair;
  int32_t* cellDoubletId;
  uint8_t* cellUsed;
  // cells by outer hit (isOuterHitOfCell), CSR sorted ascending
  uint32_t* ohCount;         // [maxEvents][cap.hits + 1]
  uint32_t* ohOff;           // [maxEvents][cap.hits + 1]
  uint32_t* hitTouch;        // [maxEvents][cap.hits]  CA link ends on cells ending at each hit
  uint32_t* fishHits;        // [maxEvents][cap.hits]  hits with >= 2 such ends (early fishbone work list)
  uint32_t* ohCells;         // [maxEvents][cap.cells]
  float4* ohRec;             // [maxEvents][cap.cells] inner hit of each ohCells entry: x, y, z, +-r (- : dca region inner)
  uint16_t* ohDet;           // [maxEvents][cap.cells] module index of that inner hit
  // CA neighbour links (outerNeighbors), CSR sorted ascending
  uint32_t* nbrCount;        // [maxEvents][cap.cells + 1]
  uint32_t* nbrOff;          // [maxEvents][cap.cells + 1]
  uint32_t* nbr;             // [maxEvents][cap.edges]
  // tuples
  uint32_t* startTupleCount; // [maxEvents][cap.cells + 1]
  uint32_t* startTupleOff;   // [maxEvents][cap.cells + 1]
  uint32_t* startHitCount;   // [maxEvents][cap.cells + 1]
  uint32_t* startHitOff;     // [maxEvents][cap.cells + 1]
  uint32_t* tupleOff;        // [maxEvents][cap.tuples + 1]
  uint32_t* tupleHits;       // [maxEvents][cap.tupleHits()]
  uint16_t* tupleDet;        // [maxEvents][cap.tupleHits()]
  uint32_t* tupleCells;      // [maxEvents][cap.tupleCells()]  (4 slots per tuple)
  uint8_t* quality;          // [maxEvents][cap.tuples]
  // cell -> tracks, CSR sorted ascending
  uint32_t* trkCount;        // [maxEvents][cap.cells + 1]
  uint32_t* trkOff;          // [maxEvents][cap.cells + 1]
  uint32_t* trk;             // [maxEvents][cap.tupleCells()]
  uint32_t* candidates;      // [maxEvents][cap.cells] cells with >= 2 tracks, in no particular order
  // tuple multiplicity
  uint32_t* tmOff;           // [maxEvents][16]
  uint32_t* tmBins;          // [maxEvents][cap.tuples]
  // fit results [maxEvents][cap.tuples * k]
  float *state, *cov, *pt, *eta, *chi2;
  // hit -> tuple
  uint32_t* h2tCount;        // [maxEvents][cap.hits + 1]
  uint32_t* h2tOff;          // [maxEvents][cap.hits + 1]
  uint32_t* h2t;             // [maxEvents][cap.h2t]
  // vertices
  float *zv, *wv, *vchi2, *ptv2;  // [maxEvents][kMaxVtx]
  int32_t* ndof;             // [maxEvents][kMaxVtx]
  uint16_t* sortInd;         // [maxEvents][kMaxVtx]
  int16_t* idv;              // [maxEvents][cap.tuples]
  // scratch: CA link lists before ordering, cleaner state
  uint32_t* scratchA;        // [maxEvents][cap.scratch]
  uint32_t* scratchB;        // [maxEvents][cap.scratch]
  // single-pass scans (scan.cu): per event and scan, a tile ticket and one
  // state word per tile; scanEpoch tags the words of the current batch
  uint64_t* scanState;       // [maxEvents][kScanCalls][scanTiles]
  uint32_t* scanTicket;      // [maxEvents][kScanCalls], cleared by kInitEvents
  uint32_t* scanEpoch;       // [maxEvents], advanced by kInitEvents
  uint32_t scanTiles;        // tiles of the longest scanned array
  uint32_t* bigSeg;          // [maxEvents][kBigSegCap] long segments awaiting the block sort
  uint32_t* segList;         // [maxEvents][cap.cells] segments with >= 2 entries (the ones to order)
};

// A CSR fill notes segment s when it places s's second entry: only those
// segments need ordering.  `list` selects the counter of the list ordering
// that follows the fill (0 cells by outer hit, 1 CA links, 2 tracks per
// cell, 3 tuples per hit); the lists share ws.segList, each consumed before
// the next fill.
__device__ __forceinline__ void noteSegment(const Workspace& ws, uint32_t e, int list, uint32_t s) {
  const uint32_t k = atomicAdd(&ws.ev[e].nSegList[list], 1u);
  ws.segList[size_t(e) * ws.cap.cells + k] = s;
}

// ---------------------------------------------------------------- kernel timing probe
// While a probe is installed on the launching host thread, every launch whose
// kernel name matches (or every launch, for "*") is bracketed by a pair of
// timing events on its stream.  Under stream capture the event records
// become graph nodes, so each replay of the graph re-times the kernel.
constexpr uint32_t kProbeMax = 256;
struct KernelProbe {
  char name[64];                 // kernel name, "*" for all
  cudaEvent_t ev[2 * kProbeMax];
  const char* launched[kProbeMax];
  uint32_t used;                 // pairs recorded by the launch sequence
};
extern thread_local KernelProbe* tProbe;
void probeBegin(const char* name, cudaStream_t s);
void probeEnd(cudaStream_t s);
#define PG_PROBED(name, stream, ...)                         \
  do {                                                       \
    const bool pgProbeOn_ = tProbe != nullptr;               \
    if (pgProbeOn_) probeBegin(name, stream);                \
    __VA_ARGS__;                                             \
    if (pgProbeOn_) probeEnd(stream);                        \
  } while (0)

// ---------------------------------------------------------------- launch API (host)
size_t workspaceBytes(uint32_t maxEvents, uint32_t wordCap, const Caps& cap);
void workspaceCarve(Workspace& ws, void* base, uint32_t maxEvents, uint32_t wordCap, const Caps& cap);

// Batches up to this many events run the per-event cooperative kernels
// (result packing, duplicate rounds, vertexing) as clusters of several CTAs
// per event, for latency; larger batches give each event one CTA, which
// leaves the other SMs to the concurrently running batch.
constexpr uint32_t kClusterMaxEvents = 16;

// Launch of kernel k on a grid of (x, nEvents) CTAs grouped in clusters of x
// CTAs along the first dimension.
template <typename... KArgs, typename... Args>
cudaError_t launchClustered(void (*k)(KArgs...), uint32_t x, uint32_t nEvents, uint32_t threads, size_t smem,
                            cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(x, nEvents);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = x;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, KArgs(args)...);
}

// Runs the whole chain on events [0, nEvents) of ws, on `stream`.  The
// word/fedId/offset inputs must already be in ws.  Returns a CUDA error code.
// riemann: the Riemann fit in place of the broken-line fit (useRiemannFit);
// vertexAlgo: the vertex clusterer (runVertices)
cudaError_t runChain(const DeviceES& es, Workspace& ws, uint32_t nEvents, cudaStream_t stream, bool riemann = false,
                     int vertexAlgo = 0);
// Individual stages (used by runChain and by the stage-level tests)
cudaError_t runLocal(const DeviceES& es, Workspace& ws, uint32_t nEvents, cudaStream_t stream);
// countModules + findClus + clusterChargeCut on digis already in ws
cudaError_t runClusters(Workspace& ws, uint32_t nEvents, cudaStream_t stream);
cudaError_t runCA(const DeviceES& es, Workspace& ws, uint32_t nEvents, cudaStream_t stream);
cudaError_t runFits(const DeviceES& es, Workspace& ws, uint32_t nEvents, cudaStream_t stream, bool riemann = false);
// algo: 0 clusterTracksByDensity (default), 1 clusterTracksDBSCAN, 2 clusterTracksIterative
cudaError_t runVertices(Workspace& ws, uint32_t nEvents, cudaStream_t stream, int algo = 0);
cudaError_t runCleaners(Workspace& ws, uint32_t nEvents, cudaStream_t stream);

// batch input descriptor and compact results (k_pack.cu)
void launchSetInput(Workspace& ws, const uint32_t* words, const uint8_t* fedIds, cudaStream_t s);
// grid x-extent of a tunable launch
inline uint32_t tunedGrid(const Workspace& ws, TuneId id, uint32_t base) {
  const int s = ws.tune.scale[id];
  uint64_t g = s >= 0 ? uint64_t(base) << s : uint64_t(base) >> (-s);
  return uint32_t(g < 1 ? 1 : (g > 65535 ? 65535 : g));
}

// device FED scan: wordOffsets, words and fedIds of the batch from ws.scan
void launchFedScan(Workspace& ws, uint32_t nEvents, cudaStream_t stream);
void launchPack(Workspace& ws, uint32_t nEvents, uint8_t* out, cudaStream_t s);

// batched segmented exclusive scan: out[e*stride + i] = sum_{k<i} in[e*stride + k]
// for i <= n_e, where n_e = lenPtr[e*lenStride] (device) or maxLen when lenPtr is
// null; n_e <= maxLen.  The total lands at out[e*stride + n_e] and, if totalPtr,
// at totalPtr[e*totalStride].  in may equal out unless zeroIn, which leaves
// in[0..n_e) zero (the count arrays are reused as fill cursors).  `call`
// selects the scan's state region (one per scan of a batch).
void segScan(const Workspace& ws, ScanCall call, uint32_t* in, uint32_t* out, uint32_t stride,
             const uint32_t* lenPtr, uint32_t lenStride, uint32_t maxLen, uint32_t* totalPtr, uint32_t totalStride,
             uint32_t nEvents, cudaStream_t stream, bool zeroIn = false);
// Two such scans of arrays with the same lengths and stride in one launch.
void segScan2(const Workspace& ws, ScanCall call0, uint32_t* in0, uint32_t* out0, uint32_t* total0, ScanCall call1,
              uint32_t* in1, uint32_t* out1, uint32_t* total1, uint32_t stride, const uint32_t* lenPtr,
              uint32_t lenStride, uint32_t maxLen, uint32_t totalStride, uint32_t nEvents, cudaStream_t stream,
              bool zeroIn = false);

}  // namespace pixgpu
