// Cellular automaton on B200: doublets, isOuterHitOfCell lists, CA links,
// early fishbone, n-tuplet search, cell->track lists, duplicate removers,
// tuple multiplicity, classification and the hit->tuple cleaner.
//
// Reference behaviour followed (src/serial paths):
//   doubletsFromHisto        plugin-PixelTriplets/gpuPixelDoubletsAlgos.h:25-238 (+ gpuPixelDoublets.h:14-66)
//   kernel_connect           plugin-PixelTriplets/CAHitNtupletGeneratorKernelsImpl.h:191-262
//                            with GPUCACell::areAlignedRZ/dcaCut (GPUCACell.h:175-206), CircleEq.h:23-107
//   fishbone (early)         plugin-PixelTriplets/gpuFishbone.h:21-90
//   kernel_find_ntuplets     CAHitNtupletGeneratorKernelsImpl.h:264-292, GPUCACell.h:278-331
//   finalizeBulk             CUDACore/HistoContainer.h:193-204
//   earlyDuplicateRemover, count/fillMultiplicity, fillHitDetIndices, classifyTracks,
//   fastDuplicateRemover, count/fillHitInTracks, tripletCleaner   CAHitNtupletGeneratorKernelsImpl.h
//   configuration            CAHitNtupletGeneratorOnGPU.cc:21-65
//
// Serial order is reproduced exactly: doublets are numbered by a count/scan/
// write pass over (layer pair, inner hit, phi window, bin content), every
// per-object list is built by counting sort and then ordered per segment, the
// DFS numbers tuples by prefix sums over starting cells, and the one
// order-dependent cleaner (fastDuplicateRemover) runs as rounds over the
// dependency graph of cells that share a track.
#include <cooperative_groups.h>

#include "device_utils.cuh"
#include "segsort.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

constexpr int kNPairs = 19;
__constant__ uint8_t cLayerPairs[2 * kNPairs] = {0, 1, 0, 4, 0, 7, 1, 2, 1, 4, 1, 7, 4, 5, 7, 8, 2, 3, 2, 4,
                                                 2, 7, 5, 6, 8, 9, 0, 2, 1, 3, 0, 5, 0, 8, 4, 6, 7, 9};
__constant__ int16_t cPhiCuts[kNPairs] = {522, 730, 730, 522, 626, 626, 522, 522, 626, 626,
                                          626, 522, 522, 522, 522, 522, 522, 522, 522};
__constant__ float cMinZ[kNPairs] = {-20., 0., -30., -22., 10., -30., -70., -70., -22., 15.,
                                     -30,  -70., -70., -20., -22., 0,   -30., -70., -70.};
__constant__ float cMaxZ[kNPairs] = {20., 30., 0., 22., 30., -10., 70., 70., 22., 30.,
                                     -15., 70., 70., 20., 22., 30., 0., 70., 70.};
__constant__ float cMaxR[kNPairs] = {20., 9., 9., 20., 7., 7., 5., 5., 20., 6., 6., 5., 5., 20., 20., 9., 9., 9., 9.};

constexpr float kPtMin = 0.899999976158f;
constexpr float kThetaCutBarrel = 0.00200000009499f;
constexpr float kThetaCutForward = 0.00300000002608f;
constexpr float kHardCurvCut = 0.0328407224959f;
constexpr float kDcaCutInner = 0.15000000596f;
constexpr float kDcaCutOuter = 0.25f;
constexpr uint8_t kBad = 0, kDup = 1, kLoose = 2;
// "no tuple" in the duplicate removers (the reference's 60000 lies above every
// index of its 32768 bins; with 32-bit tuple indices a larger one is needed)
constexpr uint32_t kNoTuple = 0xffffffffu;

__device__ __forceinline__ uint32_t phiBin(int16_t t) { return uint32_t((int(t) >> 9) & 127); }

struct HitsView {
  const float *xg, *yg, *zg, *rg;
  const int16_t *iphi, *ysize;
  const uint16_t* detInd;
  const uint32_t* phiOff;
  const uint32_t* phiBins;
};
__device__ __forceinline__ HitsView hitsOf(const Workspace& ws, uint32_t e) {
  size_t hb = size_t(e) * ws.cap.hits;
  return {ws.xg + hb, ws.yg + hb, ws.zg + hb, ws.rg + hb, ws.iphi + hb, ws.ysize + hb, ws.detInd + hb,
          ws.phiOff + size_t(e) * kPhiStride, ws.phiBins + hb};
}

// ------------------------------------------------------------------ doublets

__global__ void kDoubletSetup(Workspace ws, uint32_t nEvents) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nEvents) return;
  EventCounters* c = ws.ev + e;
  uint32_t cum = 0;
  if (c->nHits == 0) {
    for (int p = 0; p < kNPairs; ++p) c->pairCum[p] = 0;
    c->ntot = 0;
    return;
  }
  for (uint32_t p = 0; p < uint32_t(kNPairs); ++p) {
    uint8_t li = cLayerPairs[2 * p];
    if (p < ws.ca.nPairs) cum += c->layerStart[li + 1] - c->layerStart[li];
    c->pairCum[p] = cum;  // pairs beyond nPairs own no slots
  }
  if (cum > ws.cap.jCap) {
    c->flags |= kFlagJOverflow;
    cum = ws.cap.jCap;
  }
  c->ntot = cum;
}

// Doublet search for inner-hit slot j (gpuPixelDoubletsAlgos.h:25-238 with
// the PixelTriplets defaults): the per-inner-hit cuts, then the outer layer's
// phi window as one or two contiguous ranges of the phi histogram.  The
// serial order of the candidates is the window's bin order with each bin's
// stored order, i.e. the order of these ranges.
struct DoubletSeed {
  uint32_t cuts;  // bit 0 z0 cut, bit 1 cluster-size cut, bit 2 pt cut
  uint32_t pair, inner, outer, i;
  float mez, mer;
  int16_t mep, mes, iphicut;
  float maxr;
  uint32_t b0, e0, b1, e1;  // candidate ranges in phiBins
};

// per-event layer offsets staged in shared memory by each block, with the
// CA configuration
struct PairTable {
  uint32_t pairCum[kNPairs];
  uint32_t layerStart[11];
  CAConfig ca;
};

__device__ __forceinline__ void loadPairTable(const EventCounters* c, PairTable& t, const CAConfig& ca) {
  if (threadIdx.x < kNPairs) t.pairCum[threadIdx.x] = c->pairCum[threadIdx.x];
  if (threadIdx.x < 11) t.layerStart[threadIdx.x] = c->layerStart[threadIdx.x];
  if (threadIdx.x == 0) t.ca = ca;
  __syncthreads();
}

__device__ __forceinline__ bool doubletSeed(const PairTable& c, const HitsView& hh, uint32_t j, DoubletSeed& d,
                                            uint32_t* near = nullptr) {
  uint32_t pair = 0;
  while (j >= c.pairCum[pair]) ++pair;
  const uint8_t inner = cLayerPairs[2 * pair], outer = cLayerPairs[2 * pair + 1];
  uint32_t i = (0 == pair) ? j : j - c.pairCum[pair - 1];
  i += c.layerStart[inner];
  d.cuts = (c.ca.doZ0Cut ? 1u : 0u) | (c.ca.doClusterCut ? 2u : 0u) | (c.ca.doPtCut ? 4u : 0u);
  d.pair = pair;
  d.inner = inner;
  d.outer = outer;
  d.i = i;
  if (hh.detInd[i] > 2000) return false;
  d.mez = hh.zg[i];
  if (near) *near += cutNear(d.mez, cMinZ[pair]) + cutNear(d.mez, cMaxZ[pair]);
  if (d.mez < cMinZ[pair] || d.mez > cMaxZ[pair]) return false;
  d.mes = -1;
  if (c.ca.doClusterCut) {
    const bool isOuterLadder = c.ca.idealConditions ? true : 0 == (hh.detInd[i] / 8) % 2;
    d.mes = inner > 0 || isOuterLadder ? hh.ysize[i] : int16_t(-1);
    if (inner == 0 && outer > 3)
      if (d.mes > 0 && d.mes < 36) return false;
    if (inner == 1 && outer > 3)
      if (d.mes > 0 && d.mes < 28) return false;
  }
  d.mep = hh.iphi[i];
  d.mer = hh.rg[i];
  d.iphicut = cPhiCuts[pair];
  d.maxr = cMaxR[pair];
  const uint32_t kl = phiBin(int16_t(d.mep - d.iphicut)), kh = phiBin(int16_t(d.mep + d.iphicut));
  const uint32_t khh = (kh + 1) & 127;
  const uint32_t* off = hh.phiOff + 128 * outer;
  d.b0 = d.e0 = d.b1 = d.e1 = 0;
  if (kl == khh) return false;  // the serial bin loop runs no iteration
  if (kl <= kh) {
    d.b0 = off[kl];
    d.e0 = off[kh + 1];
  } else {
    d.b0 = off[kl];
    d.e0 = off[128];
    d.b1 = off[0];
    d.e1 = off[kh + 1];
  }
  return true;
}

// candidate test on a packed hit record (kPhiRec layout); with `near`, the
// float cuts evaluated that lie on their boundary are counted
template <bool kNear = false>
__device__ __forceinline__ bool doubletAccept(const DoubletSeed& d, const uint4 rec, uint32_t& near) {
  constexpr float z0cut = 12.f;
  constexpr float minRadius = 0.5f * 87.78f;
  constexpr float minRadius2T4 = 4.f * minRadius * minRadius;
  constexpr float dzdrFact = 8 * 0.0285 / 0.015;
  constexpr float i2p = 3.14159265358979323846 / 32768;
  if ((rec.w & 0x7ffu) > 2000) return false;
  const float zo = __uint_as_float(rec.x), ro = __uint_as_float(rec.y);
  const float dr = ro - d.mer;
  if (d.cuts & 1u) {
    if (kNear) near += cutNear(dr, d.maxr);
    if (dr > d.maxr || dr < 0) return false;
    if (kNear) near += cutNear(fabsf((d.mez * ro - d.mer * zo)), z0cut * dr);
    if (fabsf((d.mez * ro - d.mer * zo)) > z0cut * dr) return false;
  }
  const int16_t mop = int16_t(rec.z & 0xffffu);
  const uint16_t idphi = uint16_t(min(abs(int(int16_t(mop - d.mep))), abs(int(int16_t(d.mep - mop)))));
  if (idphi > d.iphicut) return false;
  const int16_t so = int16_t(rec.z >> 16);
  const bool cut = (d.outer < 4) ? (d.mes > 0 && so > 0 && abs(so - d.mes) > (d.inner == 0 ? 28 : 20))
                                 : ((d.inner < 4) && d.mes > 0 &&
                                    abs(d.mes - int(fabsf((d.mez - zo) / (d.mer - ro)) * dzdrFact + 0.5f)) > 20);
  if ((d.cuts & 2u) && cut) return false;
  const float dphi = float(short(idphi)) * i2p;
  if (d.cuts & 4u) {
    if (kNear) near += cutNear(dphi * dphi * (minRadius2T4 - d.mer * ro), (ro - d.mer) * (ro - d.mer));
    if (dphi * dphi * (minRadius2T4 - d.mer * ro) > (ro - d.mer) * (ro - d.mer)) return false;
  }
  return true;
}

// One warp per inner-hit slot: lanes test consecutive candidates of the
// window; the ballots give the count (pass 1) and the serial positions
// (pass 2).  F(position among the slot's doublets, outer hit).
template <bool kNear = false, typename F>
__device__ __forceinline__ uint32_t warpDoublets(const DoubletSeed& d, const uint4* rec, F&& f, uint32_t* near = nullptr) {
  uint32_t nearLane = 0;
  const uint32_t lane = laneId();
  uint32_t n = 0;
  for (int r = 0; r < 2; ++r) {
    const uint32_t b = r ? d.b1 : d.b0, en = r ? d.e1 : d.e0;
    for (uint32_t p0 = b; p0 < en; p0 += 32) {
      const uint32_t p = p0 + lane;
      uint32_t oi = 0;
      bool ok = false;
      if (p < en) {
        const uint4 h = rec[p];
        oi = h.w >> 11;
        ok = doubletAccept<kNear>(d, h, nearLane);
      }
      const uint32_t m = __ballot_sync(0xffffffffu, ok);
      if (ok) f(n + __popc(m & lanemaskLt()), oi);
      n += __popc(m);
    }
  }
  if (kNear) *near += nearLane;
  return n;
}

// Each warp looks at 32 slots at once: every lane evaluates one slot's seed
// cuts, then the warp walks the candidate ranges of the surviving slots one
// after the other.  Warp w takes slots w, w + S, w + 2S, ... (S warps per
// event), so that dense runs of consecutive slots spread over the warps.
template <typename PerSlot>
__device__ __forceinline__ void forSeedSlots(const PairTable& pt, const HitsView& hh, uint32_t ntot,
                                             PerSlot&& perSlot, uint32_t* near) {
  const uint32_t lane = laneId(), wpb = blockDim.x >> 5;
  const uint32_t S = gridDim.x * wpb, w = blockIdx.x * wpb + (threadIdx.x >> 5);
  for (uint32_t r0 = 0; w + r0 * S < ntot; r0 += 32) {
    const uint32_t j = w + (r0 + lane) * S;
    DoubletSeed d;
    const bool live = j < ntot && doubletSeed(pt, hh, j, d, near) && (d.e0 > d.b0 || d.e1 > d.b1);
    uint32_t m = __ballot_sync(0xffffffffu, live);
    perSlot(j, live, d, 0u);  // every lane sees its own slot first
    while (m) {
      const int l = __ffs(m) - 1;
      m &= m - 1;
      DoubletSeed ds;
      ds.cuts = __shfl_sync(0xffffffffu, d.cuts, l);
      ds.pair = __shfl_sync(0xffffffffu, d.pair, l);
      ds.inner = __shfl_sync(0xffffffffu, d.inner, l);
      ds.outer = __shfl_sync(0xffffffffu, d.outer, l);
      ds.i = __shfl_sync(0xffffffffu, d.i, l);
      ds.mez = __shfl_sync(0xffffffffu, d.mez, l);
      ds.mer = __shfl_sync(0xffffffffu, d.mer, l);
      ds.mep = int16_t(__shfl_sync(0xffffffffu, int(d.mep), l));
      ds.mes = int16_t(__shfl_sync(0xffffffffu, int(d.mes), l));
      ds.iphicut = int16_t(__shfl_sync(0xffffffffu, int(d.iphicut), l));
      ds.maxr = __shfl_sync(0xffffffffu, d.maxr, l);
      ds.b0 = __shfl_sync(0xffffffffu, d.b0, l);
      ds.e0 = __shfl_sync(0xffffffffu, d.e0, l);
      ds.b1 = __shfl_sync(0xffffffffu, d.b1, l);
      ds.e1 = __shfl_sync(0xffffffffu, d.e1, l);
      perSlot(w + (r0 + uint32_t(l)) * S, true, ds, 1u + uint32_t(l));
    }
  }
}

constexpr uint32_t kNoTemp = 0xffffffffu;  // the slot's doublets did not fit its warp's staging region

// Pass 1: count each slot's doublets and stage their outer hits, in serial
// order, in the staging region of the warp that found them (scratchA, an
// equal share per warp: no atomics); the slot's staging
// offset goes to scratchB.  A slot whose window could overflow the region is
// only counted, and pass 2 tests its candidates again.
// (256, 4): 76 -> 64 registers, four blocks per SM instead of three; measured
// A/B at 64 PU50 events per batch, three in flight: 671 -> 598 us, +1.5 % events/s
__global__ void __launch_bounds__(256, 4) kDoubletCount(Workspace ws) {
  __shared__ PairTable pt;
  const uint32_t e = blockIdx.y;
  const EventCounters* c = ws.ev + e;
  const uint32_t ntot = c->ntot;
  loadPairTable(c, pt, ws.ca);
  const HitsView hh = hitsOf(ws, e);
  const uint4* rec = ws.phiRec + size_t(e) * ws.cap.hits;
  uint32_t* cnt = ws.jCount + size_t(e) * (ws.cap.jCap + 1);
  uint32_t* stage = ws.scratchA + size_t(e) * ws.cap.scratch;
  uint32_t* slotStage = ws.scratchB + size_t(e) * ws.cap.scratch;
  const uint32_t wpb = blockDim.x >> 5;
  const uint32_t S = gridDim.x * wpb, w = blockIdx.x * wpb + (threadIdx.x >> 5);
  const uint32_t R = ws.cap.scratch / S;  // staging entries per warp
  uint32_t used = 0;                     // warp-uniform
  uint32_t near = 0;                     // per lane: cut decisions on their boundary
  forSeedSlots(pt, hh, ntot, [&](uint32_t j, bool live, const DoubletSeed& d, uint32_t phase) {
    if (phase == 0) {
      if (j < ntot && !live) cnt[j] = 0;
      return;
    }
    const uint32_t window = (d.e0 - d.b0) + (d.e1 - d.b1);
    const uint32_t at = used + window <= R ? w * R + used : kNoTemp;
    const uint32_t n = warpDoublets<true>(d, rec, [&](uint32_t k, uint32_t oi) {
      if (at != kNoTemp) stage[at + k] = oi;
    }, &near);
    if (at != kNoTemp) used += n;
    if (laneId() == phase - 1) {
      cnt[j] = n;
      slotStage[j] = at;
    }
  }, &near);
  near = __reduce_add_sync(0xffffffffu, near);
  if (laneId() == 0 && near) atomicAdd(&ws.ev[e].nearDoublet, near);
}

// Pass 2: each slot's doublets from its staging entries to their serial
// positions (the scan of the counts); slots that were not staged are found
// again.  Lanes take 32 slots, the warp serves the non-empty ones in turn.
__global__ void __launch_bounds__(256, 5) kDoubletWrite(Workspace ws) {
  __shared__ PairTable pt;
  const uint32_t e = blockIdx.y;
  const EventCounters* c = ws.ev + e;
  const uint32_t ntot = c->ntot;
  loadPairTable(c, pt, ws.ca);
  const HitsView hh = hitsOf(ws, e);
  const uint4* rec = ws.phiRec + size_t(e) * ws.cap.hits;
  const uint32_t* off = ws.jOffset + size_t(e) * (ws.cap.jCap + 1);
  const size_t cb = size_t(e) * ws.cap.cells;
  uint32_t* ohc = ws.ohCount + size_t(e) * (ws.cap.hits + 1);
  const uint32_t* stage = ws.scratchA + size_t(e) * ws.cap.scratch;
  const uint32_t* slotStage = ws.scratchB + size_t(e) * ws.cap.scratch;
  const uint32_t lane = laneId(), wpb = blockDim.x >> 5;
  const uint32_t S = gridDim.x * wpb, w = blockIdx.x * wpb + (threadIdx.x >> 5);
  for (uint32_t r0 = 0; w + r0 * S < ntot; r0 += 32) {
    const uint32_t jl = w + (r0 + lane) * S;
    uint32_t myBase = 0, myN = 0, myAt = kNoTemp, myI = 0, myPair = 0;
    if (jl < ntot) {
      myBase = off[jl];
      myN = myBase < ws.cap.cells ? min(off[jl + 1], ws.cap.cells) - myBase : 0u;
    }
    if (myN) {
      myAt = slotStage[jl];
      while (jl >= pt.pairCum[myPair]) ++myPair;
      myI = (0 == myPair ? jl : jl - pt.pairCum[myPair - 1]) + pt.layerStart[cLayerPairs[2 * myPair]];
    }
    auto put = [&](uint32_t idx, uint32_t i, uint32_t pair, uint32_t oi) {
      ws.cellInner[cb + idx] = i;
      ws.cellOuter[cb + idx] = oi;
      ws.cellPair[cb + idx] = uint8_t(pair);
      ws.cellDoubletId[cb + idx] = int32_t(idx);
      ws.cellUsed[cb + idx] = 0;
      atomicAdd(&ohc[oi], 1u);
    };
    // The staged slots' doublets as one flat range over the warp's 32 slots,
    // so that all lanes copy (a slot holds a few doublets): the lane of flat
    // entry f is found by a binary search over the lanes' inclusive ends.
    const uint32_t cnt = myAt != kNoTemp ? myN : 0u;
    const uint32_t incl = warpInclusiveScan(cnt), excl = incl - cnt;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t f0 = 0; f0 < total; f0 += 32) {
      const uint32_t f = f0 + lane;
      uint32_t l = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t v = __shfl_sync(0xffffffffu, incl, l + step - 1);
        if (v <= f) l += step;
      }
      l &= 31u;  // lanes past the range (f >= total) land on 32; they only read
      const uint32_t b = __shfl_sync(0xffffffffu, myBase, l), at = __shfl_sync(0xffffffffu, myAt, l);
      const uint32_t x = __shfl_sync(0xffffffffu, excl, l), i = __shfl_sync(0xffffffffu, myI, l);
      const uint32_t pair = __shfl_sync(0xffffffffu, myPair, l);
      if (f < total) {
        const uint32_t k = f - x;
        put(b + k, i, pair, stage[at + k]);
      }
    }
    // slots whose doublets did not fit the count pass's staging: found again
    uint32_t redo = __ballot_sync(0xffffffffu, myN > 0 && myAt == kNoTemp);
    while (redo) {
      const int l = __ffs(redo) - 1;
      redo &= redo - 1;
      const uint32_t j = w + (r0 + uint32_t(l)) * S;
      const uint32_t base = __shfl_sync(0xffffffffu, myBase, l), n = __shfl_sync(0xffffffffu, myN, l);
      const uint32_t i = __shfl_sync(0xffffffffu, myI, l), pair = __shfl_sync(0xffffffffu, myPair, l);
      DoubletSeed d;
      doubletSeed(pt, hh, j, d);
      warpDoublets(d, rec, [&](uint32_t k, uint32_t oi) {
        if (k < n) put(base + k, i, pair, oi);
      });
    }
  }
}

__global__ void kCellsTotal(Workspace ws, uint32_t nEvents) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nEvents) return;
  EventCounters* c = ws.ev + e;
  uint32_t raw = ws.jOffset[size_t(e) * (ws.cap.jCap + 1) + c->ntot];
  c->nCellsRaw = raw;
  c->nCells = min(raw, ws.cap.cells);
  if (raw >= ws.cap.cells) c->flags |= kFlagCellOverflow;
}

// generic CSR helpers ------------------------------------------------------

// zero n entries of each event's array
__global__ void kZero(uint32_t* p, size_t stride, uint32_t n, const uint32_t* lenPtr, uint32_t lenStride) {
  uint32_t e = blockIdx.y;
  uint32_t len = lenPtr ? min(n, lenPtr[size_t(e) * lenStride] + 1) : n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
    p[size_t(e) * stride + i] = 0;
}

// isOuterHitOfCell fill (unordered; lists longer than 128 are ordered after)
__global__ void kOuterHitFill(Workspace ws) {
  uint32_t e = blockIdx.y;
  uint32_t n = ws.ev[e].nCells;
  size_t cb = size_t(e) * ws.cap.cells;
  const uint32_t* off = ws.ohOff + size_t(e) * (ws.cap.hits + 1);
  uint32_t* cur = ws.ohCount + size_t(e) * (ws.cap.hits + 1);
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    uint32_t oi = ws.cellOuter[cb + c];
    uint32_t p = atomicAdd(&cur[oi], 1u);
    ws.ohCells[cb + off[oi] + p] = c;
    // connect and fishbone read the first 128 cells of a hit (ascending):
    // only longer lists need ordering here; fishbone orders the rest itself
    if (p == PF_MAX_CELLS_PER_HIT) noteSegment(ws, e, 0, oi);
  }
}

// ------------------------------------------------------------------ connect

// GPUCACell::areAlignedRZ, single-precision part: false only for pairs that
// fail the cut by a margin far above rounding (the squared inequality in
// float with a relative margin of 1e-4; NaN operands, and right-hand sides
// small enough for the squares to lose precision as subnormals, pass on to
// the exact test)
__device__ __forceinline__ bool alignedRZMaybe(float r1, float z1, float ri, float zi, float ro, float zo,
                                               float thetaCut) {
  float radius_diff = fabsf(r1 - ro);
  float distance_13_squared = radius_diff * radius_diff + (z1 - zo) * (z1 - zo);
  const float area = z1 * (ri - ro) + zi * (ro - r1) + zo * (r1 - ri);
  const float rhs = thetaCut * distance_13_squared * radius_diff;
  return !(rhs > 1e-15f && area * area * (kPtMin * kPtMin) * distance_13_squared > 1.0001f * rhs * rhs);
}

// GPUCACell::areAlignedRZ: fabs(float) binds to the double overload in the
// serial build, so the left-hand product is formed in double precision.
// Pairs the single-precision part drops lie far from the boundary and are
// not counted as near it.
__device__ __forceinline__ bool alignedRZ(float r1, float z1, float ri, float zi, float ro, float zo, float thetaCut,
                                          uint32_t& near) {
  if (!alignedRZMaybe(r1, z1, ri, zi, ro, zo, thetaCut)) return false;
  float radius_diff = fabsf(r1 - ro);
  float distance_13_squared = radius_diff * radius_diff + (z1 - zo) * (z1 - zo);
  const float area = z1 * (ri - ro) + zi * (ro - r1) + zo * (r1 - ri);
  const float rhs = thetaCut * distance_13_squared * radius_diff;
  float pMin = kPtMin * sqrtf(distance_13_squared);
  double lhs = fabs(double(area));
  near += cutNear(lhs * double(pMin), double(rhs));
  return lhs * double(pMin) <= double(rhs);
}

__device__ __forceinline__ bool dcaCut(float x1, float y1, float x2, float y2, float x3, float y3, float region,
                                       uint32_t& near) {
  bool noflip = fabsf(x3 - x1) < fabsf(y3 - y1);
  float x1p = noflip ? x1 - x2 : y1 - y2;
  float y1p = noflip ? y1 - y2 : x1 - x2;
  float d12 = x1p * x1p + y1p * y1p;
  float x3p = noflip ? x3 - x2 : y3 - y2;
  float y3p = noflip ? y3 - y2 : x3 - x2;
  float d32 = x3p * x3p + y3p * y3p;
  float num = x1p * y3p - y1p * x3p;
  float det = d12 * y3p - d32 * y1p;
  float st2 = (d12 * x3p - d32 * x1p);
  float seq = det * det + st2 * st2;
  float al2 = 1.f / sqrtf(seq);
  float be2 = -st2 * al2;
  float ct = 2.f * num * al2;
  al2 *= det;
  float cc = noflip ? ct : -ct;
  float alpha = noflip ? al2 : -be2;
  float beta = noflip ? be2 : -al2;
  near += cutNear(cc, kHardCurvCut);
  if (cc > kHardCurvCut) return false;
  float xx = cc * x2 + alpha;
  float yy = cc * y2 + beta;
  float dca0 = sqrtf(xx * xx + yy * yy) - 1.f;
  near += cutNear(fabsf(dca0), region * fabsf(cc));
  return fabsf(dca0) < region * fabsf(cc);
}

// inner-hit coordinates of every ohCells entry, in ohCells order, so that
// kConnect reads the candidate cells of a hit as one contiguous range; the
// sign of r carries the dca region of the candidate (negative: innermost
// barrel layer, dca cut 0.15 instead of 0.25)
__global__ void kOhRec(Workspace ws) {
  const uint32_t e = blockIdx.y;
  const uint32_t n = ws.ev[e].nCells;
  const size_t cb = size_t(e) * ws.cap.cells, hb = size_t(e) * ws.cap.hits;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t oc = ws.ohCells[cb + p];
    const uint32_t ih = ws.cellInner[cb + oc];
    const float r = ws.rg[hb + ih];
    const uint16_t det = ws.detInd[hb + ih];
    ws.ohRec[cb + p] = make_float4(ws.xg[hb + ih], ws.yg[hb + ih], ws.zg[hb + ih], det < 96 ? -r : r);
    ws.ohDet[cb + p] = det;
  }
}

// kernel_connect (CAHitNtupletGeneratorKernelsImpl.h:191-262) by doublet
// slot: the cells of slot j share their inner hit h, so they share the
// candidate list (cells ending on h, first 128 in ascending order).  A warp
// looks at 32 slots at once (warp w: slots w, w + S, ...) and takes the
// non-empty ones in turn; for a slot, lane t stages the outer hit of cell t
// and the warp takes the slot's (cell, candidate) pairs flat, 32 at a time,
// so short candidate lists still keep the lanes busy.
// Only about 2 % of the pairs pass the r-z alignment test, so only its
// single-precision part runs on every pair; the pairs it keeps are queued
// (per warp, in shared memory), and the exact r-z test (double precision,
// with its margin count) and the dca test run on 32 queued pairs at a time,
// every lane busy, instead of on every round that has one surviving lane.
// Accepted links (oc <- idx) are appended unordered with one atomic per warp
// and round.
constexpr uint32_t kConnectWarps = 8;   // 256 threads
constexpr uint32_t kConnectQueue = 64;  // ring of queued pairs per warp (a round adds at most 32)
__global__ void __launch_bounds__(kConnectWarps * 32, 5) kConnect(Workspace ws, uint32_t* edgeOc, uint32_t* edgeIdx) {
  // queued pair: ohRec/ohCells position of the candidate, the cell, the
  // slot's inner hit and the cell's outer hit
  __shared__ uint4 queueA[kConnectWarps][kConnectQueue];
  const uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  const uint32_t ntot = c->ntot;
  const uint32_t nCells = c->nCells;
  const HitsView hh = hitsOf(ws, e);
  const size_t cb = size_t(e) * ws.cap.cells;
  const uint32_t* joff = ws.jOffset + size_t(e) * (ws.cap.jCap + 1);
  const uint32_t* ohOff = ws.ohOff + size_t(e) * (ws.cap.hits + 1);
  const uint32_t* ohCells = ws.ohCells + cb;
  const float4* ohRec = ws.ohRec + cb;
  uint32_t* nbrCnt = ws.nbrCount + size_t(e) * (ws.cap.cells + 1);
  uint32_t* eOc = edgeOc + size_t(e) * ws.cap.scratch;
  uint32_t* eIdx = edgeIdx + size_t(e) * ws.cap.scratch;
  const uint32_t edgeCap = min(ws.cap.edges, ws.cap.scratch);
  const uint32_t lane = laneId(), wpb = blockDim.x >> 5;
  const uint32_t S = gridDim.x * wpb, w = blockIdx.x * wpb + (threadIdx.x >> 5);
  uint4* queue = queueA[threadIdx.x >> 5];
  uint32_t qHead = 0, qTail = 0;  // warp-uniform ring positions
  uint32_t near = 0;              // per lane: cut decisions on their boundary
  // dca test of the nq (<= 32) oldest queued pairs, one per lane
  auto drain = [&](uint32_t nq) {
    __syncwarp();
    bool ok = false;
    uint32_t p = 0, idx = 0;
    if (lane < nq) {
      const uint4 qe = queue[(qHead + lane) & (kConnectQueue - 1)];
      p = qe.x;
      idx = qe.y;
      const float4 r1 = ohRec[p];
      const float ri = hh.rg[qe.z], zi = hh.zg[qe.z];  // the slot's inner hit
      const float thetaCut = hh.detInd[qe.z] < 1184 ? kThetaCutBarrel : kThetaCutForward;
      const float region = r1.w < 0.f ? kDcaCutInner : kDcaCutOuter;
      ok = alignedRZ(fabsf(r1.w), r1.z, ri, zi, hh.rg[qe.w], hh.zg[qe.w], thetaCut, near) &&
           dcaCut(r1.x, r1.y, hh.xg[qe.z], hh.yg[qe.z], hh.xg[qe.w], hh.yg[qe.w], region, near);
    }
    qHead += nq;
    const uint32_t mask = __ballot_sync(0xffffffffu, ok);
    if (mask) {
      uint32_t at = 0;
      if (lane == 0) at = atomicAdd(&c->nEdges, uint32_t(__popc(mask)));
      at = __shfl_sync(0xffffffffu, at, 0);
      if (ok) {
        const uint32_t oc = ohCells[p];
        ws.cellUsed[cb + idx] = 1;
        ws.cellUsed[cb + oc] = 1;
        atomicAdd(&nbrCnt[oc], 1u);
        const uint32_t slot = at + __popc(mask & lanemaskLt());
        if (slot < edgeCap) {
          eOc[slot] = oc;
          eIdx[slot] = idx;
        } else {
          atomicOr(&c->flags, kFlagEdgeOverflow);
        }
      }
    }
    __syncwarp();  // the entries are read before the next round overwrites them
  };
  for (uint32_t r0 = 0; w + r0 * S < ntot; r0 += 32) {
    // each lane sets up one slot (its inner hit and that hit's r, z and
    // cut), so that the warp's loads for 32 slots overlap
    const uint32_t jl = w + (r0 + lane) * S;
    uint32_t myBase = 0, myEnd = 0, myOb = 0, myM = 0, myH = 0;
    float myRi = 0.f, myZi = 0.f, myTheta = 0.f, myInvM = 0.f;
    if (jl < ntot) {
      myBase = joff[jl];
      myEnd = min(joff[jl + 1], nCells);
      if (myBase < myEnd) {
        myH = ws.cellInner[cb + myBase];
        myOb = ohOff[myH];
        myM = min(ohOff[myH + 1] - myOb, uint32_t(PF_MAX_CELLS_PER_HIT));
        myRi = hh.rg[myH];
        myZi = hh.zg[myH];
        myTheta = hh.detInd[myH] < 1184 ? kThetaCutBarrel : kThetaCutForward;
        // the slot's (cell, candidate) pairs are enumerated flat, 32 at a
        // time: pair f is cell f / m of a chunk and candidate f % m, so only
        // the last step of a chunk leaves lanes idle.  f < 32 * 128, so the
        // quotient from the single-precision reciprocal is exact (the error,
        // below 2^-11, is far under the 0.5 / m that (f + 0.5) / m keeps
        // from an integer).
        if (myM > 0) myInvM = 1.f / float(myM);
      }
    }
    uint32_t live = __ballot_sync(0xffffffffu, myBase < myEnd && myM > 0);
    while (live) {
      const int l = __ffs(live) - 1;
      live &= live - 1;
      const uint32_t base = __shfl_sync(0xffffffffu, myBase, l);
      const uint32_t end = __shfl_sync(0xffffffffu, myEnd, l);
      const uint32_t ob = __shfl_sync(0xffffffffu, myOb, l);
      const uint32_t m = __shfl_sync(0xffffffffu, myM, l);
      const uint32_t h = __shfl_sync(0xffffffffu, myH, l);
      const float ri = __shfl_sync(0xffffffffu, myRi, l), zi = __shfl_sync(0xffffffffu, myZi, l);
      const float thetaCut = __shfl_sync(0xffffffffu, myTheta, l);
      const float invM = __shfl_sync(0xffffffffu, myInvM, l);
      for (uint32_t c0 = base; c0 < end; c0 += 32) {
        const uint32_t nc = min(32u, end - c0);
        float sro = 0.f, szo = 0.f;
        uint32_t soh = 0;
        if (lane < nc) {
          soh = ws.cellOuter[cb + c0 + lane];
          sro = hh.rg[soh];
          szo = hh.zg[soh];
        }
        const uint32_t P = nc * m;
        for (uint32_t f0 = 0; f0 < P; f0 += 32) {
          const uint32_t f = f0 + lane;
          const bool valid = f < P;
          const uint32_t t = valid ? uint32_t((float(f) + 0.5f) * invM) : 0u;
          const uint32_t k = f - t * m;
          const float ro = __shfl_sync(0xffffffffu, sro, t), zo = __shfl_sync(0xffffffffu, szo, t);
          float4 r1 = make_float4(0.f, 0.f, 0.f, 0.f);
          if (valid) r1 = ohRec[ob + k];
          const bool pass = valid && alignedRZMaybe(fabsf(r1.w), r1.z, ri, zi, ro, zo, thetaCut);
          const uint32_t mask = __ballot_sync(0xffffffffu, pass);
          if (mask == 0) continue;
          const uint32_t oh = __shfl_sync(0xffffffffu, soh, t);
          if (pass) queue[(qTail + __popc(mask & lanemaskLt())) & (kConnectQueue - 1)] = make_uint4(ob + k, c0 + t, h, oh);
          qTail += __popc(mask);
          if (qTail - qHead >= 32) drain(32);
        }
      }
    }
  }
  while (qTail != qHead) drain(min(32u, qTail - qHead));
  near = __reduce_add_sync(0xffffffffu, near);
  if (lane == 0 && near) atomicAdd(&c->nearCA, near);
}

__global__ void kEdgeScatter(Workspace ws, const uint32_t* edgeOc, const uint32_t* edgeIdx) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  const uint32_t edgeCap = min(ws.cap.edges, ws.cap.scratch);
  uint32_t n = min(c->nEdges, edgeCap);
  const uint32_t* off = ws.nbrOff + size_t(e) * (ws.cap.cells + 1);
  uint32_t* cur = ws.nbrCount + size_t(e) * (ws.cap.cells + 1);
  uint32_t* touch = ws.hitTouch + size_t(e) * ws.cap.hits;
  uint32_t* fishList = ws.ca.earlyFishbone ? ws.fishHits + size_t(e) * ws.cap.hits : nullptr;
  const size_t cb = size_t(e) * ws.cap.cells;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    uint32_t oc = edgeOc[size_t(e) * ws.cap.scratch + k];
    const uint32_t idx = edgeIdx[size_t(e) * ws.cap.scratch + k];
    uint32_t p = atomicAdd(&cur[oc], 1u);
    if (off[oc] + p < edgeCap) ws.nbr[size_t(e) * ws.cap.edges + off[oc] + p] = idx;
    if (p == 1) noteSegment(ws, e, 1, oc);
    if (fishList) {
      // the link's cells end on these two hits; a hit on which two link ends
      // land may have two used cells and goes to the early fishbone's list
      const uint32_t h0 = ws.cellOuter[cb + oc], h1 = ws.cellOuter[cb + idx];
      if (atomicAdd(&touch[h0], 1u) == 1u) fishList[atomicAdd(&c->nFishHits, 1u)] = h0;
      if (atomicAdd(&touch[h1], 1u) == 1u) fishList[atomicAdd(&c->nFishHits, 1u)] = h1;
    }
  }
}

// cells with at least one CA link must fit the 65535-list pool of the reference.
// The same pass clears the n-tuplet search's per-cell counts and lists the
// cells with links: a tuple has at least two cells, so only they can start
// one.  The list goes to startHitOff, which is free until the scan of the
// start-hit counts writes it.
__global__ void kNbrPool(Workspace ws) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  uint32_t n = c->nCells;
  const uint32_t* off = ws.nbrOff + size_t(e) * (ws.cap.cells + 1);
  uint32_t* tc = ws.startTupleCount + size_t(e) * (ws.cap.cells + 1);
  uint32_t* hc = ws.startHitCount + size_t(e) * (ws.cap.cells + 1);
  uint32_t* linked = ws.startHitOff + size_t(e) * (ws.cap.cells + 1);
  uint32_t local = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool has = off[i + 1] > off[i];
    local += has ? 1u : 0u;
    tc[i] = 0;
    hc[i] = 0;
    const uint32_t active = __activemask();
    const uint32_t bal = __ballot_sync(active, has);
    const uint32_t leader = __ffs(active) - 1;
    uint32_t at = 0;
    if (laneId() == leader && bal) at = atomicAdd(&c->nLinked, uint32_t(__popc(bal)));
    at = __shfl_sync(active, at, leader);
    if (has) linked[at + __popc(bal & lanemaskLt())] = i;
  }
  local = __reduce_add_sync(0xffffffffu, local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(&c->nNbrLists, local);
}

// ------------------------------------------------------------------ fishbone

// gpuFishbone.h:21-90 (early fishbone), one warp per hit with >= 2 cells
// ending on it.  The serial double loop compares only the hit's used cells
// (with checkTrack, used and on a tuple): about one cell in ten.  So the
// hit's cells (first 128) are filtered first, the used ones put in ascending
// order and staged in shared memory from the isOuterHitOfCell records, and
// lane ic compares used cell ic with every later one, as the serial loop
// does.  Kills only write doubletId = -1 and never change the `used` flags
// the loop reads, so the lanes are independent.
constexpr int kFishWarps = 8;
// checkTrack: the late fishbone (gpuFishbone.h:21-90 with checkTrack), which
// also skips cells that no tuple goes through
__global__ void __launch_bounds__(kFishWarps * 32) kFishbone(Workspace ws, bool checkTrack) {
  __shared__ float sxA[kFishWarps][PF_MAX_CELLS_PER_HIT], syA[kFishWarps][PF_MAX_CELLS_PER_HIT],
      szA[kFishWarps][PF_MAX_CELLS_PER_HIT];
  __shared__ uint16_t sdA[kFishWarps][PF_MAX_CELLS_PER_HIT];
  __shared__ uint8_t skA[kFishWarps][PF_MAX_CELLS_PER_HIT];
  __shared__ uint32_t rawA[kFishWarps][PF_MAX_CELLS_PER_HIT], scA[kFishWarps][PF_MAX_CELLS_PER_HIT];
  static_assert(PF_MAX_CELLS_PER_HIT <= 256, "list positions are staged as bytes");
  const uint32_t e = blockIdx.y;
  const EventCounters* c = ws.ev + e;
  const uint32_t nHits = c->nHits;
  if (nHits < 2) return;
  const HitsView hh = hitsOf(ws, e);
  const size_t cb = size_t(e) * ws.cap.cells;
  const uint32_t* ohOff = ws.ohOff + size_t(e) * (ws.cap.hits + 1);
  const uint32_t* ohCells = ws.ohCells + cb;
  const float4* ohRec = ws.ohRec + cb;
  const uint16_t* ohDet = ws.ohDet + cb;
  const uint32_t* trkOff = ws.trkOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t w = threadIdx.x >> 5, lane = laneId();
  float* sx = sxA[w];
  float* sy = syA[w];
  float* sz = szA[w];
  uint16_t* sd = sdA[w];
  uint8_t* sk = skA[w];
  uint32_t* raw = rawA[w];
  uint32_t* sc = scA[w];
  // One hit, done by the `width` lanes starting at lane g0 (the loop below
  // gives it the whole warp, for hits with more than four used cells): the
  // used cells, with their list positions, compacted at raw/sk[o..] in list
  // order, then staged in ascending cell order at sx..sc[o..] and compared.
  auto fishHit = [&](uint32_t h, uint32_t b, uint32_t s, uint32_t o, uint32_t g0, uint32_t width) {
    const uint32_t gl = lane - g0;
    const uint32_t gmask = width == 32 ? 0xffffffffu : ((1u << width) - 1u) << g0;
    uint32_t nu = 0;  // used cells (uniform over the group)
    for (uint32_t k0 = 0; k0 < s; k0 += width) {
      const uint32_t k = k0 + gl;
      uint32_t cell = 0;
      bool used = false;
      if (k < s) {
        cell = ohCells[b + k];
        used = ws.cellUsed[cb + cell] && !(checkTrack && trkOff[cell + 1] == trkOff[cell]);
      }
      const uint32_t bal = __ballot_sync(gmask, used) >> g0;
      if (used) {
        const uint32_t pos = nu + __popc(bal & ((1u << gl) - 1u));
        raw[o + pos] = cell;
        sk[o + pos] = uint8_t(k);
      }
      nu += __popc(bal);
    }
    if (nu < 2) nu = 0;  // nothing to compare
    __syncwarp();
    const float xo = nu ? hh.xg[h] : 0.f, yo = nu ? hh.yg[h] : 0.f, zo = nu ? hh.zg[h] : 0.f;
    for (uint32_t u = gl; u < nu; u += width) {
      const uint32_t cell = raw[o + u];
      uint32_t r = 0;
      for (uint32_t m = 0; m < nu; ++m) r += raw[o + m] < cell ? 1u : 0u;
      const uint32_t k = sk[o + u];
      const float4 rec = ohRec[b + k];
      sx[o + r] = rec.x - xo;
      sy[o + r] = rec.y - yo;
      sz[o + r] = rec.z - zo;
      sd[o + r] = ohDet[b + k];
      sc[o + r] = cell;
    }
    __syncwarp();
    for (uint32_t ic = gl; ic < nu; ic += width) {
      const float xi = sx[o + ic], yi = sy[o + ic], zi = sz[o + ic];
      const uint16_t di = sd[o + ic];
      const float ni = xi * xi + yi * yi + zi * zi;
      for (uint32_t jc = ic + 1; jc < nu; ++jc) {
        const float xj = sx[o + jc], yj = sy[o + jc], zj = sz[o + jc];
        const float nj = xj * xj + yj * yj + zj * zj;
        const float cos12 = xi * xj + yi * yj + zi * zj;
        if (di != sd[o + jc] && cos12 * cos12 >= 0.99999f * ni * nj) {
          if (ni > nj) {
            ws.cellDoubletId[cb + sc[o + ic]] = -1;
            break;
          } else {
            ws.cellDoubletId[cb + sc[o + jc]] = -1;
          }
        }
      }
    }
    __syncwarp();
  };
  // The hits: the list kEdgeScatter made (early fishbone, all links kept),
  // else all of them.  A lane per hit scans the hit's cells for the used
  // ones (eight loads in flight); a hit with two to four of them (nearly
  // all) is compared by its lane alone, the cells in registers put in
  // ascending order by a sorting network; a hit with more is done by the
  // whole warp (fishHit).  The lanes' memory accesses overlap instead of
  // following one another hit after hit.
  const uint32_t* list =
      checkTrack || c->nEdges > min(ws.cap.edges, ws.cap.scratch) ? nullptr : ws.fishHits + size_t(e) * ws.cap.hits;
  const uint32_t n = list ? c->nFishHits : nHits;
  const uint32_t stride = gridDim.x * kFishWarps * 32;
  for (uint32_t i0 = (blockIdx.x * kFishWarps + w) * 32; i0 < n; i0 += stride) {
    const uint32_t i = i0 + lane;
    uint32_t h = 0, b = 0, s = 0;
    if (i < n) {
      h = list ? list[i] : i;
      b = ohOff[h];
      s = min(ohOff[h + 1] - b, uint32_t(PF_MAX_CELLS_PER_HIT));
    }
    // the used cells: their number and the list positions of the first four
    uint32_t nu = 0, k0 = 0, k1 = 0, k2 = 0, k3 = 0;
    for (uint32_t kb = 0; kb < s; kb += 8) {
      uint32_t cl[8];
#pragma unroll
      for (uint32_t j = 0; j < 8; ++j) cl[j] = kb + j < s ? ohCells[b + kb + j] : 0u;
#pragma unroll
      for (uint32_t j = 0; j < 8; ++j) {
        const uint32_t k = kb + j;
        const bool used =
            k < s && ws.cellUsed[cb + cl[j]] && !(checkTrack && trkOff[cl[j] + 1] == trkOff[cl[j]]);
        if (used) {
          k0 = nu == 0 ? k : k0;
          k1 = nu == 1 ? k : k1;
          k2 = nu == 2 ? k : k2;
          k3 = nu == 3 ? k : k3;
          ++nu;
        }
      }
    }
    if (nu >= 2 && nu <= 4) {
      const float xo = hh.xg[h], yo = hh.yg[h], zo = hh.zg[h];
      uint32_t cc[4], dd[4];
      float xx[4], yy[4], zz[4];
#pragma unroll
      for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t k = j == 0 ? k0 : j == 1 ? k1 : j == 2 ? k2 : k3;
        cc[j] = 0xffffffffu;  // unused entries sort last
        dd[j] = 0;
        xx[j] = yy[j] = zz[j] = 0.f;
        if (j < nu) {
          const float4 rec = ohRec[b + k];
          cc[j] = ohCells[b + k];
          xx[j] = rec.x - xo;
          yy[j] = rec.y - yo;
          zz[j] = rec.z - zo;
          dd[j] = ohDet[b + k];
        }
      }
      // ascending cell order (the serial loop's order): a sorting network of
      // five compare-exchanges
      auto cx = [&](int a, int bb) {
        if (cc[a] > cc[bb]) {
          uint32_t t = cc[a];
          cc[a] = cc[bb];
          cc[bb] = t;
          t = dd[a];
          dd[a] = dd[bb];
          dd[bb] = t;
          float f = xx[a];
          xx[a] = xx[bb];
          xx[bb] = f;
          f = yy[a];
          yy[a] = yy[bb];
          yy[bb] = f;
          f = zz[a];
          zz[a] = zz[bb];
          zz[bb] = f;
        }
      };
      cx(0, 1);
      cx(2, 3);
      cx(0, 2);
      cx(1, 3);
      cx(1, 2);
#pragma unroll
      for (uint32_t ic = 0; ic < 3; ++ic) {
        if (ic + 1 < nu) {
          const float xi = xx[ic], yi = yy[ic], zi = zz[ic];
          const float ni = xi * xi + yi * yi + zi * zi;
          bool stop = false;
#pragma unroll
          for (uint32_t jc = ic + 1; jc < 4; ++jc) {
            if (!stop && jc < nu) {
              const float xj = xx[jc], yj = yy[jc], zj = zz[jc];
              const float nj = xj * xj + yj * yj + zj * zj;
              const float cos12 = xi * xj + yi * yj + zi * zj;
              if (dd[ic] != dd[jc] && cos12 * cos12 >= 0.99999f * ni * nj) {
                if (ni > nj) {
                  ws.cellDoubletId[cb + cc[ic]] = -1;
                  stop = true;
                } else {
                  ws.cellDoubletId[cb + cc[jc]] = -1;
                }
              }
            }
          }
        }
      }
    }
    // hits with more than four used cells: the whole warp, one at a time
    uint32_t rest = __ballot_sync(0xffffffffu, nu > 4);
    while (rest) {
      const int l = __ffs(rest) - 1;
      rest &= rest - 1;
      fishHit(__shfl_sync(0xffffffffu, h, l), __shfl_sync(0xffffffffu, b, l), __shfl_sync(0xffffffffu, s, l), 0u,
              0u, 32u);
    }
  }
}

// ------------------------------------------------------------------ n-tuplets

// DFS of GPUCACell::find_ntuplets from one starting cell, in serial order.
// Emit(depth, cells[], outerHitOfLast) is called for every saved tuple.
template <typename Emit>
__device__ __forceinline__ bool dfsNtuplets(uint32_t start, const int32_t* doubletId, const uint32_t* nbrOff,
                                            const uint32_t* nbr, uint32_t minHits, Emit&& emit) {
  uint32_t stack[5], pos[5];
  int depth = 0;
  stack[0] = start;
  pos[0] = 0;
  bool anyAlive0 = false;
  bool last[5];
  last[0] = true;
  (void)anyAlive0;
  while (depth >= 0) {
    uint32_t cell = stack[depth];
    uint32_t b = nbrOff[cell];
    uint32_t cnt = min(nbrOff[cell + 1] - b, uint32_t(PF_MAX_CELL_NEIGHBORS));
    bool descended = false;
    while (pos[depth] < cnt) {
      uint32_t other = nbr[b + pos[depth]];
      pos[depth]++;
      if (doubletId[other] < 0) continue;
      last[depth] = false;
      if (depth + 1 >= 4) return false;  // a path longer than five hits
      ++depth;
      stack[depth] = other;
      pos[depth] = 0;
      last[depth] = true;
      descended = true;
      break;
    }
    if (descended) continue;
    if (last[depth] && uint32_t(depth + 1) >= minHits - 1) emit(depth + 1, stack);
    --depth;
  }
  return true;
}

__device__ __forceinline__ bool isStartCell(const Workspace& ws, size_t cb, uint32_t idx) {
  if (ws.cellDoubletId[cb + idx] < 0) return false;
  int pid = ws.cellPair[cb + idx];
  return ws.ca.minHits > 3 ? pid < 3 : (pid < 8 || pid > 12);
}

// The count pass stages every tuple it finds, so that the write pass is a
// flat copy instead of a second search: the tuple's cells padded with ~0
// (scratchA, 16-byte aligned), and its rank and first-hit offset among the
// tuples of its start cell (scratchB).  Both regions are free between the CA
// links and the duplicate rounds.  Records are appended in any order (one
// atomic per group of lanes that find a tuple together); the write pass puts
// each at its serial position, the start cell's scanned offsets plus its
// rank.  An event with more tuples than the staging holds is written by a
// second search, as before.
struct TupleStage {
  uint4* cells;
  uint32_t* rank;
  uint32_t* hit;
  uint32_t cap;
};
__device__ __forceinline__ TupleStage tupleStage(const Workspace& ws, uint32_t e) {
  uint32_t* a = ws.scratchA + size_t(e) * ws.cap.scratch;
  const uint32_t pad = uint32_t((16u - (reinterpret_cast<uintptr_t>(a) & 15u)) & 15u) / 4u;
  TupleStage t;
  t.cap = min(ws.cap.tuples, (ws.cap.scratch - pad) / 4u);
  t.cells = reinterpret_cast<uint4*>(a + pad);
  t.rank = ws.scratchB + size_t(e) * ws.cap.scratch;
  t.hit = t.rank + t.cap;
  return t;
}

__global__ void kNtupletCount(Workspace ws) {
  namespace cg = cooperative_groups;
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  size_t cb = size_t(e) * ws.cap.cells;
  const uint32_t* nbrOff = ws.nbrOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t* nbr = ws.nbr + size_t(e) * ws.cap.edges;
  uint32_t* tc = ws.startTupleCount + size_t(e) * (ws.cap.cells + 1);
  uint32_t* hc = ws.startHitCount + size_t(e) * (ws.cap.cells + 1);
  const TupleStage st = tupleStage(ws, e);
  // the cells with links (kNbrPool; the counts of all others are zero)
  const uint32_t* linked = ws.startHitOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t nl = c->nLinked;
  for (uint32_t li = blockIdx.x * blockDim.x + threadIdx.x; li < nl; li += gridDim.x * blockDim.x) {
    const uint32_t idx = linked[li];
    uint32_t nt = 0, nh = 0;
    if (isStartCell(ws, cb, idx)) {
      bool ok = dfsNtuplets(idx, ws.cellDoubletId + cb, nbrOff, nbr, ws.ca.minHits, [&](int ncells, const uint32_t* cells) {
        const cg::coalesced_group g = cg::coalesced_threads();
        uint32_t s0 = 0;
        if (g.thread_rank() == 0) s0 = atomicAdd(&c->nStaged, g.size());
        const uint32_t s = g.shfl(s0, 0) + g.thread_rank();
        if (s < st.cap) {
          st.cells[s] = make_uint4(cells[0], ncells > 1 ? cells[1] : ~0u, ncells > 2 ? cells[2] : ~0u,
                                   ncells > 3 ? cells[3] : ~0u);
          st.rank[s] = nt;
          st.hit[s] = nh;
        }
        ++nt;
        nh += uint32_t(ncells) + 1;
      });
      if (!ok) atomicOr(&c->flags, kFlagDeepTuple);
    }
    tc[idx] = nt;
    hc[idx] = nh;
  }
}

__global__ void kNtupletWrite(Workspace ws) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  uint32_t n = c->nCells;
  size_t cb = size_t(e) * ws.cap.cells;
  const uint32_t* nbrOff = ws.nbrOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t* nbr = ws.nbr + size_t(e) * ws.cap.edges;
  const uint32_t* to = ws.startTupleOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t* ho = ws.startHitOff + size_t(e) * (ws.cap.cells + 1);
  uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  uint32_t* th = ws.tupleHits + size_t(e) * ws.cap.tupleHits();
  uint32_t* tcell = ws.tupleCells + size_t(e) * ws.cap.tupleCells();
  uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  const TupleStage st = tupleStage(ws, e);
  const uint32_t staged = c->nStaged;
  if (staged <= st.cap) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < staged; s += gridDim.x * blockDim.x) {
      const uint4 r = st.cells[s];
      const uint32_t m = to[r.x] + st.rank[s];
      if (m >= ws.cap.tuples) continue;
      const uint32_t off = ho[r.x] + st.hit[s];
      toff[m] = off;
      // the cells (at least two) and their hits; the per-event stride of
      // tcell is 4 * cap.tuples words on a 256-byte aligned base
      th[off] = ws.cellInner[cb + r.x];
      th[off + 1] = ws.cellInner[cb + r.y];
      uint32_t last = r.y, nc = 2;
      if (r.z != ~0u) {
        th[off + 2] = ws.cellInner[cb + r.z];
        last = r.z;
        nc = 3;
        if (r.w != ~0u) {
          th[off + 3] = ws.cellInner[cb + r.w];
          last = r.w;
          nc = 4;
        }
      }
      th[off + nc] = ws.cellOuter[cb + last];
      reinterpret_cast<uint4*>(tcell)[m] = r;
      q[m] = kBad;
    }
    return;
  }
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
    if (!isStartCell(ws, cb, idx)) continue;
    uint32_t m = to[idx], off = ho[idx];
    if (m >= ws.cap.tuples) continue;
    dfsNtuplets(idx, ws.cellDoubletId + cb, nbrOff, nbr, ws.ca.minHits, [&](int ncells, const uint32_t* cells) {
      if (m < ws.cap.tuples) {
        toff[m] = off;
        for (int k = 0; k < ncells; ++k) {
          th[off + k] = ws.cellInner[cb + cells[k]];
          tcell[4 * m + k] = cells[k];
        }
        th[off + ncells] = ws.cellOuter[cb + cells[ncells - 1]];
        for (int k = ncells; k < 4; ++k) tcell[4 * m + k] = 0xffffffffu;
        q[m] = kBad;
      }
      ++m;
      off += uint32_t(ncells) + 1;
    });
  }
}

// bulkFinalizeFill and the stored-tuple count
__global__ void kTupleFinalize(Workspace ws) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  uint32_t m = c->apcM, nh = c->apcN;
  uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  const uint32_t bins = ws.cap.tuples;
  if (m >= bins) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      toff[bins] = toff[bins - 1];
      c->flags |= kFlagTupleOverflow;
    }
  } else {
    for (uint32_t i = m + blockIdx.x * blockDim.x + threadIdx.x; i <= bins; i += gridDim.x * blockDim.x)
      toff[i] = nh;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) c->nTuples = min(m, bins);
}

__device__ __forceinline__ uint32_t tupleSize(const uint32_t* toff, uint32_t t) { return toff[t + 1] - toff[t]; }

// cells of stored tuple t, from its cell slots: unlike tupleSize this also
// holds for the last bin of a full container, whose size the finalize sets to
// zero after the tuple was written and added to its cells' track lists
__device__ __forceinline__ uint32_t tupleCellCount(const uint32_t* tcell, uint32_t t) {
  uint32_t n = 0;
  while (n < 4 && tcell[4 * t + n] != 0xffffffffu) ++n;
  return n;
}

// the four cell slots of tuple t in one load (the slots of a tuple are 16
// bytes, 16-byte aligned); the cells are the slots before the first 0xffffffff
__device__ __forceinline__ uint4 tupleCellSlots(const uint32_t* tcell, uint32_t t) {
  return *reinterpret_cast<const uint4*>(tcell + 4 * size_t(t));
}

// cell -> track lists: count, (scan), fill, order
__global__ void kTrackCount(Workspace ws) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  uint32_t nt = c->nTuples;
  const uint32_t* tcell = ws.tupleCells + size_t(e) * ws.cap.tupleCells();
  uint32_t* cnt = ws.trkCount + size_t(e) * (ws.cap.cells + 1);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    const uint32_t ncell = tupleCellCount(tcell, t);
    for (uint32_t k = 0; k < ncell; ++k) atomicAdd(&cnt[tcell[4 * t + k]], 1u);
  }
}

__global__ void kTrackFill(Workspace ws) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  uint32_t nt = c->nTuples;
  const uint32_t* tcell = ws.tupleCells + size_t(e) * ws.cap.tupleCells();
  const uint32_t* off = ws.trkOff + size_t(e) * (ws.cap.cells + 1);
  uint32_t* cur = ws.trkCount + size_t(e) * (ws.cap.cells + 1);
  uint32_t* trk = ws.trk + size_t(e) * ws.cap.tupleCells();
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    const uint32_t ncell = tupleCellCount(tcell, t);
    for (uint32_t k = 0; k < ncell; ++k) {
      uint32_t cc = tcell[4 * t + k];
      uint32_t p = atomicAdd(&cur[cc], 1u);
      trk[off[cc] + p] = t;
      if (p == 1) noteSegment(ws, e, 2, cc);
    }
  }
}

__device__ __forceinline__ uint32_t trkListSize(const uint32_t* off, uint32_t cell) {
  return min(off[cell + 1] - off[cell], uint32_t(PF_MAX_CELL_TRACKS));
}

// pool usage of the cell->track lists; candidate flags for the duplicate removers
__global__ void kTrackPool(Workspace ws, uint32_t* candFlag) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  uint32_t n = c->nCells;
  const uint32_t* off = ws.trkOff + size_t(e) * (ws.cap.cells + 1);
  uint32_t* flag = candFlag + size_t(e) * (ws.cap.cells + 1);
  uint32_t* cand = ws.candidates + size_t(e) * ws.cap.cells;
  uint32_t local = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t s = off[i + 1] - off[i];
    local += s > 0 ? 1u : 0u;
    const bool isCand = min(s, uint32_t(PF_MAX_CELL_TRACKS)) >= 2;
    flag[i] = isCand ? 1u : 0u;
    // the candidate list in no particular order: the duplicate removers that
    // read it do not depend on it
    const uint32_t am = __activemask();
    const uint32_t m = __ballot_sync(am, isCand);
    const uint32_t leader = uint32_t(__ffs(am) - 1);
    uint32_t at = 0;
    if (laneId() == leader && m) at = atomicAdd(&c->nCandidates, uint32_t(__popc(m)));
    at = __shfl_sync(am, at, leader);
    if (isCand) cand[at + __popc(m & lanemaskLt())] = i;
  }
  local = __reduce_add_sync(0xffffffffu, local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(&c->nTrkLists, local);
}

// kernel_earlyDuplicateRemover: per cell with >= 2 tracks
__global__ void kEarlyDup(Workspace ws) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  uint32_t nc = c->nCandidates;
  const uint32_t* cand = ws.candidates + size_t(e) * ws.cap.cells;
  const uint32_t* off = ws.trkOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t* trk = ws.trk + size_t(e) * ws.cap.tupleCells();
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
    uint32_t cell = cand[k];
    uint32_t b = off[cell], s = trkListSize(off, cell);
    uint32_t maxNh = 0;
    for (uint32_t j = 0; j < s; ++j) maxNh = max(maxNh, tupleSize(toff, trk[b + j]));
    for (uint32_t j = 0; j < s; ++j)
      if (tupleSize(toff, trk[b + j]) != maxNh) q[trk[b + j]] = kDup;
  }
}

// tuple hits -> detector indices (kernel_fillHitDetIndices)
__global__ void kTupleDet(Workspace ws) {
  uint32_t e = blockIdx.y;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  uint32_t n = toff[ws.cap.tuples];
  const uint32_t* th = ws.tupleHits + size_t(e) * ws.cap.tupleHits();
  uint16_t* td = ws.tupleDet + size_t(e) * ws.cap.tupleHits();
  const uint16_t* det = ws.detInd + size_t(e) * ws.cap.hits;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) td[k] = det[th[k]];
}

// TupleMultiplicity: counts per hit multiplicity, then fill (order irrelevant to the fits)
// TupleMultiplicity (countMultiplicity/fillMultiplicity, Impl.h:304-338):
// one block per event counts the non-duplicate tuples of 3, 4 and 5 hits,
// places the bins, and fills them in ascending tuple order (the serial fill
// order) with one scan of the three counters packed into 64 bits, so that
// the content stays deterministic when a bin overflows.
__global__ void __launch_bounds__(1024) kMultiplicity(Workspace ws) {
  __shared__ uint32_t cnt[8], start[8];
  __shared__ uint64_t scanSh[33];
  const uint32_t e = blockIdx.x;
  EventCounters* c = ws.ev + e;
  const uint32_t nt = c->nTuples;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  const uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  uint32_t* tm = ws.tmOff + size_t(e) * 16;
  uint32_t* bins = ws.tmBins + size_t(e) * ws.cap.tuples;
  auto binOf = [&](uint32_t t) -> uint32_t {  // 0: not binned
    const uint32_t nh = tupleSize(toff, t);
    return (nh < 3 || nh > 5 || q[t] == kDup) ? 0u : nh;
  };
  // Each warp takes a contiguous range of tuples, 32 consecutive ones per
  // step (coalesced loads, four steps in flight).  A lane keeps the bin of
  // each of its tuples as a 2-bit code (up to 128 steps), so the second walk,
  // which places the tuples, needs no loads.
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t R = (nt + nw * 32 - 1) / (nw * 32) * 32;
  const uint32_t w0 = min(nt, warp * R), w1 = min(nt, w0 + R);
  const uint32_t steps = (w1 - w0 + 31) / 32;
  constexpr uint32_t kKeptSteps = 128;
  const bool kept = steps <= kKeptSteps;
  uint64_t code[kKeptSteps / 32] = {0, 0, 0, 0};
  uint32_t n3 = 0, n4 = 0, n5 = 0;
#pragma unroll
  for (uint32_t g = 0; g < kKeptSteps / 32 + 1; ++g) {
    // steps [32 g, 32 g + 32); the last group takes every step beyond 128
    const uint32_t kEnd = g < kKeptSteps / 32 ? min(steps, 32 * g + 32) : steps;
    for (uint32_t k = 32 * g; k < kEnd; k += 4) {
      uint32_t bb[4];
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t t = w0 + (k + u) * 32 + lane;
        bb[u] = (k + u < kEnd && t < w1) ? binOf(t) : 0u;
      }
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        n3 += bb[u] == 3 ? 1u : 0u;
        n4 += bb[u] == 4 ? 1u : 0u;
        n5 += bb[u] == 5 ? 1u : 0u;
        if (g < kKeptSteps / 32 && bb[u]) code[g < kKeptSteps / 32 ? g : 0] |= uint64_t(bb[u] - 2) << (2 * (k + u - 32 * g));
      }
    }
  }
  n3 = __reduce_add_sync(0xffffffffu, n3);
  n4 = __reduce_add_sync(0xffffffffu, n4);
  n5 = __reduce_add_sync(0xffffffffu, n5);
  uint64_t tot;
  const uint64_t mine = uint64_t(n3) | (uint64_t(n4) << 20) | (uint64_t(n5) << 40);
  const uint64_t warpPre = __shfl_sync(0xffffffffu, blockExclusiveScan64(lane == 0 ? mine : 0ull, scanSh, &tot), 0);
  if (threadIdx.x == 0) {
    for (int b = 0; b < 8; ++b) cnt[b] = (b >= 3 && b <= 5) ? uint32_t((tot >> (20 * (b - 3))) & 0xfffffu) : 0u;
    uint32_t acc = 0;
    for (int b = 0; b < 8; ++b) {
      start[b] = acc;
      tm[8 + b] = acc;  // start of bin b
      tm[b] = cnt[b];
      if (cnt[b] > ws.cap.multiplicity) c->flags |= kFlagFitBinOverflow;
      acc += cnt[b];
    }
    if (acc > ws.cap.multiplicity) c->flags |= kFlagTmOverflow;
    // the neighbour and track list pools of the reference (CellNeighborsVector,
    // CellTracksVector: cap.lists lists including the reserved empty one);
    // beyond them its lists depend on the order the cells are visited
    if (c->nNbrLists > ws.cap.lists) c->flags |= kFlagNbrPoolOverflow;
    if (c->nTrkLists > ws.cap.lists) c->flags |= kFlagTrkPoolOverflow;
  }
  __syncthreads();
  // the serial fill order: ascending tuple index (warps in range order, then
  // steps, then lanes)
  uint32_t run[3] = {uint32_t(warpPre & 0xfffffu), uint32_t((warpPre >> 20) & 0xfffffu),
                     uint32_t((warpPre >> 40) & 0xfffffu)};
#pragma unroll
  for (uint32_t g = 0; g < kKeptSteps / 32 + 1; ++g) {
    const uint32_t kEnd = g < kKeptSteps / 32 ? min(steps, 32 * g + 32) : steps;
    for (uint32_t k = 32 * g; k < kEnd; ++k) {
      const uint32_t t = w0 + k * 32 + lane;
      uint32_t b = 0;
      if (kept && g < kKeptSteps / 32)
        b = t < w1 ? uint32_t((code[g < kKeptSteps / 32 ? g : 0] >> (2 * (k - 32 * g))) & 3u) : 0u;
      else
        b = t < w1 ? binOf(t) : 0u;
      if (kept && b) b += 2;  // codes 1, 2, 3 are the bins 3, 4, 5
#pragma unroll
      for (uint32_t bi = 0; bi < 3; ++bi) {
        const bool in = b == bi + 3;
        const uint32_t m = __ballot_sync(0xffffffffu, in);
        if (in) {
          const uint32_t pos = start[bi + 3] + run[bi] + __popc(m & lanemaskLt());
          if (pos < ws.cap.tuples) bins[pos] = t;
        }
        run[bi] += __popc(m);
      }
    }
  }
}

// ------------------------------------------------------------------ after the fit

// kernel_classifyTracks with makeQualityCuts
__global__ void kClassify(Workspace ws) {
  uint32_t e = blockIdx.y;
  uint32_t nt = ws.ev[e].nTuples;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  const float* st = ws.state + size_t(e) * ws.cap.tuples * 5;
  const float* pt = ws.pt + size_t(e) * ws.cap.tuples;
  const float* chi2 = ws.chi2 + size_t(e) * ws.cap.tuples;
  const float c0 = float(0.68177776), c1 = float(0.74609577), c2 = float(-0.08035491), c3 = float(0.00315399);
  uint32_t near = 0;  // per thread: cut decisions on their boundary
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    uint32_t nh = tupleSize(toff, t);
    if (nh == 0) continue;  // beyond the serial loop's guard (only the overflow tail)
    if (q[t] == kDup) continue;
    if (nh < 3) continue;
    bool isNaN = false;
    for (int i = 0; i < 5; ++i) isNaN |= isnan(st[size_t(t) * 5 + i]);
    if (isNaN) continue;
    float p = fminf(pt[t], 10.f);
    float chi2Cut = 30.f * (c0 + p * (c1 + p * (c2 + p * c3)));
    near += cutNear(3.f * chi2[t], chi2Cut);
    if (3.f * chi2[t] >= chi2Cut) continue;
    float maxTip = nh > 3 ? 0.5f : 0.3f, minPt = nh > 3 ? 0.3f : 0.5f;
    near += cutNear(fabsf(st[size_t(t) * 5 + 1]), maxTip) + cutNear(pt[t], minPt) +
            cutNear(fabsf(st[size_t(t) * 5 + 4]), 12.f);
    bool isOk = (fabsf(st[size_t(t) * 5 + 1]) < maxTip) && (pt[t] > minPt) && (fabsf(st[size_t(t) * 5 + 4]) < 12.f);
    if (isOk) q[t] = kLoose;
  }
  near = __reduce_add_sync(0xffffffffu, near);
  if ((threadIdx.x & 31) == 0 && near) atomicAdd(&ws.ev[e].nearQuality, near);
}

__device__ __forceinline__ bool inTrkList(const uint32_t* off, const uint32_t* trk, uint32_t cell, uint32_t t) {
  uint32_t b = off[cell], s = off[cell + 1] - b;
  if (s <= uint32_t(PF_MAX_CELL_TRACKS)) return true;  // t is known to be in the full list
  return t <= trk[b + PF_MAX_CELL_TRACKS - 1];
}

// kernel_fastDuplicateRemover in serial semantics.  Candidate cells (>= 2
// tracks) are processed in rounds: a cell is processed once every earlier
// candidate sharing one of its tracks has been processed, so every cell sees
// the track qualities that the serial loop over cells would see.
__global__ void kFastDupInDegree(Workspace ws, uint32_t* indeg, const uint32_t* candFlag) {
  uint32_t e = blockIdx.y;
  uint32_t nc = ws.ev[e].nCandidates;
  const uint32_t* cand = ws.candidates + size_t(e) * ws.cap.cells;
  const uint32_t* off = ws.trkOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t* trk = ws.trk + size_t(e) * ws.cap.tupleCells();
  const uint32_t* tcell = ws.tupleCells + size_t(e) * ws.cap.tupleCells();
  const uint32_t* flag = candFlag + size_t(e) * (ws.cap.cells + 1);
  uint32_t* deg = indeg + size_t(e) * ws.cap.cells;  // by cell
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
    uint32_t cell = cand[k];
    uint32_t b = off[cell], s = trkListSize(off, cell);
    uint32_t d = 0;
    for (uint32_t j = 0; j < s; ++j) {
      const uint32_t t = trk[b + j];
      const uint4 tc = tupleCellSlots(tcell, t);
      const uint32_t cs[4] = {tc.x, tc.y, tc.z, tc.w};
#pragma unroll
      for (uint32_t q = 0; q < 4; ++q) {
        const uint32_t o = cs[q];
        if (o == 0xffffffffu) break;
        if (o < cell && flag[o] && inTrkList(off, trk, o, t)) ++d;
      }
    }
    deg[cell] = d;
  }
}

// One thread-block cluster of P CTAs per event (kFastDupCtas for small
// batches, 2 for large ones).  A worklist
// holds the candidates whose earlier track-sharing candidates are all done;
// cells of one round share no track, so the cluster's threads process them in
// parallel, and each releases its later neighbours (the in-degree reaching
// zero queues them for the next round).  The rounds are separated by cluster
// barriers; the two worklist counters live in the shared memory of rank 0.
constexpr int kFastDupThreads = 1024;
constexpr uint32_t kFastDupCtas = 8;
constexpr uint32_t kFastDupStage = 4096;  // worklist entries a CTA stages per round in shared memory
constexpr uint32_t kDupGroup = 4;         // lanes per candidate in a round
constexpr uint32_t kDupGroupsPerWarp = 32 / kDupGroup;

// Appends of one round to the next worklist: each CTA stages its entries in
// its own shared memory (local atomics), then reserves their place in the
// worklist with one atomic on rank 0's counter (distributed shared memory)
// and copies them.  Entries beyond the staging capacity are appended directly.
struct WorklistStage {
  uint32_t n;
  uint32_t base;
  uint32_t item[kFastDupStage];
};
__device__ __forceinline__ void stagePush(WorklistStage& st, uint32_t* remoteCount, uint32_t* list, uint32_t v) {
  const uint32_t p = atomicAdd(&st.n, 1u);
  if (p < kFastDupStage)
    st.item[p] = v;
  else
    list[atomicAdd(remoteCount, 1u)] = v;
}
// called by every thread of the CTA; leaves st.n at zero
__device__ __forceinline__ void stageFlush(WorklistStage& st, uint32_t* remoteCount, uint32_t* list) {
  __syncthreads();
  const uint32_t m = min(st.n, kFastDupStage);
  if (threadIdx.x == 0) st.base = m ? atomicAdd(remoteCount, m) : 0u;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) list[st.base + i] = st.item[i];
  __syncthreads();
  if (threadIdx.x == 0) st.n = 0;
}
__global__ void __launch_bounds__(kFastDupThreads)
    kFastDupRounds(Workspace ws, uint32_t* indeg, uint32_t* lists, const uint32_t* candFlag) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t r = cl.block_rank(), P = cl.num_blocks();
  __shared__ uint32_t sN[2];
  uint32_t* N = cl.map_shared_rank(sN, 0);
  const uint32_t e = blockIdx.y;
  const uint32_t nc = ws.ev[e].nCandidates;
  const uint32_t* cand = ws.candidates + size_t(e) * ws.cap.cells;
  const uint32_t* off = ws.trkOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t* trk = ws.trk + size_t(e) * ws.cap.tupleCells();
  const uint32_t* tcell = ws.tupleCells + size_t(e) * ws.cap.tupleCells();
  const uint32_t* flag = candFlag + size_t(e) * (ws.cap.cells + 1);
  uint32_t* deg = indeg + size_t(e) * ws.cap.cells;  // by cell
  uint32_t* const L0 = lists + size_t(e) * ws.cap.scratch;  // worklists: L0 and L0 + cap.cells
  auto L = [&](int w) { return L0 + (w ? ws.cap.cells : 0u); };
  uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  const float* tip = ws.state + size_t(e) * ws.cap.tuples * 5 + 1;
  const uint32_t gtid = r * blockDim.x + threadIdx.x, gstride = P * blockDim.x;
  const uint32_t gwarp = gtid >> 5, nwarps = gstride >> 5;
  const uint32_t sub = (threadIdx.x & 31) / kDupGroup, gl = threadIdx.x % kDupGroup;
  __shared__ WorklistStage st;
  if (r == 0 && threadIdx.x < 2) sN[threadIdx.x] = 0;
  if (threadIdx.x == 0) st.n = 0;
  cl.sync();
  for (uint32_t k = gtid; k < nc; k += gstride) {
    const uint32_t cell = cand[k];
    if (deg[cell] == 0) stagePush(st, &N[0], L(0), cell);
  }
  stageFlush(st, &N[0], L(0));
  cl.sync();
  int cur = 0;
  for (;;) {
    const uint32_t n = N[cur];
    // every CTA has read the count: it may be reset, and rank 0's shared
    // memory is not read after the last round
    cl.sync();
    if (n == 0) break;
    if (r == 0 && threadIdx.x == 0) N[cur] = 0;
    const uint32_t* Lc = L(cur);
    uint32_t* Ln = L(cur ^ 1);
    // kDupGroup lanes per candidate: the lanes of a group split the cell's
    // track list, so an item costs a few dependent loads whatever its size;
    // the warp's trip counts are uniform for the shuffles
    for (uint32_t i0 = gwarp * kDupGroupsPerWarp; i0 < n; i0 += nwarps * kDupGroupsPerWarp) {
      const uint32_t i = i0 + sub;
      uint32_t cell = 0, b = 0, s = 0;
      if (i < n) {
        cell = Lc[i];
        b = off[cell];
        s = trkListSize(off, cell);
      }
      const uint32_t sMax = __reduce_max_sync(0xffffffffu, s);
      // the serial loop's choice: the first loose track of minimal |tip|
      // below 10000 (key: score bits, then list position)
      unsigned long long best = ~0ull;
      for (uint32_t j0 = 0; j0 < sMax; j0 += kDupGroup) {
        const uint32_t j = j0 + gl;
        if (j < s) {
          const uint32_t t = trk[b + j];
          const float score = fabsf(tip[size_t(t) * 5]);
          if (q[t] == kLoose && score < 10000.f) {
            const unsigned long long key = (uint64_t(__float_as_uint(score)) << 32) | j;
            best = key < best ? key : best;
          }
        }
      }
#pragma unroll
      for (uint32_t o = 1; o < kDupGroup; o <<= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
        best = other < best ? other : best;
      }
      const uint32_t im = (i < n && best != ~0ull) ? trk[b + uint32_t(best & 0xffffffffu)] : kNoTuple;
      for (uint32_t j0 = 0; j0 < sMax; j0 += kDupGroup) {
        const uint32_t j = j0 + gl;
        if (j >= s) continue;
        const uint32_t t = trk[b + j];
        if (q[t] != kBad && t != im) q[t] = kDup;
        // release later candidates sharing the track
        const uint4 tc = tupleCellSlots(tcell, t);
        const uint32_t cs[4] = {tc.x, tc.y, tc.z, tc.w};
#pragma unroll
        for (uint32_t qq = 0; qq < 4; ++qq) {
          const uint32_t o = cs[qq];
          if (o == 0xffffffffu) break;
          if (o > cell && flag[o] && inTrkList(off, trk, o, t) && atomicSub(&deg[o], 1u) == 1u)
            stagePush(st, &N[cur ^ 1], Ln, o);
        }
      }
    }
    stageFlush(st, &N[cur ^ 1], Ln);
    cur ^= 1;
    // the round's quality writes and the next worklist are complete
    cl.sync();
  }
}

// hit -> loose tuples (HitToTuple), order: descending tuple index
__global__ void kHitToTupleCount(Workspace ws) {
  uint32_t e = blockIdx.y;
  uint32_t nt = ws.ev[e].nTuples;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  const uint32_t* th = ws.tupleHits + size_t(e) * ws.cap.tupleHits();
  const uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  uint32_t* cnt = ws.h2tCount + size_t(e) * (ws.cap.hits + 1);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    if (tupleSize(toff, t) == 0 || q[t] != kLoose) continue;
    for (uint32_t k = toff[t]; k < toff[t + 1]; ++k) atomicAdd(&cnt[th[k]], 1u);
  }
}
__global__ void kHitToTupleFill(Workspace ws) {
  uint32_t e = blockIdx.y;
  EventCounters* c = ws.ev + e;
  uint32_t nt = c->nTuples;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  const uint32_t* th = ws.tupleHits + size_t(e) * ws.cap.tupleHits();
  const uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  const uint32_t* off = ws.h2tOff + size_t(e) * (ws.cap.hits + 1);
  uint32_t* cur = ws.h2tCount + size_t(e) * (ws.cap.hits + 1);
  uint32_t* h2t = ws.h2t + size_t(e) * ws.cap.h2t;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    if (tupleSize(toff, t) == 0 || q[t] != kLoose) continue;
    for (uint32_t k = toff[t]; k < toff[t + 1]; ++k) {
      uint32_t h = th[k];
      uint32_t p = atomicAdd(&cur[h], 1u);
      uint32_t pos = off[h] + p;
      if (p == 1) noteSegment(ws, e, 3, h);
      if (pos < ws.cap.h2t)
        h2t[pos] = t;
      else
        atomicOr(&c->flags, kFlagH2TOverflow);
    }
  }
}

// kernel_tripletCleaner: one thread per hit with >= 2 loose tuples
__global__ void kTripletCleaner(Workspace ws) {
  uint32_t e = blockIdx.y;
  const uint32_t* off = ws.h2tOff + size_t(e) * (ws.cap.hits + 1);
  const uint32_t* h2t = ws.h2t + size_t(e) * ws.cap.h2t;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  const float* tip = ws.state + size_t(e) * ws.cap.tuples * 5 + 1;
  const uint32_t nHits = min(ws.ev[e].nHits, ws.cap.hits);  // the offsets are scanned up to nHits
  for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < nHits; h += gridDim.x * blockDim.x) {
    uint32_t b = off[h], en = min(off[h + 1], ws.cap.h2t);
    if (en <= b || en - b < 2) continue;
    uint32_t maxNh = 0;
    for (uint32_t p = b; p < en; ++p) maxNh = max(maxNh, tupleSize(toff, h2t[p]));
    for (uint32_t p = b; p < en; ++p)
      if (tupleSize(toff, h2t[p]) != maxNh) q[h2t[p]] = kDup;
    if (maxNh > 3) continue;
    float mc = 10000.f;
    uint32_t im = kNoTuple;
    for (uint32_t p = b; p < en; ++p) {
      uint32_t t = h2t[p];
      float s = fabsf(tip[size_t(t) * 5]);
      if (q[t] != kBad && s < mc) {
        mc = s;
        im = t;
      }
    }
    for (uint32_t p = b; p < en; ++p) {
      uint32_t t = h2t[p];
      if (q[t] != kBad && t != im) q[t] = kDup;
    }
  }
}

// kernel_fishboneCleaner (CAHitNtupletGeneratorKernelsImpl.h:104-116): the
// tuples through a cell the late fishbone killed are bad
__global__ void kFishboneCleaner(Workspace ws) {
  const uint32_t e = blockIdx.y;
  const uint32_t n = ws.ev[e].nCells;
  const size_t cb = size_t(e) * ws.cap.cells;
  const uint32_t* off = ws.trkOff + size_t(e) * (ws.cap.cells + 1);
  const uint32_t* trk = ws.trk + size_t(e) * ws.cap.tupleCells();
  uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (ws.cellDoubletId[cb + i] >= 0) continue;
    const uint32_t b = off[i], s = trkListSize(off, i);
    for (uint32_t j = 0; j < s; ++j) q[trk[b + j]] = kBad;
  }
}

}  // namespace

#define EVF(field) (&ws.ev[0].field), (sizeof(EventCounters) / 4)

cudaError_t runCA(const DeviceES& es, Workspace& ws, uint32_t nEvents, cudaStream_t stream) {
  (void)es;
  const uint32_t kHitCap = ws.cap.hits, kCellCap = ws.cap.cells, kJCap = ws.cap.jCap;
  const uint32_t kTupleCellCap = ws.cap.tupleCells();
  const uint32_t gx = nEvents >= 32 ? 16 : (nEvents >= 8 ? 64 : 296);  // blocks per event for flat loops
  dim3 g(gx, nEvents);
  // ---- doublets: count per inner-hit slot, scan, write in serial order
  PG_PROBED("kDoubletSetup", stream, kDoubletSetup<<<(nEvents + 63) / 64, 64, 0, stream>>>(ws, nEvents));
  PG_PROBED("kZero", stream, kZero<<<dim3(48, nEvents), 256, 0, stream>>>(ws.ohCount, kHitCap + 1, kHitCap + 1, EVF(nHits)));
  PG_PROBED("kDoubletCount", stream, kDoubletCount<<<dim3(tunedGrid(ws, kTuneDoubletCount, gx * 4), nEvents), 256, 0, stream>>>(ws));
  segScan(ws, kScanDoubletSlots, ws.jCount, ws.jOffset, kJCap + 1, EVF(ntot), kJCap, nullptr, 0, nEvents, stream);
  PG_PROBED("kDoubletWrite", stream, kDoubletWrite<<<dim3(tunedGrid(ws, kTuneDoubletWrite, gx * 4), nEvents), 256, 0, stream>>>(ws));
  PG_PROBED("kCellsTotal", stream, kCellsTotal<<<(nEvents + 63) / 64, 64, 0, stream>>>(ws, nEvents));
  // ---- isOuterHitOfCell: scan of the per-hit counts, unordered fill, order per hit
  segScan(ws, kScanOuterHits, ws.ohCount, ws.ohOff, kHitCap + 1, EVF(nHits), kHitCap, nullptr, 0, nEvents, stream, true);
  PG_PROBED("kOuterHitFill", stream, kOuterHitFill<<<dim3(tunedGrid(ws, kTuneOuterHitFill, gx), nEvents), 256, 0, stream>>>(ws));
  sortSegments<uint32_t>(ws, nEvents, stream, gx * 2, ws.ohCells, kCellCap, ws.ohOff, kHitCap + 1, EVF(nHits), 0, false, kCellCap, 0);
  PG_PROBED("kOhRec", stream, kOhRec<<<dim3(tunedGrid(ws, kTuneOhRec, gx), nEvents), 256, 0, stream>>>(ws));
  // ---- CA links: edges appended unordered, then CSR by inner cell, ordered ascending
  PG_PROBED("kZero", stream, kZero<<<dim3(gx * 2, nEvents), 256, 0, stream>>>(ws.nbrCount, kCellCap + 1, kCellCap + 1, EVF(nCells)));
  if (ws.ca.earlyFishbone)
    PG_PROBED("kZero", stream, kZero<<<dim3(gx, nEvents), 256, 0, stream>>>(ws.hitTouch, kHitCap, kHitCap, EVF(nHits)));
  PG_PROBED("kConnect", stream, kConnect<<<dim3(tunedGrid(ws, kTuneConnect, gx * 4), nEvents), kConnectWarps * 32, 0, stream>>>(ws, ws.scratchA, ws.scratchB));
  segScan(ws, kScanNeighbours, ws.nbrCount, ws.nbrOff, kCellCap + 1, EVF(nCells), kCellCap, nullptr, 0, nEvents, stream,
          true);
  PG_PROBED("kEdgeScatter", stream, kEdgeScatter<<<dim3(tunedGrid(ws, kTuneEdgeScatter, gx), nEvents), 256, 0, stream>>>(ws, ws.scratchA, ws.scratchB));
  sortSegments<uint32_t>(ws, nEvents, stream, gx * 2, ws.nbr, ws.cap.edges, ws.nbrOff, kCellCap + 1, EVF(nCells), 0, false,
                         min(ws.cap.edges, ws.cap.scratch), 1);
  PG_PROBED("kNbrPool", stream, kNbrPool<<<dim3(tunedGrid(ws, kTuneNbrPool, gx), nEvents), 256, 0, stream>>>(ws));
  // ---- early fishbone
  if (ws.ca.earlyFishbone)
    PG_PROBED("kFishbone", stream, kFishbone<<<dim3(tunedGrid(ws, kTuneFishbone, gx * 2), nEvents), 256, 0, stream>>>(ws, false));
  // ---- n-tuplets: DFS count, scans, DFS write, finalize
  PG_PROBED("kNtupletCount", stream, kNtupletCount<<<dim3(tunedGrid(ws, kTuneNtupletCount, gx * 8), nEvents), 128, 0, stream>>>(ws));
  segScan2(ws, kScanStartTuples, ws.startTupleCount, ws.startTupleOff, &ws.ev[0].apcM, kScanStartHits, ws.startHitCount,
           ws.startHitOff, &ws.ev[0].apcN, kCellCap + 1, EVF(nCells), kCellCap, sizeof(EventCounters) / 4, nEvents,
           stream);
  PG_PROBED("kNtupletWrite", stream, kNtupletWrite<<<dim3(tunedGrid(ws, kTuneNtupletWrite, gx * 8), nEvents), 128, 0, stream>>>(ws));
  PG_PROBED("kTupleFinalize", stream, kTupleFinalize<<<dim3(32, nEvents), 1024, 0, stream>>>(ws));
  // ---- cell -> track lists
  PG_PROBED("kZero", stream, kZero<<<dim3(gx * 2, nEvents), 256, 0, stream>>>(ws.trkCount, kCellCap + 1, kCellCap + 1, EVF(nCells)));
  PG_PROBED("kTrackCount", stream, kTrackCount<<<dim3(tunedGrid(ws, kTuneTrackCount, gx), nEvents), 256, 0, stream>>>(ws));
  segScan(ws, kScanCellTracks, ws.trkCount, ws.trkOff, kCellCap + 1, EVF(nCells), kCellCap, nullptr, 0, nEvents, stream,
          true);
  PG_PROBED("kTrackFill", stream, kTrackFill<<<dim3(tunedGrid(ws, kTuneTrackFill, gx), nEvents), 256, 0, stream>>>(ws));
  sortSegments<uint32_t>(ws, nEvents, stream, gx * 2, ws.trk, kTupleCellCap, ws.trkOff, kCellCap + 1, EVF(nCells), 0, false, kTupleCellCap, 2);
  uint32_t* candFlag = ws.startTupleCount;  // scratch
  PG_PROBED("kTrackPool", stream, kTrackPool<<<dim3(tunedGrid(ws, kTuneTrackPool, gx), nEvents), 256, 0, stream>>>(ws, candFlag));
  PG_PROBED("kEarlyDup", stream, kEarlyDup<<<dim3(tunedGrid(ws, kTuneEarlyDup, gx), nEvents), 256, 0, stream>>>(ws));
  PG_PROBED("kTupleDet", stream, kTupleDet<<<dim3(tunedGrid(ws, kTuneTupleDet, gx), nEvents), 256, 0, stream>>>(ws));
  // ---- tuple multiplicity for the fits
  PG_PROBED("kMultiplicity", stream, kMultiplicity<<<nEvents, 1024, 0, stream>>>(ws));
  // ---- late fishbone (CAHitNtupletGeneratorKernels.cc:133-136)
  if (ws.ca.lateFishbone)
    PG_PROBED("kFishbone", stream, kFishbone<<<dim3(tunedGrid(ws, kTuneFishbone, gx * 2), nEvents), 256, 0, stream>>>(ws, true));
  return cudaGetLastError();
}

cudaError_t runCleaners(Workspace& ws, uint32_t nEvents, cudaStream_t stream) {
  const uint32_t kHitCap = ws.cap.hits;
  const uint32_t gx = nEvents >= 32 ? 16 : (nEvents >= 8 ? 64 : 296);
  dim3 g(gx, nEvents);
  PG_PROBED("kClassify", stream, kClassify<<<dim3(tunedGrid(ws, kTuneClassify, gx), nEvents), 256, 0, stream>>>(ws));
  // kernel_fishboneCleaner with the late fishbone (CAHitNtupletGeneratorKernels.cc:159-162)
  if (ws.ca.lateFishbone) PG_PROBED("kFishboneCleaner", stream, kFishboneCleaner<<<g, 256, 0, stream>>>(ws));
  // fastDuplicateRemover (candFlag survives in startTupleCount from runCA)
  uint32_t* candFlag = ws.startTupleCount;
  uint32_t* indeg = ws.scratchA;        // [maxEvents][cap.scratch], cap.cells per event used
  uint32_t* lists = ws.scratchB;        // two worklists of cap.cells per event (cap.scratch >= 2 cap.cells)
  PG_PROBED("kFastDupInDegree", stream, kFastDupInDegree<<<dim3(tunedGrid(ws, kTuneFastDupInDegree, gx), nEvents), 256, 0, stream>>>(ws, indeg, candFlag));
  const uint32_t P = nEvents <= kClusterMaxEvents ? kFastDupCtas : 2;
  cudaError_t le = cudaSuccess;
  PG_PROBED("kFastDupRounds", stream,
            le = launchClustered(kFastDupRounds, P, nEvents, kFastDupThreads, 0, stream, ws, indeg, lists, candFlag));
  if (le != cudaSuccess) return le;
  // hit -> tuple map and triplet cleaner
  PG_PROBED("kZero", stream, kZero<<<dim3(48, nEvents), 256, 0, stream>>>(ws.h2tCount, kHitCap + 1, kHitCap + 1, EVF(nHits)));
  PG_PROBED("kHitToTupleCount", stream, kHitToTupleCount<<<dim3(tunedGrid(ws, kTuneHitToTupleCount, gx), nEvents), 256, 0, stream>>>(ws));
  segScan(ws, kScanHitTuples, ws.h2tCount, ws.h2tOff, kHitCap + 1, EVF(nHits), kHitCap, nullptr, 0, nEvents, stream, true);
  PG_PROBED("kHitToTupleFill", stream, kHitToTupleFill<<<dim3(tunedGrid(ws, kTuneHitToTupleFill, gx), nEvents), 256, 0, stream>>>(ws));
  sortSegments<uint32_t>(ws, nEvents, stream, gx * 2, ws.h2t, ws.cap.h2t, ws.h2tOff, kHitCap + 1, nullptr, 0, kHitCap, true,
                         ws.cap.h2t, 3);
  PG_PROBED("kTripletCleaner", stream, kTripletCleaner<<<dim3(tunedGrid(ws, kTuneTripletCleaner, gx * 2), nEvents), 256, 0, stream>>>(ws));
  return cudaGetLastError();
}

}  // namespace pixgpu
