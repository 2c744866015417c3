// Local reconstruction on B200: FED words -> digis (decode + gain calibration
// fused), module runs, clustering with the charge cut fused, hit-module
// starts, CPE rechits and the phi-binned hit histogram.
//
// Reference behaviour followed (src/serial paths):
//   RawToDigi_kernel         plugin-SiPixelClusterizer/SiPixelRawToClusterGPUKernel.cc:342-462
//   calibDigis               plugin-SiPixelClusterizer/gpuCalibPixel.h:22-66
//   countModules             plugin-SiPixelClusterizer/gpuClustering.h:19-37
//   findClus                 plugin-SiPixelClusterizer/gpuClustering.h:40-273
//   clusterChargeCut         plugin-SiPixelClusterizer/gpuClusterChargeCut.h:14-114
//   fillHitsModuleStart      plugin-SiPixelClusterizer/SiPixelRawToClusterGPUKernel.cc:464-506
//   getHits + CPE            plugin-SiPixelRecHits/gpuPixelRecHits.h:16-207, CondFormats/pixelCPEforGPU.h:118-340
//   setHitsLayerStart / phi histogram  plugin-SiPixelRecHits/PixelRecHits.cc:15-53, CUDACore/HistoContainer.h:18-73
//
// Ordering: every ordered product is produced in the serial backend's order
// (module runs by word index, clusters by their lowest pixel index, phi-bin
// contents by descending hit index) with scans and per-segment sorts instead
// of atomics whose order depends on scheduling.
#include <cstdio>

#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

constexpr uint16_t kInvId = PF_INV_ID;

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ uint32_t eventOfWord(const uint32_t* off, uint32_t nEvents, uint32_t g) {
  return upperBoundIdx(off, nEvents, g);
}

__device__ __forceinline__ uint32_t cablingIndex(uint32_t fed, uint32_t link, uint32_t roc) {
  return fed * PF_MAX_LINK * PF_MAX_ROC + (link - 1) * PF_MAX_ROC + roc;
}

__device__ uint8_t checkROC(uint32_t w, uint8_t fedId, uint32_t link, const PfCablingMap* cab) {
  uint8_t errorType = (w >> 21) & 0x1f;
  if (errorType < 25) return 0;
  bool found = false;
  switch (errorType) {
    case 25: {
      found = true;
      uint32_t index = cablingIndex(fedId, link, 1);
      if (index > 1 && index <= cab->size)
        if (!(link == cab->link[index] && 1 == cab->roc[index])) found = false;
      break;
    }
    case 26:
    case 27:
    case 28:
    case 29:
    case 31:
      found = true;
      break;
    case 30:
      if (((w >> 8) & 0xf) == 1) errorType = 40;
      found = true;
      break;
    default:
      found = false;
  }
  return found ? errorType : 0;
}

__device__ uint32_t getErrRawID(uint8_t fedId, uint32_t w, uint32_t errorType, const PfCablingMap* cab) {
  uint32_t rID = 0xffffffffu;
  uint32_t link = 0, roc = 1;
  switch (errorType) {
    case 25:
    case 30:
    case 31:
    case 36:
    case 40:
      link = (w >> 26) & 0x3f;
      break;
    case 29: {
      int localCH = 0;
      for (int k = 0; k < 5; ++k) localCH += (k + 1) * int((w >> k) & 1);
      int block = (w >> 8) & 0x7;
      int chan = (block % 2 == 0) ? (block / 2) * 9 + localCH : ((block - 1) / 2) * 9 + 4 + localCH;
      if (chan < 1 || chan > 36) return rID;
      link = uint32_t(chan);
      break;
    }
    case 37:
    case 38:
      roc = (w >> 21) & 0x1f;
      link = (w >> 26) & 0x3f;
      break;
    default:
      return rID;
  }
  uint32_t t = cab->rawId[cablingIndex(fedId, link, roc)];
  if (t != 9999) rID = t;
  return rID;
}

// Geometry/phase1PixelTopology.h:115-158
__device__ __forceinline__ uint16_t divu52(uint16_t n) {
  n = n >> 2;
  uint16_t q = (n >> 1) + (n >> 4);
  q = q + (q >> 4) + (q >> 5);
  q = q >> 3;
  uint16_t r = n - q * 13;
  return q + ((r + 3) >> 4);
}
__device__ __forceinline__ bool isBigPixX(uint16_t px) { return (px == 79) | (px == 80); }
__device__ __forceinline__ bool isBigPixY(uint16_t py) {
  uint16_t ly = py - 52 * divu52(py);
  return (ly == 0) | (ly == 51);
}
__device__ __forceinline__ uint16_t localX(uint16_t px) {
  int shift = 0;
  if (px > 79) shift += 1;
  if (px > 80) shift += 1;
  return px + shift;
}
__device__ __forceinline__ uint16_t localY(uint16_t py) {
  uint16_t roc = divu52(py);
  int shift = 2 * roc;
  int yInRoc = py - 52 * roc;
  if (yInRoc > 0) shift += 1;
  return py + shift;
}

__device__ float cpeCorrection(int sizeM1, int Q_f, int Q_l, uint16_t upper_edge_first_pix,
                               uint16_t lower_edge_last_pix, float lorentz_shift, float theThickness,
                               float cot_angle, float pitch, bool first_is_big, bool last_is_big) {
  if (0 == sizeM1) return 0;
  float W_eff = 0;
  bool simple = true;
  if (1 == sizeM1) {
    float W_inner = pitch * float(lower_edge_last_pix - upper_edge_first_pix);
    float W_pred = theThickness * cot_angle - lorentz_shift;
    W_eff = fabsf(W_pred) - W_inner;
    simple = (W_eff < 0.0f) | (W_eff > pitch);
  }
  if (simple) {
    float sum_of_edge = 2.0f;
    if (first_is_big) sum_of_edge += 1.0f;
    if (last_is_big) sum_of_edge += 1.0f;
    W_eff = pitch * 0.5f * sum_of_edge;
  }
  float Qdiff = Q_l - Q_f;
  float Qsum = Q_l + Q_f;
  if (Qsum == 0) Qsum = 1.0f;
  return 0.5f * (Qdiff / Qsum) * W_eff;
}

// DataFormats/approx_atan2.h:245-263, degree 7 (the reference's coefficients)
__device__ __forceinline__ int16_t unsafeAtan2s7(float y, float x) {
  float r = (fabsf(x) - fabsf(y)) / (fabsf(x) + fabsf(y));
  if (x < 0) r = -r;
  float z = r * r;
  float p = r * ((-10422.177734375f) + z * (3349.97412109375f + z * ((-1525.589599609375f) + z * 406.64190673828125f)));
  short angle = (x >= 0) ? short(8192) : short(24576);
  angle += short(p);
  return (y < 0) ? short(-angle) : angle;
}

// ------------------------------------------------------------------ kernels

// per-event initialisation of counters and module tables
__global__ void kInitEvents(Workspace ws, uint32_t nEvents) {
  uint32_t e = blockIdx.x;
  if (e >= nEvents) return;
  EventCounters* c = ws.ev + e;
  if (threadIdx.x == 0) {
    c->wordStart = ws.wordOffsets[e];
    c->nWords = ws.wordOffsets[e + 1] - ws.wordOffsets[e];
    c->nModules = 0;
    c->nHits = 0;
    c->ntot = 0;
    c->nCellsRaw = c->nCells = c->nEdges = 0;
    c->nNbrLists = c->nTrkLists = 1;
    c->apcM = c->apcN = c->nTuples = c->nTupleCells = 0;
    c->nCandidates = c->nLoose = 0;
    c->nVertices = c->nErrors = c->nVtxTracks = 0;
    c->nBig[0] = c->nBig[1] = c->nBig[2] = c->nBig[3] = 0;
    c->nBigMod = 0;
    c->nSegList[0] = c->nSegList[1] = c->nSegList[2] = c->nSegList[3] = 0;
    c->nBigHitMod = 0;
    c->nearDoublet = c->nearCA = c->nearQuality = 0;
    c->nStaged = c->nFishHits = c->nLinked = 0;
    c->flags = c->nWords > ws.cap.fedWords ? kFlagTooManyWords : 0u;
    ws.scanEpoch[e] += 1;  // tags this batch's scan state words
  }
  if (threadIdx.x < kScanCalls) ws.scanTicket[size_t(e) * kScanCalls + threadIdx.x] = 0;
  // the module-run start bitmap of kModuleBoundaries (in scratchA, free until the doublets)
  uint32_t* bm = ws.scratchA + size_t(e) * ws.cap.scratch;
  const uint32_t nbw = (min(ws.wordOffsets[e + 1] - ws.wordOffsets[e], ws.cap.fedWords) + 31) / 32;
  for (uint32_t i = threadIdx.x; i < nbw; i += blockDim.x) bm[i] = 0;
  uint32_t* cim = ws.clusInModule + size_t(e) * kModStride;
  for (uint32_t i = threadIdx.x; i < kModStride; i += blockDim.x) {
    cim[i] = 0;
    ws.moduleId[size_t(e) * kModStride + i] = 0;
    ws.moduleStart[size_t(e) * kModStride + i] = 0;
  }
}

// RawToDigi_kernel + calibDigis for every word of the batch
__global__ void kRawToDigi(DeviceES es, Workspace ws, uint32_t nEvents) {
  const uint32_t total = ws.wordOffsets[nEvents];
  const PfCablingMap* cab = es.cab;
  const PfGainHeader* gh = es.gainHdr;
  const uint32_t* words = ws.input->words;
  const uint8_t* fedIds = ws.input->fedIds;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    uint32_t e = eventOfWord(ws.wordOffsets, nEvents, g);
    uint32_t start = ws.wordOffsets[e];
    uint32_t i = g - start;
    uint8_t fedId = fedIds[g >> 1];
    uint16_t xx = 0, yy = 0, adc = 0, mid = 9999;
    uint32_t pdigi = 0, rawIdOut = 0;
    uint32_t ww = words[g];
    bool err = false;
    PfPixelError perr;
    if (ww != 0) {
      uint32_t link = (ww >> 26) & 0x3f;
      uint32_t roc = (ww >> 21) & 0x1f;
      uint32_t index = cablingIndex(fedId, link, roc);
      if (link == 0 || index >= uint32_t(PF_MAX_SIZE)) {
        // outside the cabling tables (the reference reads out of bounds here)
        atomicOr(&ws.ev[e].flags, kFlagBadInput);
        ww = 0;
      }
    }
    if (ww != 0) {
      uint32_t link = (ww >> 26) & 0x3f;
      uint32_t roc = (ww >> 21) & 0x1f;
      uint32_t index = cablingIndex(fedId, link, roc);
      uint8_t errorType = checkROC(ww, fedId, link, cab);
      bool skipROC = (roc < 8) ? false : (errorType != 0);
      if (skipROC) {
        err = true;
        perr = {getErrRawID(fedId, ww, errorType, cab), ww, errorType, fedId};
      } else {
        uint32_t rawId = cab->rawId[index];
        uint32_t rocInDet = cab->rocInDet[index];
        uint32_t moduleId = cab->moduleId[index];
        bool barrel = 1 == ((rawId >> 25) & 0x7);
        if (!cab->badRocs[index] && !es.modToUnp[index]) {
          uint32_t layer = 0;
          int side;
          if (barrel) {
            layer = (rawId >> 20) & 0xf;
            int module = (rawId >> 2) & 0x3ff;
            side = (module < 5) ? -1 : 1;
          } else {
            int panel = (rawId >> 10) & 0x3;
            side = (panel == 1) ? -1 : 1;
          }
          uint32_t row, col;
          bool bad;
          if (layer == 1) {
            col = (ww >> 15) & 0x3f;
            row = (ww >> 8) & 0x7f;
            bad = !((row < 80) & (col < 52));
          } else {
            uint32_t dcol = (ww >> 16) & 0x1f;
            uint32_t pxid = (ww >> 8) & 0xff;
            row = 80 - pxid / 2;
            col = dcol * 2 + pxid % 2;
            bad = !((dcol < 26) & (2 <= pxid) & (pxid < 162));
          }
          if (bad) {
            err = true;
            perr = {rawId, ww, 37, fedId};
          } else {
            // frameConversion (:72-138)
            bool minusSide = barrel ? (side == -1 && layer != 1) : true;
            int slopeRow, slopeCol, rowOffset, colOffset;
            if (minusSide == (rocInDet < 8)) {
              slopeRow = 1;
              slopeCol = -1;
              rowOffset = 0;
              colOffset = (minusSide ? 8 : 16) * 52 - int(rocInDet) * 52 - 1;
            } else {
              slopeRow = -1;
              slopeCol = 1;
              rowOffset = 159;
              colOffset = (minusSide ? int(rocInDet) - 8 : int(rocInDet)) * 52;
            }
            uint32_t gRow = rowOffset + slopeRow * int(row);
            uint32_t gCol = colOffset + slopeCol * int(col);
            xx = uint16_t(gRow);
            yy = uint16_t(gCol);
            adc = uint16_t(ww & 0xff);
            pdigi = gRow | (gCol << 11) | (min(uint32_t(adc), 1023u) << 22);
            mid = uint16_t(moduleId);
            rawIdOut = rawId;
          }
        }
      }
    }
    ws.pdigi[g] = pdigi;
    ws.rawIdArr[g] = rawIdOut;
    if (mid != kInvId && (mid >= kMaxModules || xx > 159 || yy > 415)) {
      atomicOr(&ws.ev[e].flags, kFlagBadInput);
      mid = kInvId;
    }
    // calibDigis (isRun2)
    if (mid != kInvId) {
      float conversionFactor = mid < 96 ? 50.f : 47.f;
      float offset = mid < 96 ? -670.f : -60.f;
      const PfRangeAndCols rc = gh->rangeAndCols[mid];
      unsigned int lengthOfColumnData = (rc.second - rc.first) / rc.nCols;
      unsigned int blocks = xx / gh->numberOfRowsAveragedOver;
      uint32_t o = rc.first + yy * lengthOfColumnData + 2 * blocks;
      if (o + 1 >= es.gainPayloadSize) o = 0;  // malformed gain ranges (validated at upload)
      uint8_t gb = es.gainPayload[o], pb = es.gainPayload[o + 1];
      float pedestal = float(unsigned(pb)) * gh->pedPrecision + gh->minPed;
      float gain = float(unsigned(gb)) * gh->gainPrecision + gh->minGain;
      if ((pb == gh->deadFlag) | (pb == gh->noisyFlag)) {
        mid = kInvId;
        adc = 0;
      } else {
        float vcal = float(int(adc)) * gain - pedestal * gain;
        adc = uint16_t(max(100, int(vcal * conversionFactor + offset)));
      }
    }
    ws.xx[g] = xx;
    ws.yy[g] = yy;
    ws.adc[g] = adc;
    ws.moduleInd[g] = mid;
    ws.clus[g] = int32_t(i);
    if (err) {
      uint32_t k = atomicAdd(&ws.ev[e].nErrors, 1u);
      if (k < kErrCap) {
        ws.errors[size_t(e) * kErrCap + k] = perr;
        ws.errWordIdx[size_t(e) * kErrCap + k] = i;
      } else {
        atomicOr(&ws.ev[e].flags, kFlagErrOverflow);
      }
    }
  }
}

// module-run boundaries (countModules): each run start is marked in a bitmap
// of the event's digis, which kSortModules reads in order
__global__ void kModuleBoundaries(Workspace ws, uint32_t nEvents) {
  const uint32_t total = ws.wordOffsets[nEvents];
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    uint16_t id = ws.moduleInd[g];
    if (id == kInvId) continue;
    uint32_t e = eventOfWord(ws.wordOffsets, nEvents, g);
    uint32_t start = ws.wordOffsets[e];
    int j = int(g) - 1;
    while (j >= int(start) && ws.moduleInd[j] == kInvId) --j;
    if (j < int(start) || ws.moduleInd[j] != id) {
      const uint32_t i = g - start;
      if (i < ws.cap.fedWords) atomicOr(&ws.scratchA[size_t(e) * ws.cap.scratch + (i >> 5)], 1u << (i & 31));
    }
  }
}

// the module-run starts of each event (<= 2000) in ascending order, from the boundary bitmap
__global__ void kSortModules(Workspace ws, uint32_t nEvents) {
  __shared__ uint32_t s[2048];
  __shared__ uint32_t scanShMod[33];
  __shared__ uint32_t sTmp[2048];
  __shared__ uint32_t sRuns;
  uint32_t e = blockIdx.x;
  EventCounters* c = ws.ev + e;
  uint32_t* ms = ws.moduleStart + size_t(e) * kModStride;
  // the run starts in position order: each thread takes a contiguous chunk
  // of the bitmap, a block scan of the chunks' bit counts places them
  {
    const uint32_t* bm = ws.scratchA + size_t(e) * ws.cap.scratch;
    const uint32_t nbw = (min(c->nWords, ws.cap.fedWords) + 31) / 32;
    const uint32_t chunk = (nbw + blockDim.x - 1) / blockDim.x;
    const uint32_t w0 = min(nbw, threadIdx.x * chunk), w1 = min(nbw, w0 + chunk);
    uint32_t mine = 0;
    for (uint32_t w = w0; w < w1; ++w) mine += __popc(bm[w]);
    uint32_t tot;
    uint32_t at = blockExclusiveScan(mine, scanShMod, &tot);
    for (uint32_t w = w0; w < w1; ++w) {
      uint32_t bits = bm[w];
      while (bits) {
        const uint32_t b = __ffs(bits) - 1;
        bits &= bits - 1;
        if (at < kMaxModules) s[at] = 32 * w + b;
        ++at;
      }
    }
    if (threadIdx.x == 0) sRuns = tot;
    __syncthreads();
  }
  // more than 2000 runs: the reference's counter stops at its capacity
  // (gpuClustering.h:33); the first 2000 in position order are kept, flagged
  if (threadIdx.x == 0) c->nModules = sRuns;
  uint32_t n = min(sRuns, kMaxModules);
  // A module whose digis come in more than one run (only in corrupted data:
  // a module is read out in one block per link) is clustered run by run by the
  // reference, whose serial build then overwrites the module's cluster count
  // and hit slots in loop order and whose CUDA build races on them.  Here the
  // first run is kept and the later runs are read as padding (zero words);
  // the event is flagged.
  __shared__ uint32_t sFirst[kMaxModules];
  __shared__ uint8_t sDrop[2048];
  __shared__ uint32_t sNDrop;
  const uint32_t start = ws.wordOffsets[e];
  const uint16_t* mind = ws.moduleInd + start;
  for (uint32_t i = threadIdx.x; i < kMaxModules; i += blockDim.x) sFirst[i] = 0xffffffffu;
  if (threadIdx.x == 0) sNDrop = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint16_t mid = mind[s[i]];
    if (mid < kMaxModules) atomicMin(&sFirst[mid], i);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint16_t mid = mind[s[i]];
    const bool drop = mid < kMaxModules && sFirst[mid] != i;
    sDrop[i] = drop ? 1 : 0;
    if (drop) atomicAdd(&sNDrop, 1u);
  }
  __syncthreads();
  if (sNDrop) {
    const uint32_t nw = c->nWords;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      if (!sDrop[i]) continue;
      const uint16_t mid = mind[s[i]];
      const uint32_t end = i + 1 < n ? s[i + 1] : nw;
      for (uint32_t g = s[i]; g < end; ++g) {
        const size_t w = size_t(start) + g;
        if (ws.moduleInd[w] != mid) continue;
        ws.moduleInd[w] = kInvId;
        ws.xx[w] = ws.yy[w] = ws.adc[w] = 0;
        ws.pdigi[w] = 0;
        ws.rawIdArr[w] = 0;
      }
    }
    __syncthreads();
    // drop the later runs from the list, keeping the others in order
    {
      uint32_t carry = 0;
      for (uint32_t i0 = 0; i0 < n; i0 += blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        const uint32_t keep = (i < n && !sDrop[i]) ? 1u : 0u;
        uint32_t tot;
        const uint32_t pre = blockExclusiveScan(keep, scanShMod, &tot);
        if (keep) sTmp[carry + pre] = s[i];
        carry += tot;
      }
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < carry; i += blockDim.x) s[i] = sTmp[i];
      __syncthreads();
    }
  }
  const uint32_t kept = n - sNDrop;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) ms[1 + i] = i < kept ? s[i] : 0u;
  if (threadIdx.x == 0) {
    ms[0] = kept;
    if (c->nModules > kMaxModules) c->flags |= kFlagTooManyRuns;
    c->nModules = kept;
    if (sNDrop) c->flags |= kFlagSplitModule;
  }
}

// findClus + clusterChargeCut: one block per (module run, event)
constexpr int kClusThreads = 256;
constexpr uint32_t kSmallPix = 128;  // modules up to this many pixels are clustered by one warp
constexpr int kSmallWarps = 8;
constexpr uint32_t kModCols = 416;  // pixel columns (y) of a module

// findClus + clusterChargeCut of one module run by the whole block (modules
// with more than kSmallPix pixels): column histogram, union-find with roots
// hooked under the smaller pixel index, numbering by ascending root.
__device__ void clusterModuleBlock(const Workspace& ws, uint32_t e, uint32_t module) {
  __shared__ uint16_t sx[PF_MAX_PIX_IN_MODULE], sy[PF_MAX_PIX_IN_MODULE];
  __shared__ int32_t lab[PF_MAX_PIX_IN_MODULE];
  __shared__ uint16_t colList[PF_MAX_PIX_IN_MODULE];
  __shared__ uint32_t colStart[420];
  __shared__ int32_t charge[PF_MAX_CLUS_PER_MODULE];
  __shared__ uint32_t scanSh[33];
  __shared__ uint32_t sFound, sNewTotal;

  const EventCounters* c = ws.ev + e;
  const uint32_t nModules = c->nModules;
  if (module >= nModules) return;
  const uint32_t start = c->wordStart, nW = c->nWords;
  const uint32_t* ms = ws.moduleStart + size_t(e) * kModStride;
  const uint32_t firstPixel = ms[1 + module];
  uint32_t msize = (module + 1 < nModules) ? ms[2 + module] : nW;
  const uint16_t thisModuleId = ws.moduleInd[start + firstPixel];
  if (thisModuleId >= kMaxModules) {
    if (threadIdx.x == 0) ws.moduleId[size_t(e) * kModStride + module] = 0xffffffffu;
    return;
  }
  const uint32_t moduleEnd = msize;  // the run's end before the 4000-pixel cap
  if (msize - firstPixel > PF_MAX_PIX_IN_MODULE) {
    if (threadIdx.x == 0) atomicOr(&ws.ev[e].flags, kFlagModuleTooBig);
    msize = firstPixel + PF_MAX_PIX_IN_MODULE;
  }
  const uint32_t np = msize - firstPixel;
  uint16_t* gmid = ws.moduleInd + start + firstPixel;
  int32_t* gclus = ws.clus + start + firstPixel;

  for (uint32_t k = threadIdx.x; k < 420; k += blockDim.x) colStart[k] = 0;
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
    bool valid = gmid[k] != kInvId;
    uint16_t y = ws.yy[start + firstPixel + k];
    sx[k] = ws.xx[start + firstPixel + k];
    sy[k] = valid ? y : uint16_t(0xffff);
    lab[k] = int32_t(k);
    if (valid) atomicAdd(&colStart[y + 1], 1u);
  }
  __syncthreads();
  // column offsets (exclusive), 419 entries
  {
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < 420; b0 += blockDim.x) {
      uint32_t b = b0 + threadIdx.x;
      uint32_t v = b < 420 ? colStart[b] : 0u;
      uint32_t tot;
      uint32_t inc = blockExclusiveScan(v, scanSh, &tot) + v;
      if (b < 420) colStart[b] = carry + inc;
      carry += tot;
      __syncthreads();
    }
  }
  // fill column lists (order inside a column is irrelevant for components)
  for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
    uint16_t y = sy[k];
    if (y == 0xffff) continue;
    uint32_t pos = atomicAdd(&colStart[y], 1u);
    colList[pos] = uint16_t(k);
  }
  __syncthreads();
  // after the fill colStart[y] points at the end of column y; column y spans
  // [colStart[y-1], colStart[y]) with colStart[-1] = 0
  auto colBegin = [&](uint32_t y) { return y == 0 ? 0u : colStart[y - 1]; };
  auto find = [&](int32_t a) {
    while (true) {
      int32_t p = lab[a];
      if (p == a) return a;
      int32_t gp = lab[p];
      if (gp != p) lab[a] = gp;  // path halving (benign race: only ever lowers towards a root)
      a = p;
    }
  };
  // union of 8-neighbours (|dx| <= 1, dy in {0, 1}); roots hook under the smaller index
  for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
    uint16_t y = sy[k];
    if (y == 0xffff) continue;
    int xk = sx[k];
    for (uint32_t yy = y; yy <= uint32_t(y) + 1 && yy < 418; ++yy) {
      uint32_t b = colBegin(yy), en = colStart[yy];
      for (uint32_t p = b; p < en; ++p) {
        uint32_t m = colList[p];
        if (yy == y && m <= k) continue;
        if (abs(int(sx[m]) - xk) > 1) continue;
        int32_t a = int32_t(k), bb = int32_t(m);
        while (true) {
          a = find(a);
          bb = find(bb);
          if (a == bb) break;
          if (a > bb) {
            int32_t t = a;
            a = bb;
            bb = t;
          }
          int32_t old = atomicCAS(&lab[bb], bb, a);
          if (old == bb) break;
          bb = old;
        }
      }
    }
  }
  __syncthreads();
  // flatten: read-only walk to the root (path halving here would race with
  // the final root writes of other threads and could leave a non-root label)
  for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
    if (sy[k] == 0xffff) continue;
    int32_t r = lab[k];
    while (lab[r] != r) r = lab[r];
    lab[k] = r;
  }
  __syncthreads();
  // number the roots in ascending pixel order
  {
    uint32_t carry = 0;
    for (uint32_t k0 = 0; k0 < np; k0 += blockDim.x) {
      uint32_t k = k0 + threadIdx.x;
      uint32_t isRoot = (k < np && sy[k] != 0xffff && lab[k] == int32_t(k)) ? 1u : 0u;
      uint32_t tot;
      uint32_t pre = blockExclusiveScan(isRoot, scanSh, &tot);
      if (isRoot) colList[k] = uint16_t(carry + pre);  // colList reused as root rank
      carry += tot;
    }
    if (threadIdx.x == 0) sFound = carry;
  }
  __syncthreads();
  const uint32_t found = sFound;
  // cluster id of each pixel (serial findClus numbering)
  for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
    if (sy[k] == 0xffff) continue;
    lab[k] = int32_t(colList[lab[k]]);
  }
  for (uint32_t k = threadIdx.x; k < PF_MAX_CLUS_PER_MODULE; k += blockDim.x) charge[k] = 0;
  __syncthreads();
  // ---- clusterChargeCut
  uint32_t nclus = found;
  if (nclus > uint32_t(PF_MAX_CLUS_PER_MODULE)) {
    for (uint32_t k = threadIdx.x; k < np; k += blockDim.x)
      if (sy[k] != 0xffff && lab[k] >= PF_MAX_CLUS_PER_MODULE) {
        sy[k] = 0xfffe;  // becomes invalid with cluster id InvId
      }
    if (threadIdx.x == 0) atomicOr(&ws.ev[e].flags, kFlagModuleTooBig);
    nclus = PF_MAX_CLUS_PER_MODULE;
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < np; k += blockDim.x)
    if (sy[k] < 0xfffe) atomicAdd(&charge[lab[k]], int32_t(ws.adc[start + firstPixel + k]));
  __syncthreads();
  const int chargeCut = thisModuleId < 96 ? 2000 : 4000;
  // inclusive scan of ok flags -> new ids (stored back into charge[] as id+1, 0 = bad)
  {
    uint32_t carry = 0;
    for (uint32_t k0 = 0; k0 < nclus; k0 += blockDim.x) {
      uint32_t k = k0 + threadIdx.x;
      uint32_t ok = (k < nclus && charge[k] > chargeCut) ? 1u : 0u;
      uint32_t tot;
      uint32_t pre = blockExclusiveScan(ok, scanSh, &tot);
      if (k < nclus) charge[k] = ok ? int32_t(carry + pre + 1) : 0;
      carry += tot;
    }
    if (threadIdx.x == 0) sNewTotal = carry;
  }
  __syncthreads();
  const uint32_t newTotal = sNewTotal;
  const bool allGood = (nclus == newTotal);
  for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
    uint16_t y = sy[k];
    if (y == 0xffff) {
      gclus[k] = -9999;
    } else if (y == 0xfffe) {
      gmid[k] = kInvId;
      gclus[k] = kInvId;
    } else if (allGood) {
      gclus[k] = lab[k];
    } else {
      int32_t nid = charge[lab[k]];
      if (nid == 0) {
        gclus[k] = kInvId;
        gmid[k] = kInvId;
      } else {
        gclus[k] = nid - 1;
      }
    }
  }
  // pixels past the 4000-pixel cap kept their initial index (countModules);
  // the cluster-count cap then invalidates them, as it does every index of
  // 1024 and above (gpuClusterChargeCut.h:46-59).  (With at most 1024
  // clusters the reference's charge sums index past their array: undefined,
  // flagged, left as is.)
  if (found > uint32_t(PF_MAX_CLUS_PER_MODULE))
    for (uint32_t g = firstPixel + np + threadIdx.x; g < moduleEnd; g += blockDim.x)
      if (ws.moduleInd[start + g] == thisModuleId) {
        ws.moduleInd[start + g] = kInvId;
        ws.clus[start + g] = kInvId;
      }
  if (threadIdx.x == 0) {
    ws.clusInModule[size_t(e) * kModStride + thisModuleId] = (found == 0 || allGood) ? found : newTotal;
    ws.moduleId[size_t(e) * kModStride + module] = thisModuleId;
  }
  __syncthreads();
}

// the modules queued by kFindClustersSmall, one block each
__global__ void __launch_bounds__(kClusThreads) kFindClustersBig(Workspace ws) {
  const uint32_t e = blockIdx.y;
  const uint32_t n = min(ws.ev[e].nBigMod, kMaxModules);
  const uint32_t* list = ws.bigSeg + size_t(e) * kBigSegCap;
  for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) clusterModuleBlock(ws, e, list[k]);
}

// One warp per module run.  Runs of at most kSmallPix pixels are clustered
// here: the pixels binned by column (a counting sort in shared memory), each
// pixel's neighbours (|dx| <= 1, |dy| <= 1) looked up in its own column and
// the next, union-find in shared memory, roots ranked by ascending pixel
// index, then the charge cut with renumbering -- the same numbering as the
// block path.  Larger runs are queued for kFindClustersBig.
// (256, 7): at most 32 registers (no spills), seven blocks per SM beside their 28 KB
// of shared memory (214 -> 205 us per 64-event batch against six)
__global__ void __launch_bounds__(kSmallWarps * 32, 7) kFindClustersSmall(Workspace ws) {
  __shared__ uint16_t sxA[kSmallWarps][kSmallPix], syA[kSmallWarps][kSmallPix], rkA[kSmallWarps][kSmallPix];
  __shared__ int32_t labA[kSmallWarps][kSmallPix], chgA[kSmallWarps][kSmallPix];
  __shared__ uint32_t colA[kSmallWarps][kModCols];  // column bins: counts, then bin ends
  __shared__ uint8_t ordA[kSmallWarps][kSmallPix];  // pixels ordered by column
  const uint32_t e = blockIdx.y, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t module = blockIdx.x * kSmallWarps + w;
  EventCounters* c = ws.ev + e;
  const uint32_t nModules = c->nModules;
  if (module >= nModules || module >= kMaxModules) return;
  const uint32_t start = c->wordStart, nW = c->nWords;
  const uint32_t* ms = ws.moduleStart + size_t(e) * kModStride;
  const uint32_t firstPixel = ms[1 + module];
  const uint32_t msize = (module + 1 < nModules) ? ms[2 + module] : nW;
  const uint16_t thisModuleId = ws.moduleInd[start + firstPixel];
  if (thisModuleId >= kMaxModules) {
    if (lane == 0) ws.moduleId[size_t(e) * kModStride + module] = 0xffffffffu;
    return;
  }
  const uint32_t np = msize - firstPixel;
  if (np > kSmallPix) {
    if (lane == 0) {
      const uint32_t k = atomicAdd(&c->nBigMod, 1u);
      if (k < kMaxModules) ws.bigSeg[size_t(e) * kBigSegCap + k] = module;
    }
    return;
  }
  uint16_t* sx = sxA[w];
  uint16_t* sy = syA[w];
  uint16_t* rk = rkA[w];
  int32_t* lab = labA[w];
  int32_t* chg = chgA[w];
  uint16_t* gmid = ws.moduleInd + start + firstPixel;
  int32_t* gclus = ws.clus + start + firstPixel;
  // a lane holds at most kSmallPix / 32 pixels: their charges stay in registers
  int32_t adcR[kSmallPix / 32];
  bool colOk = true;  // every valid pixel inside the module's columns
#pragma unroll
  for (uint32_t u = 0; u < kSmallPix / 32; ++u) {
    const uint32_t k = lane + 32 * u;
    adcR[u] = 0;
    if (k < np) {
      const bool valid = gmid[k] != kInvId;
      const uint16_t y = ws.yy[start + firstPixel + k];
      sx[k] = ws.xx[start + firstPixel + k];
      sy[k] = valid ? y : uint16_t(0xffff);
      adcR[u] = int32_t(ws.adc[start + firstPixel + k]);
      lab[k] = int32_t(k);
      colOk &= !valid || y < kModCols;
    }
  }
  colOk = __all_sync(0xffffffffu, colOk);
  __syncwarp();
  auto find = [&](int32_t a) {
    while (true) {
      const int32_t p = lab[a];
      if (p == a) return a;
      const int32_t gp = lab[p];
      if (gp != p) lab[a] = gp;  // path halving: only ever moves towards a root
      a = p;
    }
  };
  // union of neighbours (|dx| <= 1, |dy| <= 1).  The components, and with
  // them the roots (the smallest pixel index of each), do not depend on the
  // order the neighbour pairs are found in.
  auto unite = [&](int32_t a, int32_t bb) {
    while (true) {
      a = find(a);
      bb = find(bb);
      if (a == bb) break;
      if (a > bb) {
        const int32_t t = a;
        a = bb;
        bb = t;
      }
      const int32_t old = atomicCAS(&lab[bb], bb, a);
      if (old == bb) break;
      bb = old;
    }
  };
  if (colOk) {
    // pixels binned by column (counting sort): a pixel's neighbours lie in
    // its own column and the next one
    uint32_t* col = colA[w];
    uint8_t* ord = ordA[w];
    for (uint32_t b = lane; b < kModCols; b += 32) col[b] = 0;
    __syncwarp();
    for (uint32_t k = lane; k < np; k += 32)
      if (sy[k] != 0xffff) atomicAdd(&col[sy[k]], 1u);
    __syncwarp();
    {
      constexpr uint32_t per = kModCols / 32;  // consecutive bins per lane
      static_assert(kModCols % 32 == 0, "column bins per lane");
      uint32_t v[per], run = 0;
#pragma unroll
      for (uint32_t j = 0; j < per; ++j) {
        v[j] = run;
        run += col[lane * per + j];
      }
      const uint32_t base = warpInclusiveScan(run) - run;
#pragma unroll
      for (uint32_t j = 0; j < per; ++j) col[lane * per + j] = base + v[j];
    }
    __syncwarp();
    for (uint32_t k = lane; k < np; k += 32)
      if (sy[k] != 0xffff) ord[atomicAdd(&col[sy[k]], 1u)] = uint8_t(k);
    __syncwarp();
    // col[b] is now the end of bin b and the start of bin b + 1
    for (uint32_t k = lane; k < np; k += 32) {
      const uint16_t yk = sy[k];
      if (yk == 0xffff) continue;
      const int xk = sx[k];
      const uint32_t p0 = yk > 0 ? col[yk - 1] : 0u;
      const uint32_t p1 = col[min(uint32_t(yk) + 1u, kModCols - 1u)];
      for (uint32_t p = p0; p < p1; ++p) {
        const uint32_t m = ord[p];
        if (m != k && abs(int(sx[m]) - xk) <= 1) unite(int32_t(k), int32_t(m));
      }
    }
  } else {
    for (uint32_t k = lane; k < np; k += 32) {
      const uint16_t yk = sy[k];
      if (yk == 0xffff) continue;
      const int xk = sx[k];
      for (uint32_t m = k + 1; m < np; ++m) {
        const uint16_t ym = sy[m];
        if (ym == 0xffff || abs(int(ym) - int(yk)) > 1 || abs(int(sx[m]) - xk) > 1) continue;
        unite(int32_t(k), int32_t(m));
      }
    }
  }
  __syncwarp();
  // flatten by a read-only walk (path halving here could race with the root
  // writes of other lanes)
  for (uint32_t k = lane; k < np; k += 32) {
    if (sy[k] == 0xffff) continue;
    int32_t r = lab[k];
    while (lab[r] != r) r = lab[r];
    lab[k] = r;
  }
  __syncwarp();
  // rank the roots in ascending pixel order
  uint32_t found = 0;
  for (uint32_t k0 = 0; k0 < np; k0 += 32) {
    const uint32_t k = k0 + lane;
    const bool isRoot = k < np && sy[k] != 0xffff && lab[k] == int32_t(k);
    const uint32_t m = __ballot_sync(0xffffffffu, isRoot);
    if (isRoot) rk[k] = uint16_t(found + __popc(m & lanemaskLt()));
    found += __popc(m);
  }
  for (uint32_t k = lane; k < found; k += 32) chg[k] = 0;
  __syncwarp();
#pragma unroll
  for (uint32_t u = 0; u < kSmallPix / 32; ++u) {
    const uint32_t k = lane + 32 * u;
    if (k >= np || sy[k] == 0xffff) continue;
    const int32_t id = rk[lab[k]];
    lab[k] = id;
    atomicAdd(&chg[id], adcR[u]);
  }
  __syncwarp();
  // charge cut: new ids (stored as id + 1, 0 = removed)
  const int chargeCut = thisModuleId < 96 ? 2000 : 4000;
  uint32_t newTotal = 0;
  for (uint32_t k0 = 0; k0 < found; k0 += 32) {
    const uint32_t k = k0 + lane;
    const bool ok = k < found && chg[k] > chargeCut;
    const uint32_t m = __ballot_sync(0xffffffffu, ok);
    if (k < found) chg[k] = ok ? int32_t(newTotal + __popc(m & lanemaskLt()) + 1) : 0;
    newTotal += __popc(m);
  }
  __syncwarp();
  const bool allGood = (found == newTotal);
  for (uint32_t k = lane; k < np; k += 32) {
    if (sy[k] == 0xffff) {
      gclus[k] = -9999;
    } else if (allGood) {
      gclus[k] = lab[k];
    } else {
      const int32_t nid = chg[lab[k]];
      if (nid == 0) {
        gclus[k] = kInvId;
        gmid[k] = kInvId;
      } else {
        gclus[k] = nid - 1;
      }
    }
  }
  if (lane == 0) {
    ws.clusInModule[size_t(e) * kModStride + thisModuleId] = (found == 0 || allGood) ? found : newTotal;
    ws.moduleId[size_t(e) * kModStride + module] = thisModuleId;
  }
}

// fillHitsModuleStart + setHitsLayerStart + beam-spot corrected average geometry
__global__ void kHitsModuleStart(DeviceES es, Workspace ws) {
  __shared__ uint32_t scanSh[33];
  uint32_t e = blockIdx.x;
  const uint32_t* cim = ws.clusInModule + size_t(e) * kModStride;
  uint32_t* cms = ws.clusModuleStart + size_t(e) * kModStride;
  uint32_t carry = 0;
  for (uint32_t i0 = 0; i0 < kMaxModules; i0 += blockDim.x) {
    uint32_t i = i0 + threadIdx.x;
    uint32_t v = i < kMaxModules ? min(uint32_t(PF_MAX_CLUS_PER_MODULE), cim[i]) : 0u;
    uint32_t tot;
    uint32_t inc = blockExclusiveScan(v, scanSh, &tot) + v;
    if (i < kMaxModules) cms[i + 1] = min(carry + inc, ws.cap.hits);
    carry += tot;
  }
  if (threadIdx.x == 0) cms[0] = 0;
  __syncthreads();
  EventCounters* c = ws.ev + e;
  if (threadIdx.x == 0) {
    c->nHits = cms[kMaxModules];
    if (carry > ws.cap.hits) c->flags |= kFlagHitOverflow;
  }
  if (threadIdx.x < 11) c->layerStart[threadIdx.x] = cms[es.lg->layerStart[threadIdx.x]];
  PfAverageGeometry* agc = ws.agc + e;
  const PfAverageGeometry* ag = es.ag;
  const PfBeamSpot* bs = es.bs;
  for (uint32_t il = threadIdx.x; il < PF_N_LADDERS_BARREL; il += blockDim.x) {
    agc->ladderZ[il] = ag->ladderZ[il] - bs->z;
    agc->ladderX[il] = ag->ladderX[il] - bs->x;
    agc->ladderY[il] = ag->ladderY[il] - bs->y;
    agc->ladderR[il] = sqrtf(agc->ladderX[il] * agc->ladderX[il] + agc->ladderY[il] * agc->ladderY[il]);
    agc->ladderMinZ[il] = ag->ladderMinZ[il] - bs->z;
    agc->ladderMaxZ[il] = ag->ladderMaxZ[il] - bs->z;
  }
  if (threadIdx.x == 0) {
    agc->endCapZ[0] = ag->endCapZ[0] - bs->z;
    agc->endCapZ[1] = ag->endCapZ[1] - bs->z;
  }
}

// getHits: one block per (module run, event); all clusters of a module in one pass
// gpuPixelRecHits.h:100-207 for one cluster: sizes, CPE position and
// errors, global position, iphi; written to hit slot h of event e
__device__ __forceinline__ void writeHit(const Workspace& ws, size_t hb, uint32_t h, uint32_t me,
                                         const PfDetParams& dp, const PfCommonParams& cp, const PfBeamSpot& bs,
                                         uint32_t minRow, uint32_t maxRow, uint32_t minCol, uint32_t maxCol,
                                         int32_t Qfx, int32_t Qlx, int32_t Qfy, int32_t Qly, int32_t chg) {
  uint16_t llx = uint16_t(minRow + 1), lly = uint16_t(minCol + 1);
  uint16_t urx = uint16_t(maxRow), ury = uint16_t(maxCol);
  uint16_t llxl = localX(llx), llyl = localY(lly), urxl = localX(urx), uryl = localY(ury);
  int mx = llxl + urxl, my = llyl + uryl;
  int xsize = int(urxl) + 2 - int(llxl);
  int ysize = int(uryl) + 2 - int(llyl);
  bool bigMinX = isBigPixX(uint16_t(minRow)), bigMaxX = isBigPixX(uint16_t(maxRow));
  bool bigMinY = isBigPixY(uint16_t(minCol)), bigMaxY = isBigPixY(uint16_t(maxCol));
  if (bigMinX) ++xsize;
  if (bigMaxX) ++xsize;
  if (bigMinY) ++ysize;
  if (bigMaxY) ++ysize;
  // the reference computes these ratios in double precision
  int unbalanceX = int(8. * double(fabsf(float(Qfx - Qlx))) / double(float(Qfx + Qlx)));
  int unbalanceY = int(8. * double(fabsf(float(Qfy - Qly))) / double(float(Qfy + Qly)));
  xsize = 8 * xsize - unbalanceX;
  ysize = 8 * ysize - unbalanceY;
  int16_t sxv = int16_t(min(xsize, 1023)), syv = int16_t(min(ysize, 1023));
  if (minRow == 0 || maxRow == 159) sxv = int16_t(-sxv);
  if (minCol == 0 || maxCol == 415) syv = int16_t(-syv);
  float xPos = dp.shiftX + cp.pitchX * (0.5f * float(mx) + float(-81));
  float yPos = dp.shiftY + cp.pitchY * (0.5f * float(my) + float(-216));
  float gvz = -1.f / dp.z0;
  float cotalpha = (xPos - dp.x0) * gvz, cotbeta = (yPos - dp.y0) * gvz;
  float thickness = dp.isBarrel ? cp.thicknessB : cp.thicknessE;
  float xcorr = cpeCorrection(int(maxRow - minRow), Qfx, Qlx, llxl, urxl, dp.chargeWidthX,
                              thickness, cotalpha, cp.pitchX, bigMinX, bigMaxX);
  float ycorr = cpeCorrection(int(maxCol - minCol), Qfy, Qly, llyl, uryl, dp.chargeWidthY,
                              thickness, cotbeta, cp.pitchY, bigMinY, bigMaxY);
  float xpos = xPos + xcorr, ypos = yPos + ycorr;
  float xerr = 0.0050f, yerr = 0.0085f;
  uint32_t sx = maxRow - minRow, sy = maxCol - minCol;
  bool isEdgeX = minRow == 0 || maxRow == 159;
  bool isEdgeY = minCol == 0 || maxCol == 415;
  uint32_t ix = (0 == sx), iy = (0 == sy);
  ix += (0 == sx) && bigMinX;
  iy += (0 == sy) && bigMinY;
  if (!isEdgeX) xerr = dp.sx[ix];
  if (!isEdgeY) yerr = dp.sy[iy];
  const PfFrame& f = dp.frame;
  float xg = f.R11 * xpos + f.R21 * ypos;
  float yg = f.R12 * xpos + f.R22 * ypos;
  float zg = f.R13 * xpos + f.R23 * ypos;
  xg += f.px;
  yg += f.py;
  zg += f.pz;
  xg -= bs.x;
  yg -= bs.y;
  zg -= bs.z;
  ws.charge[hb + h] = chg;
  ws.detInd[hb + h] = uint16_t(me);
  ws.xl[hb + h] = xpos;
  ws.yl[hb + h] = ypos;
  ws.xsize[hb + h] = sxv;
  ws.ysize[hb + h] = syv;
  ws.xerr[hb + h] = xerr * xerr;
  ws.yerr[hb + h] = yerr * yerr;
  ws.xg[hb + h] = xg;
  ws.yg[hb + h] = yg;
  ws.zg[hb + h] = zg;
  ws.rg[hb + h] = sqrtf(xg * xg + yg * yg);
  ws.iphi[hb + h] = unsafeAtan2s7(yg, xg);
}

constexpr int kHitThreads = 128;
constexpr int kHitBatch = 256;
constexpr uint32_t kSmallClus = 32;  // modules with at most this many clusters are handled by one warp
constexpr int kHitWarps = 8;

// getHits for one module run by the whole block (modules with more than
// kSmallClus clusters): per-cluster extremes and edge charges by shared
// atomics, in batches of kHitBatch clusters
__device__ void hitsModuleBlock(const DeviceES& es, const Workspace& ws, uint32_t e, uint32_t module) {
  __shared__ uint32_t minRow[kHitBatch], maxRow[kHitBatch], minCol[kHitBatch], maxCol[kHitBatch];
  __shared__ int32_t Qfx[kHitBatch], Qlx[kHitBatch], Qfy[kHitBatch], Qly[kHitBatch], chg[kHitBatch];
  const EventCounters* c = ws.ev + e;
  const uint32_t nModules = c->nModules;
  if (module >= nModules) return;
  const uint32_t me = ws.moduleId[size_t(e) * kModStride + module];
  if (me >= es.nDet) return;  // runs the clustering rejected carry no valid module id
  const int nclus = int(ws.clusInModule[size_t(e) * kModStride + me]);
  if (nclus == 0) return;
  const uint32_t start = c->wordStart, nW = c->nWords;
  const uint32_t* ms = ws.moduleStart + size_t(e) * kModStride;
  const uint32_t first = ms[1 + module];
  const uint32_t last = (module + 1 < nModules) ? ms[2 + module] : nW;
  const PfDetParams& dp = es.det[me];
  const PfCommonParams& cp = *es.common;
  const PfBeamSpot& bs = *es.bs;
  const size_t hb = size_t(e) * ws.cap.hits;
  const uint32_t cmsMe = ws.clusModuleStart[size_t(e) * kModStride + me];
  for (int startClus = 0; startClus < nclus; startClus += kHitBatch) {
    int nIn = min(kHitBatch, nclus - startClus);
    int lastClus = startClus + nIn;
    for (int k = threadIdx.x; k < nIn; k += blockDim.x) {
      minRow[k] = minCol[k] = 0xffffffffu;
      maxRow[k] = maxCol[k] = 0;
      chg[k] = Qfx[k] = Qlx[k] = Qfy[k] = Qly[k] = 0;
    }
    __syncthreads();
    for (uint32_t i = first + threadIdx.x; i < last; i += blockDim.x) {
      uint16_t id = ws.moduleInd[start + i];
      if (id == kInvId || id != me) continue;
      int cl = ws.clus[start + i];
      if (cl < startClus || cl >= lastClus) continue;
      cl -= startClus;
      uint32_t x = ws.xx[start + i], y = ws.yy[start + i];
      atomicMin(&minRow[cl], x);
      atomicMax(&maxRow[cl], x);
      atomicMin(&minCol[cl], y);
      atomicMax(&maxCol[cl], y);
    }
    __syncthreads();
    for (uint32_t i = first + threadIdx.x; i < last; i += blockDim.x) {
      uint16_t id = ws.moduleInd[start + i];
      if (id == kInvId || id != me) continue;
      int cl = ws.clus[start + i];
      if (cl < startClus || cl >= lastClus) continue;
      cl -= startClus;
      uint32_t x = ws.xx[start + i], y = ws.yy[start + i];
      int32_t ch = ws.adc[start + i];
      atomicAdd(&chg[cl], ch);
      if (minRow[cl] == x) atomicAdd(&Qfx[cl], ch);
      if (maxRow[cl] == x) atomicAdd(&Qlx[cl], ch);
      if (minCol[cl] == y) atomicAdd(&Qfy[cl], ch);
      if (maxCol[cl] == y) atomicAdd(&Qly[cl], ch);
    }
    __syncthreads();
    for (int ic = threadIdx.x; ic < nIn; ic += blockDim.x) {
      uint32_t h = cmsMe + startClus + ic;
      if (h >= ws.cap.hits) continue;
      writeHit(ws, hb, h, me, dp, cp, bs, minRow[ic], maxRow[ic], minCol[ic], maxCol[ic], Qfx[ic], Qlx[ic], Qfy[ic],
               Qly[ic], chg[ic]);
    }
    __syncthreads();
  }
}

// the modules queued by kGetHitsSmall, one block each
__global__ void __launch_bounds__(kHitThreads) kGetHitsBig(DeviceES es, Workspace ws) {
  const uint32_t e = blockIdx.y;
  const uint32_t n = min(ws.ev[e].nBigHitMod, kMaxModules);
  const uint32_t* list = ws.bigSeg + size_t(e) * kBigSegCap;
  for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) hitsModuleBlock(es, ws, e, list[k]);
}

// One warp per module run with at most kSmallClus clusters (the others are
// queued for kGetHitsBig): lanes walk the pixels, the per-cluster extremes
// and edge charges collect in per-warp shared arrays, lane k writes hit k.
// (256, 6): 48 -> 40 registers (137 -> 131 us per 64-event batch)
__global__ void __launch_bounds__(kHitWarps * 32, 6) kGetHitsSmall(DeviceES es, Workspace ws) {
  __shared__ uint32_t mnR[kHitWarps][kSmallClus], mxR[kHitWarps][kSmallClus], mnC[kHitWarps][kSmallClus],
      mxC[kHitWarps][kSmallClus];
  __shared__ int32_t qfx[kHitWarps][kSmallClus], qlx[kHitWarps][kSmallClus], qfy[kHitWarps][kSmallClus],
      qly[kHitWarps][kSmallClus], chA[kHitWarps][kSmallClus];
  const uint32_t e = blockIdx.y, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t module = blockIdx.x * kHitWarps + w;
  EventCounters* c = ws.ev + e;
  const uint32_t nModules = c->nModules;
  if (module >= nModules || module >= kMaxModules) return;
  const uint32_t me = ws.moduleId[size_t(e) * kModStride + module];
  if (me >= es.nDet) return;  // runs the clustering rejected carry no valid module id
  const uint32_t nclus = ws.clusInModule[size_t(e) * kModStride + me];
  if (nclus == 0) return;
  if (nclus > kSmallClus) {
    if (lane == 0) {
      const uint32_t k = atomicAdd(&c->nBigHitMod, 1u);
      if (k < kMaxModules) ws.bigSeg[size_t(e) * kBigSegCap + k] = module;
    }
    return;
  }
  const uint32_t start = c->wordStart, nW = c->nWords;
  const uint32_t* ms = ws.moduleStart + size_t(e) * kModStride;
  const uint32_t first = ms[1 + module];
  const uint32_t last = (module + 1 < nModules) ? ms[2 + module] : nW;
  uint32_t* minRow = mnR[w];
  uint32_t* maxRow = mxR[w];
  uint32_t* minCol = mnC[w];
  uint32_t* maxCol = mxC[w];
  int32_t* Qfx = qfx[w];
  int32_t* Qlx = qlx[w];
  int32_t* Qfy = qfy[w];
  int32_t* Qly = qly[w];
  int32_t* chg = chA[w];
  if (lane < nclus) {
    minRow[lane] = minCol[lane] = 0xffffffffu;
    maxRow[lane] = maxCol[lane] = 0;
    chg[lane] = Qfx[lane] = Qlx[lane] = Qfy[lane] = Qly[lane] = 0;
  }
  __syncwarp();
  for (uint32_t i = first + lane; i < last; i += 32) {
    const uint16_t id = ws.moduleInd[start + i];
    if (id == kInvId || id != me) continue;
    const int cl = ws.clus[start + i];
    if (cl < 0 || cl >= int(nclus)) continue;
    const uint32_t x = ws.xx[start + i], y = ws.yy[start + i];
    atomicMin(&minRow[cl], x);
    atomicMax(&maxRow[cl], x);
    atomicMin(&minCol[cl], y);
    atomicMax(&maxCol[cl], y);
  }
  __syncwarp();
  for (uint32_t i = first + lane; i < last; i += 32) {
    const uint16_t id = ws.moduleInd[start + i];
    if (id == kInvId || id != me) continue;
    const int cl = ws.clus[start + i];
    if (cl < 0 || cl >= int(nclus)) continue;
    const uint32_t x = ws.xx[start + i], y = ws.yy[start + i];
    const int32_t ch = ws.adc[start + i];
    atomicAdd(&chg[cl], ch);
    if (minRow[cl] == x) atomicAdd(&Qfx[cl], ch);
    if (maxRow[cl] == x) atomicAdd(&Qlx[cl], ch);
    if (minCol[cl] == y) atomicAdd(&Qfy[cl], ch);
    if (maxCol[cl] == y) atomicAdd(&Qly[cl], ch);
  }
  __syncwarp();
  if (lane < nclus) {
    const uint32_t h = ws.clusModuleStart[size_t(e) * kModStride + me] + lane;
    if (h < ws.cap.hits)
      writeHit(ws, size_t(e) * ws.cap.hits, h, me, es.det[me], *es.common, *es.bs, minRow[lane], maxRow[lane],
               minCol[lane], maxCol[lane], Qfx[lane], Qlx[lane], Qfy[lane], Qly[lane], chg[lane]);
  }
}

__device__ __forceinline__ uint32_t phiBinOf(int16_t t) { return uint32_t((int(t) >> 9) & 127); }
__device__ __forceinline__ uint32_t layerOfHit(const uint32_t* ls, uint32_t i) {
  uint32_t l = 0;
#pragma unroll
  for (int k = 1; k < 10; ++k) l += (i >= ls[k]) ? 1u : 0u;
  return l;
}

// phi histogram: count per (layer, bin)
__global__ void kPhiCount(Workspace ws) {
  uint32_t e = blockIdx.y;
  const EventCounters* c = ws.ev + e;
  uint32_t nt = c->layerStart[10];
  uint32_t* off = ws.phiOff + size_t(e) * kPhiStride;
  const int16_t* iphi = ws.iphi + size_t(e) * ws.cap.hits;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
    uint32_t b = phiBinOf(iphi[i]) + 128 * layerOfHit(c->layerStart, i);
    atomicAdd(&off[b], 1u);
  }
}

// fill (unordered within a bin); off holds the exclusive scan, cursor counts
__global__ void kPhiFill(Workspace ws, uint32_t* cursor) {
  uint32_t e = blockIdx.y;
  const EventCounters* c = ws.ev + e;
  uint32_t nt = c->layerStart[10];
  const uint32_t* off = ws.phiOff + size_t(e) * kPhiStride;
  uint32_t* cur = cursor + size_t(e) * kPhiStride;
  const int16_t* iphi = ws.iphi + size_t(e) * ws.cap.hits;
  uint32_t* bins = ws.phiBins + size_t(e) * ws.cap.hits;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
    uint32_t b = phiBinOf(iphi[i]) + 128 * layerOfHit(c->layerStart, i);
    uint32_t p = atomicAdd(&cur[b], 1u);
    bins[off[b] + p] = i;
  }
}

// order every bin by descending hit index (the serial fill order); one warp per bin
__global__ void kPhiSort(Workspace ws) {
  uint32_t e = blockIdx.y;
  uint32_t b = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (b >= kPhiTot - 1) return;
  if (ws.ev[e].nHits == 0) return;
  const uint32_t* off = ws.phiOff + size_t(e) * kPhiStride;
  uint32_t* bins = ws.phiBins + size_t(e) * ws.cap.hits;
  warpSortSegment(bins + off[b], off[b + 1] - off[b], true);
}

// packed copy of the hits in phi-histogram order, read as contiguous
// candidate ranges by the doublet search
__global__ void kPhiRec(Workspace ws) {
  const uint32_t e = blockIdx.y;
  const uint32_t n = ws.phiOff[size_t(e) * kPhiStride + kPhiTot - 1];
  const size_t hb = size_t(e) * ws.cap.hits;
  const uint32_t* bins = ws.phiBins + hb;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t h = bins[p];
    uint4 r;
    r.x = __float_as_uint(ws.zg[hb + h]);
    r.y = __float_as_uint(ws.rg[hb + h]);
    r.z = uint32_t(uint16_t(ws.iphi[hb + h])) | (uint32_t(uint16_t(ws.ysize[hb + h])) << 16);
    // the module index saturates at 2047, which the doublet search rejects
    // like any index above 2000; the hit index takes the upper 21 bits
    r.w = min(uint32_t(ws.detInd[hb + h]), 2047u) | (h << 11);
    ws.phiRec[hb + p] = r;
  }
}

__global__ void kZeroU32(uint32_t* p, size_t stride, uint32_t n, uint32_t nEvents) {
  uint32_t e = blockIdx.y;
  if (e >= nEvents) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[e * stride + i] = 0;
}

// order each event's error list by word index (the serial push order)
__global__ void kSortErrors(Workspace ws) {
  uint32_t e = blockIdx.x;
  uint32_t n = min(ws.ev[e].nErrors, kErrCap);
  if (threadIdx.x == 0) {
    PfPixelError* er = ws.errors + size_t(e) * kErrCap;
    uint32_t* wi = ws.errWordIdx + size_t(e) * kErrCap;
    for (uint32_t i = 1; i < n; ++i) {
      PfPixelError x = er[i];
      uint32_t k = wi[i];
      int j = int(i) - 1;
      while (j >= 0 && wi[j] > k) {
        er[j + 1] = er[j];
        wi[j + 1] = wi[j];
        --j;
      }
      er[j + 1] = x;
      wi[j + 1] = k;
    }
    if (ws.ev[e].nErrors > kErrCap) ws.ev[e].nErrors = kErrCap;
  }
}

}  // namespace

// countModules, findClus and clusterChargeCut alone, on digis already in ws
// (xx, yy, calibrated adc, moduleInd, clus = index) with their word offsets
cudaError_t runClusters(Workspace& ws, uint32_t nEvents, cudaStream_t stream) {
  PG_PROBED("kInitEvents", stream, kInitEvents<<<nEvents, 256, 0, stream>>>(ws, nEvents));
  const int flatBlocks = 148 * 8;
  PG_PROBED("kModuleBoundaries", stream, kModuleBoundaries<<<tunedGrid(ws, kTuneModuleBoundaries, flatBlocks), 256, 0, stream>>>(ws, nEvents));
  PG_PROBED("kSortModules", stream, kSortModules<<<nEvents, 1024, 0, stream>>>(ws, nEvents));
  PG_PROBED("kFindClusters", stream,
            kFindClustersSmall<<<dim3((kMaxModules + kSmallWarps - 1) / kSmallWarps, nEvents), kSmallWarps * 32, 0,
                                 stream>>>(ws));
  PG_PROBED("kFindClustersBig", stream, kFindClustersBig<<<dim3(tunedGrid(ws, kTuneFindClustersBig, 64), nEvents), kClusThreads, 0, stream>>>(ws));
  return cudaGetLastError();
}

cudaError_t runLocal(const DeviceES& es, Workspace& ws, uint32_t nEvents, cudaStream_t stream) {
  PG_PROBED("kInitEvents", stream, kInitEvents<<<nEvents, 256, 0, stream>>>(ws, nEvents));
  const int flatBlocks = 148 * 8;
  PG_PROBED("kRawToDigi", stream, kRawToDigi<<<tunedGrid(ws, kTuneRawToDigi, flatBlocks), 256, 0, stream>>>(es, ws, nEvents));
  PG_PROBED("kModuleBoundaries", stream, kModuleBoundaries<<<tunedGrid(ws, kTuneModuleBoundaries, flatBlocks), 256, 0, stream>>>(ws, nEvents));
  PG_PROBED("kSortModules", stream, kSortModules<<<nEvents, 1024, 0, stream>>>(ws, nEvents));
  PG_PROBED("kSortErrors", stream, kSortErrors<<<nEvents, 32, 0, stream>>>(ws));
  PG_PROBED("kFindClusters", stream,
            kFindClustersSmall<<<dim3((kMaxModules + kSmallWarps - 1) / kSmallWarps, nEvents), kSmallWarps * 32, 0,
                                 stream>>>(ws));
  PG_PROBED("kFindClustersBig", stream, kFindClustersBig<<<dim3(tunedGrid(ws, kTuneFindClustersBig, 64), nEvents), kClusThreads, 0, stream>>>(ws));
  PG_PROBED("kHitsModuleStart", stream, kHitsModuleStart<<<nEvents, 1024, 0, stream>>>(es, ws));
  PG_PROBED("kGetHits", stream,
            kGetHitsSmall<<<dim3((kMaxModules + kHitWarps - 1) / kHitWarps, nEvents), kHitWarps * 32, 0, stream>>>(es,
                                                                                                               ws));
  PG_PROBED("kGetHitsBig", stream, kGetHitsBig<<<dim3(tunedGrid(ws, kTuneGetHitsBig, 64), nEvents), kHitThreads, 0, stream>>>(es, ws));
  // phi histogram: count, exclusive scan, unordered fill, per-bin ordering
  uint32_t* cursor = ws.jCount;  // scratch: the doublet counters are not in use yet
  PG_PROBED("kZeroU32", stream, kZeroU32<<<dim3(2, nEvents), 1024, 0, stream>>>(ws.phiOff, kPhiStride, kPhiStride, nEvents));
  PG_PROBED("kZeroU32", stream, kZeroU32<<<dim3(2, nEvents), 1024, 0, stream>>>(cursor, kPhiStride, kPhiStride, nEvents));
  PG_PROBED("kPhiCount", stream, kPhiCount<<<dim3(tunedGrid(ws, kTunePhiCount, 16), nEvents), 256, 0, stream>>>(ws));
  // in place exclusive scan of the 1280 counters; the total lands in the extra bin
  segScan(ws, kScanPhi, ws.phiOff, ws.phiOff, kPhiStride, nullptr, 0, kPhiTot - 1, nullptr, 0, nEvents, stream);
  PG_PROBED("kPhiFill", stream, kPhiFill<<<dim3(tunedGrid(ws, kTunePhiFill, 16), nEvents), 256, 0, stream>>>(ws, cursor));
  PG_PROBED("kPhiSort", stream, kPhiSort<<<dim3((kPhiTot - 1 + 7) / 8, nEvents), 256, 0, stream>>>(ws));
  PG_PROBED("kPhiRec", stream, kPhiRec<<<dim3(tunedGrid(ws, kTunePhiRec, 16), nEvents), 256, 0, stream>>>(ws));
  return cudaGetLastError();
}

}  // namespace pixgpu
