// Batched segmented exclusive scan over per-event arrays with fixed stride
// and device-resident lengths (no host synchronisation), in one pass with
// decoupled look-back: the CTAs of an event take the tiles of its array in
// ticket order; a tile publishes its sum at once, then adds up the sums of
// the tiles before it (32 at a time, stopping at the first tile that has
// published its full prefix), publishes its own prefix and writes its
// outputs.  Each element is read once and written once.
// out[i] = in[0] + ... + in[i-1] for i <= n (out[n] the total).  The
// reference's counterpart is the prefix scan of its OneToManyAssoc fills
// (HistoContainer.h / prefixScan.h, one event at a time).
//
// A tile waits only on tiles with smaller tickets, which were taken by CTAs
// already running, so every wait ends; the wait is bounded all the same and
// sets kFlagScanStall if the bound is reached.
#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

constexpr uint32_t kScanThreads = 512;
constexpr uint32_t kScanPer = kScanTile / kScanThreads;  // 8 elements per thread in a tile
// A warp owns 32 * kScanPer consecutive elements of a tile; lane l holds
// element j * 32 + l of that run in v[j] (coalesced loads and stores).

// state word of a tile: tag (30 bits) | status (2 bits) | value (32 bits).
// The tag names the batch and the scan, so words left by earlier batches
// read as "not yet published".
constexpr uint64_t kStatusSum = 1, kStatusPrefix = 2;
__device__ __forceinline__ uint64_t stateWord(uint32_t tag, uint64_t status, uint32_t v) {
  return (uint64_t(tag) << 34) | (status << 32) | v;
}
__device__ __forceinline__ void publish(uint64_t* p, uint64_t w) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ uint64_t peek(const uint64_t* p) {
  uint64_t w;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
  return w;
}

constexpr uint32_t kLookBackPolls = 1u << 22;  // bound on the polls of one look-back (~0.3 s)

// one of the arrays a launch scans (two arrays of the same lengths may share
// a launch, each with its own tile states; the first one's ticket orders
// the tiles)
struct ScanArray {
  uint32_t* in;
  uint32_t* out;
  uint32_t* total;  // per-event total (may be null)
  uint32_t call;    // ScanCall: state region
};

template <uint32_t kArrays>
__global__ void __launch_bounds__(kScanThreads, 3)
    kScanOnePass(ScanArray a0, ScanArray a1, uint32_t stride, const uint32_t* lenPtr, uint32_t lenStride,
                 uint32_t fixedLen, uint32_t totalStride, bool zeroIn, Workspace ws) {
  __shared__ uint32_t sh[kArrays][33];
  __shared__ uint32_t sTile, sPrefix[kArrays];
  const uint32_t e = blockIdx.y;
  const uint32_t n = lenPtr ? min(lenPtr[size_t(e) * lenStride], fixedLen) : fixedLen;  // fixedLen: the capacity
  const uint32_t tiles = max(1u, (n + kScanTile - 1) / kScanTile);
  auto arr = [&](uint32_t q) -> const ScanArray& { return q == 0 ? a0 : a1; };
  uint32_t* ticket = ws.scanTicket + size_t(e) * kScanCalls + a0.call;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) sTile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t t = sTile;
    if (t >= tiles) return;
    const uint32_t lo = t * kScanTile, hi = min(n, lo + kScanTile);
    const uint32_t w0 = lo + warp * 32 * kScanPer + lane;
    uint32_t v[kArrays][kScanPer];
    uint32_t base[kArrays], tileTot[kArrays];
#pragma unroll
    for (uint32_t q = 0; q < kArrays; ++q) {
      const uint32_t* src = arr(q).in + size_t(e) * stride;
#pragma unroll
      for (uint32_t j = 0; j < kScanPer; ++j) {
        const uint32_t i = w0 + j * 32;
        v[q][j] = i < hi ? src[i] : 0u;
      }
    }
#pragma unroll
    for (uint32_t q = 0; q < kArrays; ++q) {
      uint32_t run = 0;  // exclusive prefix of the warp's run so far
#pragma unroll
      for (uint32_t j = 0; j < kScanPer; ++j) {
        const uint32_t x = v[q][j];
        const uint32_t inc = warpInclusiveScan(x);
        v[q][j] = run + inc - x;
        run += __shfl_sync(0xffffffffu, inc, 31);
      }
      const uint32_t wpre = blockExclusiveScan(lane == 31 ? run : 0u, sh[q], &tileTot[q]);
      base[q] = __shfl_sync(0xffffffffu, wpre, 31);
    }
    // publish each array's tile sum, then look back (warp q for array q)
    if (warp < kArrays) {
      const uint32_t q = warp;
      const uint32_t tot = q == 0 ? tileTot[0] : tileTot[kArrays - 1];
      uint64_t* state = ws.scanState + (size_t(e) * kScanCalls + arr(q).call) * ws.scanTiles;
      const uint32_t tag = (ws.scanEpoch[e] * kScanCalls + arr(q).call) & 0x3fffffffu;
      uint32_t prefix = 0;
      if (t == 0) {
        if (lane == 0) publish(state, stateWord(tag, kStatusPrefix, tot));
      } else {
        if (lane == 0) publish(state + t, stateWord(tag, kStatusSum, tot));
        int32_t k = int32_t(t) - 1;  // the window covers tiles k - 31 .. k
        uint32_t polls = 0;
        bool stalled = false;
        while (k >= 0) {
          const int32_t idx = k - int32_t(lane);
          uint64_t w = idx >= 0 ? peek(state + idx) : stateWord(tag, kStatusPrefix, 0u);
          const bool ready = uint32_t(w >> 34) == tag && ((w >> 32) & 3u) != 0;
          if (__all_sync(0xffffffffu, ready)) {
            // the nearest tile with its full prefix ends the walk
            const uint32_t pm = __ballot_sync(0xffffffffu, ((w >> 32) & 3u) == kStatusPrefix);
            const uint32_t stop = pm ? uint32_t(__ffs(pm) - 1) : 32u;
            const uint32_t val = lane <= stop ? uint32_t(w) : 0u;
            prefix += __reduce_add_sync(0xffffffffu, val);
            if (pm) break;
            k -= 32;
          } else if (++polls > kLookBackPolls) {
            stalled = true;
            break;
          } else {
            __nanosleep(64);
          }
        }
        if (lane == 0) {
          if (stalled) atomicOr(&ws.ev[e].flags, kFlagScanStall);
          publish(state + t, stateWord(tag, kStatusPrefix, prefix + tot));
        }
      }
      if (lane == 0) sPrefix[q] = prefix;
    }
    __syncthreads();
#pragma unroll
    for (uint32_t q = 0; q < kArrays; ++q) {
      uint32_t* src = arr(q).in + size_t(e) * stride;
      uint32_t* dst = arr(q).out + size_t(e) * stride;
      const uint32_t carry = sPrefix[q] + base[q];
#pragma unroll
      for (uint32_t j = 0; j < kScanPer; ++j) {
        const uint32_t i = w0 + j * 32;
        if (i < hi) {
          if (zeroIn) src[i] = 0u;
          dst[i] = carry + v[q][j];
        }
      }
      if (t == tiles - 1 && threadIdx.x == 0) {
        dst[n] = sPrefix[q] + tileTot[q];
        if (arr(q).total) arr(q).total[size_t(e) * totalStride] = sPrefix[q] + tileTot[q];
      }
    }
    __syncthreads();  // sTile and sPrefix are rewritten by the next tile
  }
}

// CTAs per event: every tile of the longest array at once for small
// batches; a CTA takes further tiles while there are any
dim3 scanGrid(uint32_t maxLen, uint32_t nEvents) {
  const uint32_t tiles = max(1u, (maxLen + kScanTile - 1) / kScanTile);
  const uint32_t S = max(1u, min(tiles, max(8u, 1024u / max(nEvents, 1u))));
  return dim3(S, nEvents);
}

}  // namespace

void segScan(const Workspace& ws, ScanCall call, uint32_t* in, uint32_t* out, uint32_t stride,
             const uint32_t* lenPtr, uint32_t lenStride, uint32_t maxLen, uint32_t* totalPtr, uint32_t totalStride,
             uint32_t nEvents, cudaStream_t stream, bool zeroIn) {
  const ScanArray a{in, out, totalPtr, uint32_t(call)};
  PG_PROBED("kScanOnePass", stream,
            kScanOnePass<1><<<scanGrid(maxLen, nEvents), kScanThreads, 0, stream>>>(
                a, a, stride, lenPtr, lenStride, maxLen, totalStride, zeroIn, ws));
}

void segScan2(const Workspace& ws, ScanCall call0, uint32_t* in0, uint32_t* out0, uint32_t* total0, ScanCall call1,
              uint32_t* in1, uint32_t* out1, uint32_t* total1, uint32_t stride, const uint32_t* lenPtr,
              uint32_t lenStride, uint32_t maxLen, uint32_t totalStride, uint32_t nEvents, cudaStream_t stream,
              bool zeroIn) {
  const ScanArray a0{in0, out0, total0, uint32_t(call0)}, a1{in1, out1, total1, uint32_t(call1)};
  PG_PROBED("kScanOnePass", stream,
            kScanOnePass<2><<<scanGrid(maxLen, nEvents), kScanThreads, 0, stream>>>(
                a0, a1, stride, lenPtr, lenStride, maxLen, totalStride, zeroIn, ws));
}

}  // namespace pixgpu
