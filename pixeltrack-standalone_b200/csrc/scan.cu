// Batched segmented exclusive scan over per-event arrays with fixed stride
// and device-resident lengths (no host synchronisation), in two launches:
// each event's array is cut into S slices of whole tiles; the first kernel
// sums every slice, the second rescans every slice (from L2) starting at the
// sum of the slices before it, which each CTA adds up itself.  S grows as the
// batch shrinks, so that a small batch still spreads over the SMs.
// out[i] = in[0] + ... + in[i-1] for i <= n (out[n] the total).  The
// reference's counterpart is the prefix scan of its OneToManyAssoc fills
// (HistoContainer.h / prefixScan.h, one event at a time).
#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

constexpr uint32_t kScanThreads = 512;
constexpr uint32_t kScanPer = 8;                           // elements per thread in a tile
constexpr uint32_t kScanTile = kScanThreads * kScanPer;  // 4096
// A warp owns 32 * kScanPer consecutive elements of a tile; lane l holds
// element j * 32 + l of that run in v[j] (coalesced loads and stores).

struct Slice {
  uint32_t n, lo, hi;
};

__device__ __forceinline__ Slice sliceOf(const uint32_t* lenPtr, uint32_t lenStride, uint32_t fixedLen, uint32_t e,
                                         uint32_t r, uint32_t S) {
  Slice s;
  s.n = lenPtr ? min(lenPtr[size_t(e) * lenStride], fixedLen) : fixedLen;  // fixedLen: the capacity
  const uint32_t tiles = (s.n + kScanTile - 1) / kScanTile;
  s.lo = min(s.n, tiles * r / S * kScanTile);
  s.hi = min(s.n, tiles * (r + 1) / S * kScanTile);
  return s;
}

__global__ void __launch_bounds__(kScanThreads)
    kScanSums(const uint32_t* in, uint32_t stride, const uint32_t* lenPtr, uint32_t lenStride, uint32_t fixedLen,
              uint32_t* sums) {
  __shared__ uint32_t sh[33];
  const uint32_t e = blockIdx.y, r = blockIdx.x, S = gridDim.x;
  const Slice sl = sliceOf(lenPtr, lenStride, fixedLen, e, r, S);
  const uint32_t* src = in + size_t(e) * stride;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t s = 0;
  for (uint32_t b = sl.lo; b < sl.hi; b += kScanTile) {
    const uint32_t w0 = b + warp * 32 * kScanPer + lane;
#pragma unroll
    for (uint32_t j = 0; j < kScanPer; ++j) {
      const uint32_t i = w0 + j * 32;
      s += i < sl.hi ? src[i] : 0u;
    }
  }
  uint32_t tot;
  blockExclusiveScan(s, sh, &tot);
  if (threadIdx.x == 0) sums[size_t(e) * kScanMaxSlices + r] = tot;
}

__global__ void __launch_bounds__(kScanThreads, 3)
    kScanSlices(uint32_t* in, uint32_t* out, uint32_t stride, const uint32_t* lenPtr, uint32_t lenStride,
                uint32_t fixedLen, const uint32_t* sums, uint32_t* totalPtr, uint32_t totalStride, bool zeroIn) {
  __shared__ uint32_t sh[33];
  __shared__ uint32_t sOff;
  const uint32_t e = blockIdx.y, r = blockIdx.x, S = gridDim.x;
  const Slice sl = sliceOf(lenPtr, lenStride, fixedLen, e, r, S);
  uint32_t* src = in + size_t(e) * stride;
  uint32_t* dst = out + size_t(e) * stride;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp == 0) {
    uint32_t o = 0;
    for (uint32_t k = lane; k < r; k += 32) o += sums[size_t(e) * kScanMaxSlices + k];
    o = __reduce_add_sync(0xffffffffu, o);
    if (lane == 0) sOff = o;
  }
  __syncthreads();
  uint32_t carry = sOff;
  for (uint32_t b = sl.lo; b < sl.hi; b += kScanTile) {
    const uint32_t w0 = b + warp * 32 * kScanPer + lane;
    uint32_t v[kScanPer];
    uint32_t run = 0;  // exclusive prefix of the warp's run so far
#pragma unroll
    for (uint32_t j = 0; j < kScanPer; ++j) {
      const uint32_t i = w0 + j * 32;
      const uint32_t x = i < sl.hi ? src[i] : 0u;
      const uint32_t inc = warpInclusiveScan(x);
      v[j] = run + inc - x;
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    uint32_t tileTot;
    const uint32_t wpre = blockExclusiveScan(lane == 31 ? run : 0u, sh, &tileTot);
    const uint32_t base = carry + __shfl_sync(0xffffffffu, wpre, 31);
#pragma unroll
    for (uint32_t j = 0; j < kScanPer; ++j) {
      const uint32_t i = w0 + j * 32;
      if (i < sl.hi) {
        if (zeroIn) src[i] = 0u;
        dst[i] = base + v[j];
      }
    }
    carry += tileTot;
  }
  if (r == S - 1 && threadIdx.x == 0) {
    dst[sl.n] = carry;
    if (totalPtr) totalPtr[size_t(e) * totalStride] = carry;
  }
}

}  // namespace

void segScan(uint32_t* in, uint32_t* out, uint32_t stride, const uint32_t* lenPtr, uint32_t lenStride,
             uint32_t maxLen, uint32_t* totalPtr, uint32_t totalStride, uint32_t* sums, uint32_t nEvents,
             cudaStream_t stream, bool zeroIn) {
  // slices per event: enough CTAs for a few waves, no slice shorter than a tile
  const uint32_t tiles = (maxLen + kScanTile - 1) / kScanTile;
  uint32_t S = min(kScanMaxSlices, max(16u, 1024u / max(nEvents, 1u)));
  S = max(1u, min(S, tiles));
  const dim3 g(S, nEvents);
  PG_PROBED("kScanSums", stream,
            kScanSums<<<g, kScanThreads, 0, stream>>>(in, stride, lenPtr, lenStride, maxLen, sums));
  PG_PROBED("kScanSlices", stream,
            kScanSlices<<<g, kScanThreads, 0, stream>>>(in, out, stride, lenPtr, lenStride, maxLen, sums, totalPtr,
                                                        totalStride, zeroIn));
}

}  // namespace pixgpu
