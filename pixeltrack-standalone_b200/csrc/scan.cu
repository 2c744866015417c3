// Batched segmented exclusive scan over per-event arrays with fixed stride
// and device-resident lengths (no host synchronisation), in one launch: one
// thread-block cluster of kScanCtas CTAs per event.  Each CTA sums one slice
// of the event's array; the slice totals are exchanged through distributed
// shared memory; each CTA then rescans its slice (from L2) with its offset.
// out[i] = in[0] + ... + in[i-1] for i <= n (out[n] the total).  The
// reference's counterpart is the prefix scan of its OneToManyAssoc fills
// (HistoContainer.h / prefixScan.h, one event at a time).
#include <cooperative_groups.h>

#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

constexpr uint32_t kScanCtas = 8;
constexpr uint32_t kScanThreads = 1024;
constexpr uint32_t kScanPer = 8;                           // elements per thread in a tile
constexpr uint32_t kScanTile = kScanThreads * kScanPer;  // 8192
// A warp owns 32 * kScanPer consecutive elements of a tile; lane l holds
// element j * 32 + l of that run in v[j] (coalesced loads and stores).

__global__ void __cluster_dims__(kScanCtas, 1, 1) __launch_bounds__(kScanThreads)
    kSegScan(uint32_t* in, uint32_t* out, uint32_t stride, const uint32_t* lenPtr, uint32_t lenStride,
             uint32_t fixedLen, uint32_t* totalPtr, uint32_t totalStride, bool zeroIn) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t r = cl.block_rank();
  __shared__ uint32_t sh[33];
  __shared__ uint32_t sSum;
  __shared__ uint32_t sOff;
  const uint32_t e = blockIdx.y;
  const uint32_t n = lenPtr ? min(lenPtr[size_t(e) * lenStride], fixedLen) : fixedLen;  // fixedLen: the capacity
  uint32_t* src = in + size_t(e) * stride;
  uint32_t* dst = out + size_t(e) * stride;
  // whole tiles per CTA
  const uint32_t tiles = (n + kScanTile - 1) / kScanTile;
  const uint32_t lo = min(n, tiles * r / kScanCtas * kScanTile);
  const uint32_t hi = min(n, tiles * (r + 1) / kScanCtas * kScanTile);
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // ---- slice total
  uint32_t s = 0;
  for (uint32_t b = lo; b < hi; b += kScanTile) {
    const uint32_t w0 = b + warp * 32 * kScanPer + lane;
#pragma unroll
    for (uint32_t j = 0; j < kScanPer; ++j) {
      const uint32_t i = w0 + j * 32;
      s += i < hi ? src[i] : 0u;
    }
  }
  uint32_t tot;
  blockExclusiveScan(s, sh, &tot);
  if (threadIdx.x == 0) sSum = tot;
  cl.sync();
  if (threadIdx.x == 0) {
    uint32_t o = 0;
    for (uint32_t k = 0; k < r; ++k) o += *cl.map_shared_rank(&sSum, k);
    sOff = o;
  }
  // every CTA has read what it needs from the others' shared memory
  cl.sync();
  // ---- rescan of the slice with its offset
  uint32_t carry = sOff;
  for (uint32_t b = lo; b < hi; b += kScanTile) {
    const uint32_t w0 = b + warp * 32 * kScanPer + lane;
    uint32_t v[kScanPer];
    uint32_t run = 0;  // exclusive prefix of the warp's run so far
#pragma unroll
    for (uint32_t j = 0; j < kScanPer; ++j) {
      const uint32_t i = w0 + j * 32;
      const uint32_t x = i < hi ? src[i] : 0u;
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
      if (i < hi) {
        if (zeroIn) src[i] = 0u;
        dst[i] = base + v[j];
      }
    }
    carry += tileTot;
  }
  if (r == kScanCtas - 1 && threadIdx.x == 0) {
    dst[n] = carry;
    if (totalPtr) totalPtr[size_t(e) * totalStride] = carry;
  }
}

}  // namespace

void segScan(uint32_t* in, uint32_t* out, uint32_t stride, const uint32_t* lenPtr, uint32_t lenStride,
             uint32_t maxLen, uint32_t* totalPtr, uint32_t totalStride, uint32_t nEvents, cudaStream_t stream,
             bool zeroIn) {
  PG_PROBED("kSegScan", stream,
            kSegScan<<<dim3(kScanCtas, nEvents), kScanThreads, 0, stream>>>(in, out, stride, lenPtr, lenStride, maxLen,
                                                                          totalPtr, totalStride, zeroIn));
}

}  // namespace pixgpu
