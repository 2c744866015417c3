// Batched segmented exclusive scan over per-event arrays with fixed stride
// and device-resident lengths (no host synchronisation): chunk scans, a scan
// of the chunk totals per event, then the chunk offsets are added.
#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

constexpr uint32_t kThreads = 1024;
constexpr uint32_t kPerThread = kScanChunk / kThreads;  // 4

__global__ void scanChunks(const uint32_t* in, uint32_t* out, uint32_t stride, const uint32_t* lenPtr,
                           uint32_t lenStride, uint32_t fixedLen, uint32_t* tmp) {
  __shared__ uint32_t sh[33];
  uint32_t e = blockIdx.y;
  uint32_t n = lenPtr ? lenPtr[size_t(e) * lenStride] : fixedLen;
  uint32_t base = blockIdx.x * kScanChunk;
  if (base >= n + 1) return;  // nothing (the total slot at index n belongs to some chunk)
  const uint32_t* src = in + size_t(e) * stride;
  uint32_t* dst = out + size_t(e) * stride;
  uint32_t v[kPerThread];
  uint32_t s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kPerThread; ++k) {
    uint32_t i = base + threadIdx.x * kPerThread + k;
    v[k] = i < n ? src[i] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t pre = blockExclusiveScan(s, sh, &total);
#pragma unroll
  for (uint32_t k = 0; k < kPerThread; ++k) {
    uint32_t i = base + threadIdx.x * kPerThread + k;
    if (i <= n) dst[i] = pre;
    pre += v[k];
  }
  if (threadIdx.x == 0) tmp[size_t(e) * kScanTmpStride + blockIdx.x] = total;
}

__global__ void scanTotals(uint32_t* tmp, const uint32_t* lenPtr, uint32_t lenStride, uint32_t fixedLen,
                           uint32_t* totalPtr, uint32_t totalStride) {
  __shared__ uint32_t sh[33];
  uint32_t e = blockIdx.x;
  uint32_t n = lenPtr ? lenPtr[size_t(e) * lenStride] : fixedLen;
  uint32_t nChunks = (n + 1 + kScanChunk - 1) / kScanChunk;
  uint32_t* t = tmp + size_t(e) * kScanTmpStride;
  uint32_t carry = 0;
  for (uint32_t c0 = 0; c0 < nChunks; c0 += blockDim.x) {
    uint32_t c = c0 + threadIdx.x;
    uint32_t v = c < nChunks ? t[c] : 0u;
    uint32_t total;
    uint32_t pre = blockExclusiveScan(v, sh, &total);
    if (c < nChunks) t[c] = carry + pre;
    carry += total;
  }
  if (threadIdx.x == 0) {
    if (totalPtr) totalPtr[size_t(e) * totalStride] = carry;
  }
}

__global__ void scanAdd(uint32_t* out, uint32_t stride, const uint32_t* lenPtr, uint32_t lenStride,
                        uint32_t fixedLen, const uint32_t* tmp) {
  uint32_t e = blockIdx.y;
  uint32_t n = lenPtr ? lenPtr[size_t(e) * lenStride] : fixedLen;
  uint32_t base = blockIdx.x * kScanChunk;
  if (base >= n + 1 || blockIdx.x == 0) return;
  uint32_t add = tmp[size_t(e) * kScanTmpStride + blockIdx.x];
  uint32_t* dst = out + size_t(e) * stride;
  for (uint32_t k = threadIdx.x; k < kScanChunk; k += blockDim.x) {
    uint32_t i = base + k;
    if (i <= n) dst[i] += add;
  }
}

}  // namespace

void segScan(const uint32_t* in, uint32_t* out, uint32_t stride, const uint32_t* lenPtr, uint32_t lenStride,
             uint32_t maxLen, uint32_t* totalPtr, uint32_t totalStride, uint32_t* tmp, uint32_t nEvents,
             cudaStream_t stream) {
  uint32_t nChunks = (maxLen + 1 + kScanChunk - 1) / kScanChunk;
  dim3 g(nChunks, nEvents);
  PG_PROBED("scanChunks", stream, scanChunks<<<g, kThreads, 0, stream>>>(in, out, stride, lenPtr, lenStride, maxLen, tmp));
  PG_PROBED("scanTotals", stream, scanTotals<<<nEvents, 1024, 0, stream>>>(tmp, lenPtr, lenStride, maxLen, totalPtr, totalStride));
  PG_PROBED("scanAdd", stream, scanAdd<<<g, 256, 0, stream>>>(out, stride, lenPtr, lenStride, maxLen, tmp));
}

}  // namespace pixgpu
