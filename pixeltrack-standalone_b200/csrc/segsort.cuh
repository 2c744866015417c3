// Ordering of many small CSR segments in place (cells by outer hit, CA
// links, tracks per cell, tuples per hit).  The lists are filled by atomics
// in arbitrary order; the serial reference fills them in ascending producer
// order, which is the order restored here (keys inside one segment are
// distinct).
//
//  kSortListed one thread per segment the fill noted (the segments that got
//              a second entry): n <= 32 sorted in registers by a bitonic
//              network; 32 < n <= 256 handed to the warp (rank sort, one
//              segment at a time, ballot over the lanes that hold one);
//              n > 256 appended to a per-event list for kSortBig.
//  kSortBig    one block per long segment: rank sort in shared memory.
#pragma once

#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

constexpr uint32_t kBigSort = 4096;  // longest segment ordered in shared memory

// bitonic network over N registers (N a power of two, n <= N elements)
template <uint32_t N, typename T>
__device__ __forceinline__ void sortRegs(T* seg, uint32_t n, bool desc) {
  T v[N];
  const T pad = desc ? T(0) : T(~T(0));
#pragma unroll
  for (uint32_t i = 0; i < N; ++i) v[i] = i < n ? seg[i] : pad;
#pragma unroll
  for (uint32_t k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (uint32_t i = 0; i < N; ++i) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const T a = v[i], b = v[l];
          const bool sw = up ? (a > b) : (a < b);
          v[i] = sw ? b : a;
          v[l] = sw ? a : b;
        }
      }
    }
  }
  // ascending with the pads last; descending reads it backwards (pads are 0)
#pragma unroll
  for (uint32_t i = 0; i < N; ++i)
    if (i < n) seg[i] = desc ? v[N - 1 - i] : v[i];
}

template <typename T>
__device__ void serialSort(T* seg, uint32_t n, bool desc) {
  for (uint32_t i = 1; i < n; ++i) {
    T x = seg[i];
    int j = int(i) - 1;
    while (j >= 0 && (desc ? seg[j] < x : seg[j] > x)) {
      seg[j + 1] = seg[j];
      --j;
    }
    seg[j + 1] = x;
  }
}

template <typename T>
__global__ void kSortListed(T* data, size_t dataStride, const uint32_t* off, size_t offStride, const uint32_t* list,
                            size_t listStride, const uint32_t* nList, uint32_t nListStride, bool desc,
                            uint32_t dataCap, uint32_t* big, uint32_t* nBig, uint32_t nBigStride) {
  const uint32_t e = blockIdx.y;
  const uint32_t nseg = nList[size_t(e) * nListStride];
  const uint32_t* o = off + size_t(e) * offStride;
  const uint32_t* L = list + size_t(e) * listStride;
  T* d = data + size_t(e) * dataStride;
  for (uint32_t s0 = blockIdx.x * blockDim.x; s0 < nseg; s0 += gridDim.x * blockDim.x) {
    const uint32_t k = s0 + threadIdx.x;
    uint32_t b = 0, n = 0, s = 0;
    if (k < nseg) {
      s = L[k];
      b = min(o[s], dataCap);
      n = min(o[s + 1], dataCap) - b;
    }
    if (n >= 2 && n <= 16)
      sortRegs<16>(d + b, n, desc);
    else if (n > 16 && n <= 32)
      sortRegs<32>(d + b, n, desc);
    uint32_t m = __ballot_sync(0xffffffffu, n > 32 && n <= 256);
    while (m) {
      const int l = __ffs(m) - 1;
      m &= m - 1;
      const uint32_t bb = __shfl_sync(0xffffffffu, b, l), nn = __shfl_sync(0xffffffffu, n, l);
      warpSortSegment(d + bb, nn, desc);
    }
    if (n > 256) {
      const uint32_t q = atomicAdd(&nBig[size_t(e) * nBigStride], 1u);
      if (q < kBigSegCap)
        big[size_t(e) * kBigSegCap + q] = s;
      else
        serialSort(d + b, n, desc);  // more long segments than the list holds
    }
  }
}

template <typename T>
__global__ void kSortBig(T* data, size_t dataStride, const uint32_t* off, size_t offStride, bool desc,
                         uint32_t dataCap, const uint32_t* big, const uint32_t* nBig, uint32_t nBigStride) {
  __shared__ T sh[kBigSort];
  const uint32_t e = blockIdx.y;
  const uint32_t nb = min(nBig[size_t(e) * nBigStride], kBigSegCap);
  const uint32_t* o = off + size_t(e) * offStride;
  T* d = data + size_t(e) * dataStride;
  for (uint32_t k = blockIdx.x; k < nb; k += gridDim.x) {
    const uint32_t s = big[size_t(e) * kBigSegCap + k];
    const uint32_t b = min(o[s], dataCap), n = min(o[s + 1], dataCap) - b;
    if (n <= kBigSort) {
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sh[i] = d[b + i];
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const T v = sh[i];
        uint32_t r = 0;
        for (uint32_t j = 0; j < n; ++j) r += desc ? (sh[j] > v) : (sh[j] < v);
        d[b + r] = v;
      }
    } else if (threadIdx.x == 0) {
      serialSort(d + b, n, desc);
    }
    __syncthreads();
  }
}

// Orders segment s = [off[s], off[s+1]) of data for every segment the
// preceding fill noted in list `slot` (those with >= 2 entries); `slot` also
// picks the per-event long-segment counter.  lenPtr/fixedLen (the number of
// segments) are kept for the callers' readability only.
template <typename T>
void sortSegments(Workspace& ws, uint32_t nEvents, cudaStream_t stream, uint32_t gx, T* data, size_t dataStride,
                  const uint32_t* off, size_t offStride, const uint32_t* lenPtr, uint32_t lenStride, uint32_t fixedLen,
                  bool desc, uint32_t dataCap, int slot) {
  uint32_t* nBig = &ws.ev[0].nBig[slot];
  const uint32_t stride = sizeof(EventCounters) / 4;
  (void)lenPtr;
  (void)lenStride;
  (void)fixedLen;
  PG_PROBED("kSortSegments", stream,
            kSortListed<T><<<dim3(gx, nEvents), 256, 0, stream>>>(data, dataStride, off, offStride, ws.segList,
                                                                  ws.cap.cells, &ws.ev[0].nSegList[slot], stride,
                                                                  desc, dataCap, ws.bigSeg, nBig, stride));
  PG_PROBED("kSortBig", stream,
            kSortBig<T><<<dim3(8, nEvents), 256, 0, stream>>>(data, dataStride, off, offStride, desc, dataCap,
                                                              ws.bigSeg, nBig, stride));
}

}  // namespace pixgpu
