// Small device primitives: warp/block scans and per-segment ordering.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pixgpu {

__device__ __forceinline__ uint32_t laneId() { return threadIdx.x & 31; }
__device__ __forceinline__ uint32_t lanemaskLt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// inclusive warp scan
__device__ __forceinline__ uint32_t warpInclusiveScan(uint32_t v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (laneId() >= uint32_t(o)) v += t;
  }
  return v;
}

// Exclusive block scan of one value per thread; blockDim.x multiple of 32,
// <= 1024.  `sh` holds >= 33 uint32_t.  Returns the exclusive prefix and the
// block total in *total.  Contains __syncthreads.
__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* sh, uint32_t* total) {
  uint32_t w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t inc = warpInclusiveScan(v);
  if (laneId() == 31) sh[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t x = laneId() < nw ? sh[laneId()] : 0;
    uint32_t xi = warpInclusiveScan(x);
    if (laneId() < nw) sh[laneId()] = xi - x;
    if (laneId() == nw - 1) sh[32] = xi;
  }
  __syncthreads();
  uint32_t r = sh[w] + inc - v;
  *total = sh[32];
  __syncthreads();
  return r;
}

// The same for 64-bit values (several packed counters scanned at once);
// `sh` holds >= 33 uint64_t.
__device__ __forceinline__ uint64_t blockExclusiveScan64(uint64_t v, uint64_t* sh, uint64_t* total) {
  uint32_t w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint64_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (laneId() >= uint32_t(o)) inc += t;
  }
  if (laneId() == 31) sh[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint64_t x = laneId() < nw ? sh[laneId()] : 0;
    uint64_t xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t t = __shfl_up_sync(0xffffffffu, xi, o);
      if (laneId() >= uint32_t(o)) xi += t;
    }
    if (laneId() < nw) sh[laneId()] = xi - x;
    if (laneId() == nw - 1) sh[32] = xi;
  }
  __syncthreads();
  uint64_t r = sh[w] + inc - v;
  *total = sh[32];
  __syncthreads();
  return r;
}

// Orders the n elements of seg[] in place (ascending, or descending if desc),
// using one warp: rank of each element = number of smaller elements.  Keys
// are distinct.  For n <= 32*kPer only; larger segments fall back to a
// warp-serial insertion sort.
template <typename T>
__device__ void warpSortSegment(T* seg, uint32_t n, bool desc) {
  if (n < 2) return;
  constexpr uint32_t kPer = 8;
  if (n <= 32 * kPer) {
    T v[kPer];
    uint32_t r[kPer];
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
      uint32_t i = laneId() + 32 * k;
      v[k] = i < n ? seg[i] : T(0);
      r[k] = 0;
    }
    for (uint32_t j = 0; j < n; ++j) {
      T x = seg[j];
#pragma unroll
      for (uint32_t k = 0; k < kPer; ++k) r[k] += desc ? (x > v[k]) : (x < v[k]);
    }
    __syncwarp();
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
      uint32_t i = laneId() + 32 * k;
      if (i < n) seg[r[k]] = v[k];
    }
    __syncwarp();
  } else {
    if (laneId() == 0) {
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
    __syncwarp();
  }
}

// index of the last offset <= x among off[0..n] (n+1 entries, ascending)
__device__ __forceinline__ uint32_t upperBoundIdx(const uint32_t* off, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;  // find largest e in [0, n) with off[e] <= x
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= x)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

}  // namespace pixgpu
