// Result packing and small batch-setup kernels.
//
// kPackResults writes, per event, the compact result that a consumer of the
// chain needs (the role of the PixelTrackSoAFromCUDA / PixelVertexSoAFromCUDA
// transfer modules of the CUDA program): counts, the loose tracks (quality >=
// loose, in tuple order) with their fit state, covariance, hits and vertex
// assignment, and the vertices.  The destination is mapped pinned host memory,
// so the transfer is exact-sized and needs no host synchronisation.
#include <atomic>

#include <cooperative_groups.h>

#include "device_utils.cuh"
#include "pixgpu_internal.cuh"
#include "pixgpu_results.h"

namespace pixgpu {

namespace {

__global__ void kSetInput(BatchInput* in, const uint32_t* words, const uint8_t* fedIds) {
  in->words = words;
  in->fedIds = fedIds;
}

// 32-bit word w of a byte (or 16-bit) array assembled from its elements
template <typename F>
__device__ __forceinline__ uint32_t packBytes(uint32_t w, uint32_t n, F&& get) {
  uint32_t x = 0;
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k) {
    const uint32_t i = 4 * w + k;
    x |= (i < n ? uint32_t(get(i)) & 0xffu : 0u) << (8 * k);
  }
  return x;
}
template <typename F>
__device__ __forceinline__ uint32_t packHalves(uint32_t w, uint32_t n, F&& get) {
  const uint32_t i = 2 * w;
  const uint32_t lo = i < n ? uint32_t(get(i)) & 0xffffu : 0u;
  const uint32_t hi = i + 1 < n ? uint32_t(get(i + 1)) & 0xffffu : 0u;
  return lo | (hi << 16);
}

// One thread-block cluster of P CTAs per event (P = 1 for large batches, where
// the bus, not the SMs, bounds the copy).  Each CTA compacts
// the loose tuples of one slice of the tuple range; the slices' counts give
// the offsets (read across the cluster from distributed shared memory), and
// every CTA gathers the whole list into its own shared memory.  Each CTA then
// writes one slice of every output array.  The destination is host memory
// reached over the bus: every array is written as consecutive 32-bit words
// by consecutive threads (whole lines per warp), from all the cluster's SMs
// at once; the gathers come from device memory.
constexpr uint32_t kPackCtas = 8;  // CTAs per event in a small batch

// dynamic shared memory: the slice's loose tuple indices and the whole list
constexpr size_t kPackSmemBytes = 2 * size_t(kResultTracks) * sizeof(uint32_t);

__global__ void __launch_bounds__(512) kPackResults(Workspace ws, uint8_t* out) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t r = cl.block_rank(), P = cl.num_blocks();
  extern __shared__ __align__(16) uint32_t packSm[];
  uint32_t* sLocal = packSm;
  uint32_t* sIdx = packSm + kResultTracks;
  __shared__ uint32_t scanSh[33];
  __shared__ uint32_t sCount;
  __shared__ uint32_t sOff[kPackCtas + 1];  // P <= kPackCtas
  const uint32_t e = blockIdx.y;
  const EventCounters* c = ws.ev + e;
  uint8_t* base = out + size_t(e) * kResultStride;
  const uint32_t bins = ws.cap.tuples;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (bins + 1);
  const uint32_t* th = ws.tupleHits + size_t(e) * ws.cap.tupleHits();
  const uint8_t* q = ws.quality + size_t(e) * bins;
  const size_t tb = size_t(e) * bins;
  const uint32_t guard = c->apcM >= bins ? bins - 1 : c->nTuples;
  // ---- this CTA's slice of the tuples: loose ones in tuple order
  const uint32_t chunk = (guard + P - 1) / P;
  const uint32_t lo = min(guard, r * chunk), hi = min(guard, lo + chunk);
  uint32_t carry = 0;
  for (uint32_t t0 = lo; t0 < hi; t0 += blockDim.x) {
    const uint32_t t = t0 + threadIdx.x;
    const uint32_t loose = (t < hi && q[t] >= 2) ? 1u : 0u;
    uint32_t tot;
    const uint32_t p = carry + blockExclusiveScan(loose, scanSh, &tot);
    if (loose && p < kResultTracks) sLocal[p] = t;
    carry += tot;
  }
  if (threadIdx.x == 0) sCount = carry;
  cl.sync();
  if (threadIdx.x == 0) {
    uint32_t o = 0;
    for (uint32_t k = 0; k < P; ++k) {
      sOff[k] = o;
      o += *cl.map_shared_rank(&sCount, k);
    }
    sOff[P] = o;
  }
  __syncthreads();
  const uint32_t nLoose = sOff[P];
  const uint32_t n = min(nLoose, kResultTracks);
  // ---- the whole list, gathered from the cluster's shared memories
  for (uint32_t k = 0; k < P; ++k) {
    const uint32_t* src = cl.map_shared_rank(sLocal, k);
    const uint32_t o = sOff[k], m = min(sOff[k + 1], n) > o ? min(sOff[k + 1], n) - o : 0u;
    for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) sIdx[o + j] = src[j];
  }
  // no CTA may leave (and release its shared memory) before all have read
  cl.sync();
  // ---- this CTA's slice of every output array
  auto sl = [&](uint32_t len, uint32_t& a, uint32_t& b) {
    a = uint32_t(uint64_t(len) * r / P);
    b = uint32_t(uint64_t(len) * (r + 1) / P);
  };
  const uint32_t T = blockDim.x;
  uint32_t a, b;
  uint32_t* w32 = reinterpret_cast<uint32_t*>(base + kResOffTupleIndex);
  sl(n, a, b);
  for (uint32_t j = a + threadIdx.x; j < b; j += T) w32[j] = sIdx[j];
  w32 = reinterpret_cast<uint32_t*>(base + kResOffNHits);
  sl((n + 3) / 4, a, b);
  for (uint32_t w = a + threadIdx.x; w < b; w += T)
    w32[w] = packBytes(w, n, [&](uint32_t i) { return toff[sIdx[i] + 1] - toff[sIdx[i]]; });
  w32 = reinterpret_cast<uint32_t*>(base + kResOffQuality);
  for (uint32_t w = a + threadIdx.x; w < b; w += T) w32[w] = packBytes(w, n, [&](uint32_t i) { return q[sIdx[i]]; });
  float* f = reinterpret_cast<float*>(base + kResOffState);
  sl(5 * n, a, b);
  for (uint32_t j = a + threadIdx.x; j < b; j += T) f[j] = ws.state[tb * 5 + size_t(sIdx[j / 5]) * 5 + j % 5];
  f = reinterpret_cast<float*>(base + kResOffCov);
  sl(15 * n, a, b);
  for (uint32_t j = a + threadIdx.x; j < b; j += T) f[j] = ws.cov[tb * 15 + size_t(sIdx[j / 15]) * 15 + j % 15];
  sl(n, a, b);
  f = reinterpret_cast<float*>(base + kResOffPt);
  for (uint32_t j = a + threadIdx.x; j < b; j += T) f[j] = ws.pt[tb + sIdx[j]];
  f = reinterpret_cast<float*>(base + kResOffEta);
  for (uint32_t j = a + threadIdx.x; j < b; j += T) f[j] = ws.eta[tb + sIdx[j]];
  f = reinterpret_cast<float*>(base + kResOffChi2);
  for (uint32_t j = a + threadIdx.x; j < b; j += T) f[j] = ws.chi2[tb + sIdx[j]];
  w32 = reinterpret_cast<uint32_t*>(base + kResOffHits);
  sl(5 * n, a, b);
  for (uint32_t i = a + threadIdx.x; i < b; i += T) {
    const uint32_t t = sIdx[i / 5], k = i % 5;
    w32[i] = k < toff[t + 1] - toff[t] ? th[toff[t] + k] : 0xffffffffu;
  }
  const bool hasVtx = c->nVertices > 0;
  w32 = reinterpret_cast<uint32_t*>(base + kResOffVertex);
  sl((n + 1) / 2, a, b);
  for (uint32_t w = a + threadIdx.x; w < b; w += T)
    w32[w] = packHalves(w, n, [&](uint32_t i) { return hasVtx ? uint32_t(uint16_t(ws.idv[tb + sIdx[i]])) : 0xffffu; });
  const uint32_t nv = min(c->nVertices, uint32_t(kMaxVtx));
  const size_t vb = size_t(e) * kMaxVtx;
  ResultVertices vtx = resultVertices(base);
  sl(nv, a, b);
  for (uint32_t v = a + threadIdx.x; v < b; v += T) {
    vtx.zv[v] = ws.zv[vb + v];
    vtx.wv[v] = ws.wv[vb + v];
    vtx.chi2[v] = ws.vchi2[vb + v];
    vtx.ptv2[v] = ws.ptv2[vb + v];
    vtx.ndof[v] = ws.ndof[vb + v];
  }
  w32 = reinterpret_cast<uint32_t*>(base + kResOffSortInd);
  sl((nv + 1) / 2, a, b);
  for (uint32_t w = a + threadIdx.x; w < b; w += T)
    w32[w] = packHalves(w, nv, [&](uint32_t i) { return uint32_t(ws.sortInd[vb + i]); });
  if (r == 0 && threadIdx.x == 0) {
    ResultHeader h{};
    h.nTracks = n;
    h.nLooseAll = nLoose;
    h.nVertices = nv;
    h.nHits = c->nHits;
    h.nTuples = guard;
    h.nDigis = c->nWords;
    h.nCells = c->nCells;
    h.flags = c->flags | (nLoose > kResultTracks ? kFlagResultOverflow : 0u);
    h.nEdges = c->nEdges;
    h.nTupleHits = toff[guard];
    h.nModules = c->nModules;
    h.nearDoublet = c->nearDoublet;
    h.nearCA = c->nearCA;
    h.nearQuality = c->nearQuality;
    *reinterpret_cast<ResultHeader*>(base) = h;
    // the loose-track count of pg_event_counts (the last writer of the
    // quality codes, the triplet cleaner, has finished)
    ws.ev[e].nLoose = nLoose;
  }
}

}  // namespace

void launchSetInput(Workspace& ws, const uint32_t* words, const uint8_t* fedIds, cudaStream_t s) {
  PG_PROBED("kSetInput", s, kSetInput<<<1, 1, 0, s>>>(ws.input, words, fedIds));
}

void launchPack(Workspace& ws, uint32_t nEvents, uint8_t* out, cudaStream_t s) {
  // opt in to more than 48 KB of dynamic shared memory, once per device
  static std::atomic<uint64_t> ready{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = uint64_t(1) << (dev & 63);
  if (!(ready.load() & bit)) {
    if (cudaFuncSetAttribute(kPackResults, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kPackSmemBytes)) ==
        cudaSuccess)
      ready.fetch_or(bit);
  }
  const uint32_t P = nEvents <= kClusterMaxEvents ? kPackCtas : 1;
  // a failed launch is reported by the stream's next error check
  PG_PROBED("kPackResults", s, (void)launchClustered(kPackResults, P, nEvents, 512, kPackSmemBytes, s, ws, out));
}

}  // namespace pixgpu
