// Pixel vertexing on B200: one block per event runs loadTracks,
// clusterTracksByDensity, fitVertices(50), splitVertices(9),
// fitVertices(5000) and sortByPt2 with the PixelVertexProducerCUDA
// configuration (minT=2, eps=0.07, errmax=0.01, chi2max=9, ptMin=0.5).
// Reference: plugin-PixelVertexFinding/gpuVertexFinderImpl.h:10-43,
// gpuClusterTracksByDensity.h:20-207, gpuFitVertices.h:15-98,
// gpuSplitVertices.h:15-125, gpuSortByPt2.h:15-55,
// PixelVertexProducerCUDA.cc:16-26.
//
// All float sums run sequentially per vertex in ascending track order (the
// serial order), histogram bins are scanned in the serial storage order
// (descending track index inside a bin) and new split vertices are numbered
// by a prefix over the parent vertex index.
#include <atomic>

#include <cooperative_groups.h>

#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

// the per-event scratch stride is at least the reference's 2 x 458752 words
// (pixgpu_internal.cuh referenceCaps; larger capacities only widen it)
static_assert(kVtxScratchAWords <= 2 * size_t(PF_MAX_DOUBLETS_PARAM) &&
                  kVtxScratchBWords <= 2 * size_t(PF_MAX_DOUBLETS_PARAM),
              "vertex scratch exceeds the per-event scratchA/scratchB stride");
constexpr int kVtxThreads = 1024;
// events with at most this many vertex tracks keep every per-track array in
// shared memory (40 bytes per track: 220 KB, about the vertex tracks of a
// PU 250 event); larger ones use the global scratch
constexpr uint32_t kSmemTracks = 5500;
constexpr size_t kTrackBytes = 9 * 4 + 2 + 2;
constexpr size_t kVtxSmemBytes = kSmemTracks * kTrackBytes;
// with the kernel's static shared memory (about 9.4 KB) within the 227 KB of a block
static_assert(kVtxSmemBytes + 10 * 1024 <= 227 * 1024, "vertex shared memory");
constexpr uint32_t kVtxCtas = 4;  // CTAs per event in a small batch

struct VtxScratch {
  float *zt, *ezt2, *ptt2, *zz;
  uint32_t* itrk;    // tuple index of each vertex track
  uint8_t *izt, *newV;
  int32_t *iv, *nn, *root;
  uint32_t* list;    // tracks grouped by vertex
  uint16_t* hbins;   // z-histogram content
};

__device__ __forceinline__ VtxScratch carve(char* p, uint32_t cap) {
  VtxScratch s;
  s.zt = reinterpret_cast<float*>(p);
  s.ezt2 = s.zt + cap;
  s.ptt2 = s.ezt2 + cap;
  s.zz = s.ptt2 + cap;
  s.iv = reinterpret_cast<int32_t*>(s.zz + cap);
  s.nn = s.iv + cap;
  s.root = s.nn + cap;
  s.list = reinterpret_cast<uint32_t*>(s.root + cap);
  s.itrk = s.list + cap;
  s.hbins = reinterpret_cast<uint16_t*>(s.itrk + cap);
  s.izt = reinterpret_cast<uint8_t*>(s.hbins + cap);
  s.newV = s.izt + cap;
  return s;
}

__device__ __forceinline__ VtxScratch scratchOf(const Workspace& ws, uint32_t e) {
  // carve per-event scratch out of scratchA/scratchB (cap.scratch words each;
  // kVtxScratchAWords and kVtxScratchBWords of them are used)
  uint32_t* a = ws.scratchA + size_t(e) * ws.cap.scratch;
  uint32_t* b = ws.scratchB + size_t(e) * ws.cap.scratch;
  VtxScratch s;
  s.zt = reinterpret_cast<float*>(a);
  s.ezt2 = reinterpret_cast<float*>(a + kMaxVtxTracks);
  s.ptt2 = reinterpret_cast<float*>(a + 2 * kMaxVtxTracks);
  s.zz = reinterpret_cast<float*>(a + 3 * kMaxVtxTracks);
  s.iv = reinterpret_cast<int32_t*>(a + 4 * kMaxVtxTracks);
  s.nn = reinterpret_cast<int32_t*>(a + 5 * kMaxVtxTracks);
  s.root = reinterpret_cast<int32_t*>(a + 6 * kMaxVtxTracks);
  s.list = a + 7 * kMaxVtxTracks;
  s.itrk = a + 8 * kMaxVtxTracks;
  static_assert(9 * size_t(kMaxVtxTracks) == kVtxScratchAWords, "scratch A layout");
  s.hbins = reinterpret_cast<uint16_t*>(b);
  s.izt = reinterpret_cast<uint8_t*>(b + kMaxVtxTracks / 2);
  s.newV = reinterpret_cast<uint8_t*>(b + kMaxVtxTracks / 2) + kMaxVtxTracks;
  static_assert(size_t(kMaxVtxTracks) / 2 + 2 * size_t(kMaxVtxTracks) / 4 == kVtxScratchBWords, "scratch B layout");
  return s;
}

// group tracks by vertex id (ascending track order inside each vertex)
__device__ void groupByVertex(const VtxScratch& s, uint32_t nt, uint32_t nv, uint32_t* vOff, uint32_t* vCur,
                              uint32_t* scanSh) {
  for (uint32_t v = threadIdx.x; v <= nv; v += blockDim.x) {
    vOff[v] = 0;
    vCur[v] = 0;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
    int32_t v = s.iv[i];
    if (v >= 0 && uint32_t(v) < nv) atomicAdd(&vOff[v], 1u);
  }
  __syncthreads();
  uint32_t carry = 0;
  for (uint32_t v0 = 0; v0 <= nv; v0 += blockDim.x) {
    uint32_t v = v0 + threadIdx.x;
    uint32_t c = v <= nv ? vOff[v] : 0u;
    uint32_t tot;
    uint32_t pre = blockExclusiveScan(c, scanSh, &tot);
    if (v <= nv) vOff[v] = carry + pre;
    carry += tot;
  }
  __syncthreads();
  // ordered fill (ascending track order inside each vertex).  Few vertices:
  // one warp per vertex walks the tracks, 128 at a time, until it has found
  // them all.  Many: warp w owns a range of vertices and walks the tracks
  // once, 32 at a time; lanes of the same vertex are ranked among themselves
  // (match) and its cursor (vCur) advances by their number.
  const uint32_t lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (nv <= 2 * nw) {
    for (uint32_t v = threadIdx.x >> 5; v < nv; v += nw) {
      uint32_t pos = vOff[v];
      const uint32_t end = vOff[v + 1];
      for (uint32_t i0 = 0; i0 < nt && pos < end; i0 += 128) {
        bool in[4];
#pragma unroll
        for (uint32_t u = 0; u < 4; ++u) {
          const uint32_t i = i0 + u * 32 + lane;
          in[u] = i < nt && s.iv[i] == int32_t(v);
        }
#pragma unroll
        for (uint32_t u = 0; u < 4; ++u) {
          const uint32_t m = __ballot_sync(0xffffffffu, in[u]);
          if (in[u]) s.list[pos + __popc(m & lanemaskLt())] = i0 + u * 32 + lane;
          pos += __popc(m);
        }
      }
    }
  } else {
    for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) vCur[v] = vOff[v];
    __syncthreads();
    const uint32_t vpw = (nv + nw - 1) / nw, vLo = (threadIdx.x >> 5) * vpw, vHi = min(nv, vLo + vpw);
    for (uint32_t i0 = 0; i0 < nt && vLo < vHi; i0 += 32) {
      const uint32_t i = i0 + lane;
      const int32_t v = i < nt ? s.iv[i] : -1;
      const bool in = v >= int32_t(vLo) && v < int32_t(vHi);
      const uint32_t m = __ballot_sync(0xffffffffu, in);
      if (m) {
        const uint32_t peers = __match_any_sync(0xffffffffu, in ? uint32_t(v) : 0xffffffffu) & m;
        if (in) {
          s.list[vCur[v] + __popc(peers & lanemaskLt())] = i;
          __syncwarp(peers);
          if ((peers & lanemaskLt()) == 0) vCur[v] += __popc(peers);
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();
}

// Float sums that must follow the serial order (ascending track order inside
// a vertex) are formed by a warp: the lanes evaluate 32 consecutive terms at
// once and every lane adds them in order from the shuffles.  Terms of tracks
// that the serial loop skips are +0.0, which leaves a sum unchanged (a sum
// that starts at +0.0 never becomes -0.0 under round-to-nearest).

// sum + the 32 lanes' terms, added in lane order (every lane gets the sum).
// All 32 terms are added: the lanes past the vertex's tracks hold +0.0, which
// leaves the sum unchanged.  Unrolled, the shuffles issue back to back and
// only the additions form the dependent chain.
__device__ __forceinline__ float laneOrderSum(float sum, float t) {
#pragma unroll
  for (int l = 0; l < 32; ++l) sum += __shfl_sync(0xffffffffu, t, l);
  return sum;
}

// fitVertices: weighted z, chi2 outlier rejection (iv = 9999), ndof and weight;
// one warp per vertex
__device__ void fitVertices(const VtxScratch& s, uint32_t nt, uint32_t nv, float chi2Max, float* zv, float* wv,
                            float* chi2, int32_t* ndof, uint32_t* vOff, uint32_t* vCur, uint32_t* scanSh) {
  groupByVertex(s, nt, nv, vOff, vCur, scanSh);
  const uint32_t lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (uint32_t v = threadIdx.x >> 5; v < nv; v += nw) {
    const uint32_t b = vOff[v], n = vOff[v + 1] - b;
    float z = 0, w = 0;
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
      const uint32_t k = k0 + lane;
      float tz = 0.f, tw = 0.f;
      if (k < n) {
        const uint32_t i = s.list[b + k];
        const float wi = 1.f / s.ezt2[i];
        tz = s.zt[i] * wi;
        tw = wi;
      }
      z = laneOrderSum(z, tz);
      w = laneOrderSum(w, tw);
    }
    z /= w;
    int32_t nd = -1;
    float c2s = 0;
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
      const uint32_t k = k0 + lane;
      float t = 0.f;
      bool acc = false;
      if (k < n) {
        const uint32_t i = s.list[b + k];
        float c2 = z - s.zt[i];
        c2 *= c2 / s.ezt2[i];
        if (c2 > chi2Max) {
          s.iv[i] = 9999;
        } else {
          acc = true;
          t = c2;
        }
      }
      nd += __popc(__ballot_sync(0xffffffffu, acc));
      c2s = laneOrderSum(c2s, t);
    }
    if (nd > 0) w *= float(nd) / c2s;
    if (lane == 0) {
      zv[v] = z;
      wv[v] = w;
      chi2[v] = c2s;
      ndof[v] = nd;
    }
  }
  __syncthreads();
}

// order-preserving map of a float to unsigned (negative values reversed)
__device__ __forceinline__ uint32_t orderedBits(float x) {
  const uint32_t u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// DBSCAN (gpuClusterTracksDBSCAN.h:16-227) and iterative
// (gpuClusterTracksIterative.h:16-201) clustering after the neighbour counts:
// iv[i] left pointing at track i's root (the numbering that follows is the
// one of the density clusterer).  One block; warp per track for the
// neighbour loops, whose serial order is reproduced by (key, position)
// reductions; a track whose candidates include a NaN is done by lane 0
// literally.
__device__ void clusterCoresAndEdges(const VtxScratch& s, uint32_t nt, const uint32_t* hoff, int algo, float eps,
                                     float chi2max, int32_t minT, int* sFlag) {
  const uint32_t lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  auto range = [&](uint32_t i, uint32_t& pb, uint32_t& pe) {
    const int b0 = max(0, int(s.izt[i]) - 1), b1 = min(255, int(s.izt[i]) + 1);
    pb = hoff[b0];
    pe = hoff[b1 + 1];
  };
  auto percolate = [&]() {
    for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
      int32_t m = s.iv[i];
      while (m != s.iv[m]) m = s.iv[m];
      s.root[i] = m;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) s.iv[i] = s.root[i];
    __syncthreads();
  };
  if (algo == 1) {
    // core tracks: the core neighbour of lowest z below the track's own
    // (first in bin order among equal z)
    for (uint32_t i = threadIdx.x >> 5; i < nt; i += nw) {
      if (s.nn[i] < minT) continue;
      uint32_t pb, pe;
      range(i, pb, pe);
      const float zi = s.zt[i];
      unsigned long long best = ~0ull;
      bool nan = isnan(zi);
      for (uint32_t p = pb + lane; p < pe; p += 32) {
        const uint32_t j = s.hbins[p];
        const float zj = s.zt[j];
        nan |= isnan(zj);
        if (!(zj < zi) || s.nn[j] < minT || fabsf(zi - zj) > eps) continue;
        const unsigned long long key = (uint64_t(orderedBits(zj)) << 32) | p;
        best = key < best ? key : best;
      }
      if (__any_sync(0xffffffffu, nan)) {
        if (lane == 0) {  // the serial loop as written
          float mz = zi;
          for (uint32_t p = pb; p < pe; ++p) {
            const uint32_t j = s.hbins[p];
            if (s.zt[j] >= mz || s.nn[j] < minT || fabsf(zi - s.zt[j]) > eps) continue;
            mz = s.zt[j];
            s.iv[i] = int32_t(j);
          }
        }
        continue;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
        best = other < best ? other : best;
      }
      if (lane == 0 && best != ~0ull) s.iv[i] = int32_t(s.hbins[uint32_t(best & 0xffffffffu)]);
    }
    __syncthreads();
    percolate();
  } else {
    // connected components of the compatible core tracks: every label
    // becomes the lowest track index of its component, the fixed point of the
    // reference's alternating min-propagation and percolation
    for (uint32_t it = 0; it <= nt + 1; ++it) {
      if (threadIdx.x == 0) *sFlag = 0;
      __syncthreads();
      for (uint32_t i = threadIdx.x >> 5; i < nt; i += nw) {
        if (s.nn[i] < minT) continue;
        uint32_t pb, pe;
        range(i, pb, pe);
        const float zi = s.zt[i], ei = s.ezt2[i];
        int32_t m = s.iv[i];
        for (uint32_t p = pb + lane; p < pe; p += 32) {
          const uint32_t j = s.hbins[p];
          if (j == i || s.nn[j] < minT) continue;
          const float dist = fabsf(zi - s.zt[j]);
          if (dist > eps || dist * dist > chi2max * (ei + s.ezt2[j])) continue;
          m = min(m, s.iv[j]);
        }
        m = __reduce_min_sync(0xffffffffu, m);
        if (lane == 0 && m < s.iv[i]) {
          atomicMin(&s.iv[i], m);
          *sFlag = 1;
        }
      }
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
        const int32_t l = s.iv[i], ll = s.iv[l];
        if (ll < l) {
          atomicMin(&s.iv[i], ll);
          *sFlag = 1;
        }
      }
      __syncthreads();
      const int more = *sFlag;
      __syncthreads();
      if (!more) break;
    }
  }
  // edge rule: a non-core track joins its closest chi2-compatible core
  // neighbour (last in bin order among equal distances)
  for (uint32_t i = threadIdx.x >> 5; i < nt; i += nw) {
    if (s.nn[i] >= minT) continue;
    uint32_t pb, pe;
    range(i, pb, pe);
    const float zi = s.zt[i], ei = s.ezt2[i];
    unsigned long long best = ~0ull;
    bool nan = false;
    for (uint32_t p = pb + lane; p < pe; p += 32) {
      const uint32_t j = s.hbins[p];
      if (s.nn[j] < minT) continue;
      const float dist = fabsf(zi - s.zt[j]);
      nan |= isnan(dist) || isnan(chi2max * (ei + s.ezt2[j]));
      if (dist > eps || dist * dist > chi2max * (ei + s.ezt2[j])) continue;
      const unsigned long long key = (uint64_t(__float_as_uint(dist)) << 32) | uint64_t(0xffffffffu - p);
      best = key < best ? key : best;
    }
    if (__any_sync(0xffffffffu, nan)) {
      if (lane == 0) {
        s.root[i] = s.iv[i];
        float mdist = eps;
        for (uint32_t p = pb; p < pe; ++p) {
          const uint32_t j = s.hbins[p];
          if (s.nn[j] < minT) continue;
          const float dist = fabsf(zi - s.zt[j]);
          if (dist > mdist || dist * dist > chi2max * (ei + s.ezt2[j])) continue;
          mdist = dist;
          s.root[i] = s.iv[j];
        }
      }
      continue;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
      best = other < best ? other : best;
    }
    if (lane == 0) s.root[i] = best != ~0ull ? s.iv[s.hbins[0xffffffffu - uint32_t(best & 0xffffffffu)]] : s.iv[i];
  }
  __syncthreads();
  // edge tracks take their core's root; the others keep theirs
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x)
    if (s.nn[i] < minT) s.iv[i] = s.root[i];
  __syncthreads();
}

// Launched as a cluster of P CTAs per event (P = 1 for large batches).  With
// P > 1 and the per-track arrays in shared memory, every CTA builds the track
// arrays and the z histogram, the two neighbour searches are divided among the
// CTAs by track, each result written into every CTA's shared memory, and rank
// 0 alone continues from there.
__global__ void __launch_bounds__(kVtxThreads) kVertices(Workspace ws, int algo) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t rank = cl.block_rank(), P = cl.num_blocks();
  extern __shared__ __align__(16) char vsm[];
  __shared__ uint32_t scanSh[33];
  __shared__ uint32_t hoff[257];
  __shared__ uint32_t vOff[kMaxVtx + 1], vCur[kMaxVtx + 1];
  __shared__ uint32_t sNt, sFound, sGuard, sNv;
  __shared__ uint32_t sCtaCnt;  // tracks this CTA selected
  __shared__ int sFlag;
  const uint32_t e = blockIdx.y;
  const uint32_t lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  EventCounters* c = ws.ev + e;
  const uint32_t nTuples = c->nTuples;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  const uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  const float* pt = ws.pt + size_t(e) * ws.cap.tuples;
  const float* st = ws.state + size_t(e) * ws.cap.tuples * 5;
  const float* cov = ws.cov + size_t(e) * ws.cap.tuples * 15;
  int16_t* idv = ws.idv + size_t(e) * ws.cap.tuples;
  float* zv = ws.zv + size_t(e) * kMaxVtx;
  float* wv = ws.wv + size_t(e) * kMaxVtx;
  float* vchi2 = ws.vchi2 + size_t(e) * kMaxVtx;
  float* ptv2 = ws.ptv2 + size_t(e) * kMaxVtx;
  int32_t* ndof = ws.ndof + size_t(e) * kMaxVtx;
  uint16_t* sortInd = ws.sortInd + size_t(e) * kMaxVtx;

  // ---- loadTracks: the serial loop stops at the first empty tuple
  if (threadIdx.x == 0) {
    uint32_t g = nTuples;
    const uint32_t bins = ws.cap.tuples;
    if (nTuples == bins && toff[bins] == toff[bins - 1]) g = bins - 1;
    sGuard = g;
  }
  __syncthreads();
  const uint32_t guard = sGuard;
  // the selection of tuple t, its four loads issued together
  auto selected = [&](uint32_t t) {
    const uint32_t nh = toff[t + 1] - toff[t];
    const uint8_t qt = q[t];
    const float ptt = pt[t];
    return (nh >= 4) & (qt == 2) & !(ptt < 0.5f);
  };
  // The cluster's CTAs split the tuples: CTA r takes [g0, g1).  Inside it each
  // warp takes a contiguous range, 32 consecutive tuples per step (coalesced
  // loads, four steps in flight).  Block scans over the warps' counts and the
  // CTAs' counts place every run, and a second walk writes the selected tracks
  // in ascending order (into every CTA's shared memory, or the global
  // scratch).  The selection of each step is kept as a bit when the range has
  // at most 32 steps, else evaluated again.
  const uint32_t g0 = uint32_t(uint64_t(guard) * rank / P), g1 = uint32_t(uint64_t(guard) * (rank + 1) / P);
  for (uint32_t t = g0 + threadIdx.x; t < g1; t += blockDim.x) idv[t] = -1;
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t R = (g1 - g0 + nw * 32 - 1) / (nw * 32) * 32;
  const uint32_t w0 = min(g1, g0 + warp * R), w1 = min(g1, w0 + R);
  const uint32_t steps = (w1 - w0 + 31) / 32;
  const bool keepBits = steps <= 32;
  uint32_t cnt = 0, bits = 0;
  for (uint32_t k = 0; k < steps; k += 4) {
    bool sel[4];
#pragma unroll
    for (uint32_t u = 0; u < 4; ++u) {
      const uint32_t t = w0 + (k + u) * 32 + lane;
      sel[u] = k + u < steps && t < w1 && selected(t);
    }
#pragma unroll
    for (uint32_t u = 0; u < 4; ++u) {
      if (sel[u] && keepBits) bits |= 1u << (k + u);
      cnt += __popc(__ballot_sync(0xffffffffu, sel[u]));
    }
  }
  uint32_t ctaTotal;
  const uint32_t first = __shfl_sync(0xffffffffu, blockExclusiveScan(lane == 0 ? cnt : 0u, scanSh, &ctaTotal), 0);
  if (threadIdx.x == 0) sCtaCnt = ctaTotal;
  // every CTA has started and holds its count (and every tuple's idv is
  // cleared): the counts are read across the cluster
  cl.sync();
  uint32_t base = 0, total = 0;
  for (uint32_t r = 0; r < P; ++r) {
    const uint32_t n = *cl.map_shared_rank(&sCtaCnt, r);
    base += r < rank ? n : 0u;
    total += n;
  }
  if (threadIdx.x == 0) {
    sNt = min(total, kMaxVtxTracks);
    // beyond ZVertexSoA::MAXTRACKS the reference writes past its arrays
    if (total > kMaxVtxTracks && rank == 0) atomicOr(&c->flags, kFlagVtxOverflow);
  }
  __syncthreads();
  // The count decides where the per-track arrays live: in the shared memory
  // of every CTA, or once in the global scratch.  The neighbour searches are
  // split among the cluster's CTAs (the density clusterer); their results go
  // to every CTA's shared memory, or once to the global scratch.
  const bool smemPath = sNt <= kSmemTracks;
  const VtxScratch s = smemPath ? carve(vsm, kSmemTracks) : scratchOf(ws, e);
  const bool split = P > 1 && algo == 0;
  const bool remote = split && smemPath;       // results written into every CTA
  const bool active = split || rank == 0;      // CTAs that take part in the searches
  const bool writer = smemPath || rank == 0;   // CTAs that build their own track arrays
  const uint32_t wFirst = split ? rank * nw : 0, wStride = split ? P * nw : nw;
  // every CTA places its selected tracks; in the shared-memory path each
  // track goes to every CTA that works on it (all with the split, else rank 0)
  const uint32_t nDst = smemPath ? (split ? P : 1u) : 1u;
  {
    uint32_t pos = base + first;
    for (uint32_t k = 0; k < steps; k += 4) {
      bool sel[4];
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t t = w0 + (k + u) * 32 + lane;
        sel[u] = keepBits ? ((bits >> (k + u)) & 1u) != 0 : (k + u < steps && t < w1 && selected(t));
      }
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t t = w0 + (k + u) * 32 + lane;
        const uint32_t m = __ballot_sync(0xffffffffu, sel[u]);
        const uint32_t it = pos + __popc(m & lanemaskLt());
        if (sel[u] && it < kMaxVtxTracks) {
          const float z = st[size_t(t) * 5 + 4], ez = cov[size_t(t) * 15 + 14], p2 = pt[t] * pt[t];
          for (uint32_t d = 0; d < nDst; ++d) {
            VtxScratch sd = s;
            if (smemPath) sd = carve(reinterpret_cast<char*>(cl.map_shared_rank(vsm, split ? d : 0u)), kSmemTracks);
            sd.itrk[it] = t;
            sd.zt[it] = z;
            sd.ezt2[it] = ez;
            sd.ptt2[it] = p2;
          }
        }
        pos += __popc(m);
      }
    }
  }
  // every track array is complete
  cl.sync();
  const uint32_t nt = sNt;
  const float eps = 0.07f, errmax = 0.01f, chi2max = 9.f;
  const float er2mx = errmax * errmax;

  if (active) {
  // ---- clusterTracksByDensity: z histogram (256 bins of 1 mm)
  for (uint32_t b = threadIdx.x; b < 257; b += blockDim.x) hoff[b] = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
    int iz = int(double(s.zt[i]) * 10.);
    iz = min(max(iz, -128), 127);
    atomicAdd(&hoff[iz + 128], 1u);
    if (writer) {
      s.izt[i] = uint8_t(iz + 128);
      s.iv[i] = int32_t(i);
      s.nn[i] = 0;
    }
  }
  __syncthreads();
  {
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < 257; b0 += blockDim.x) {
      uint32_t b = b0 + threadIdx.x;
      uint32_t v = b < 257 ? hoff[b] : 0u;
      uint32_t tot;
      uint32_t pre = blockExclusiveScan(v, scanSh, &tot);
      if (b < 257) hoff[b] = carry + pre;
      carry += tot;
    }
  }
  __syncthreads();
  // the serial fill stores each bin in descending track order.  Warp w owns
  // bins [8 w, 8 w + 8) and walks the tracks once from the last one down,
  // 32 at a time: lanes holding the same bin are ranked among themselves
  // (match), and the bin's cursor advances by their number.
  if (writer) {
    uint32_t* cur = vCur;  // free until the vertex fit: per-bin fill cursors
    for (uint32_t b = threadIdx.x; b < 256; b += blockDim.x) cur[b] = hoff[b];
    __syncthreads();
    const uint32_t bpw = (256 + nw - 1) / nw, bLo = (threadIdx.x >> 5) * bpw, bHi = min(256u, bLo + bpw);
    for (uint32_t r0 = 0; r0 < nt && bLo < bHi; r0 += 32) {
      const uint32_t r = r0 + lane;
      const uint32_t i = nt - 1 - r;
      const uint32_t b = r < nt ? s.izt[i] : 0xffffu;
      const bool in = b >= bLo && b < bHi;
      const uint32_t m = __ballot_sync(0xffffffffu, in);
      if (m) {
        const uint32_t peers = __match_any_sync(0xffffffffu, in ? b : 0xffffffffu) & m;
        if (in) {
          const uint32_t pos = cur[b] + __popc(peers & lanemaskLt());
          s.hbins[pos] = uint16_t(i);
          __syncwarp(peers);
          if ((peers & lanemaskLt()) == 0) cur[b] += __popc(peers);
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // z and its error of every track in histogram order, so that the
    // neighbour searches read their candidates contiguously (zz and list are
    // free until the fits)
    float* zP = s.zz;
    float* eP = reinterpret_cast<float*>(s.list);
    for (uint32_t p = threadIdx.x; p < nt; p += blockDim.x) {
      const uint32_t j = s.hbins[p];
      zP[p] = s.zt[j];
      eP[p] = s.ezt2[j];
    }
  }
  }
  // every CTA of the cluster has cleared its own neighbour counts before any
  // CTA writes counts into the others' shared memory; the global scratch's
  // histogram is complete
  cl.sync();
  // candidates in histogram order: z, its error and (below) the neighbour count
  const float* zP = s.zz;
  const float* eP = reinterpret_cast<const float*>(s.list);
  int32_t* nP = s.root;  // free until the percolation
  if (active) {
  // neighbour counts: one warp per track (taken in histogram order), the
  // lanes take 32 consecutive entries of the track's three bins at a time.
  // Each count is kept by track (nn) and by histogram position (nP).
  for (uint32_t pi = wFirst + (threadIdx.x >> 5); pi < nt; pi += wStride) {
    const uint32_t i = s.hbins[pi];
    const float zi = zP[pi], ei = eP[pi];
    uint32_t cnt = 0;  // per lane, summed once per track
    if (!(ei > er2mx)) {
      const int b0 = max(0, int(s.izt[i]) - 1), b1 = min(255, int(s.izt[i]) + 1);
      const uint32_t pb = hoff[b0], pe = hoff[b1 + 1];
      for (uint32_t p = pb + lane; p < pe; p += 32) {
        const uint32_t j = s.hbins[p];
        const float dist = fabsf(zi - zP[p]);
        cnt += (i != j && !(dist > eps) && (algo == 1 || !(dist * dist > chi2max * (ei + eP[p])))) ? 1u : 0u;
      }
      cnt = __reduce_add_sync(0xffffffffu, cnt);
    }
    if (remote ? lane < P : lane == 0) {
      *(remote ? cl.map_shared_rank(s.nn, lane) + i : s.nn + i) = int32_t(cnt);
      *(remote ? cl.map_shared_rank(nP, lane) + pi : nP + pi) = int32_t(cnt);
    }
  }
  }
  // every CTA holds every neighbour count
  cl.sync();
  if (active && algo != 0) clusterCoresAndEdges(s, nt, hoff, algo, eps, chi2max, 2, &sFlag);
  if (active && algo == 0) {
  // Closest denser neighbour.  The serial loop (mdist starts at eps; a
  // candidate is taken when denser, not farther than mdist and
  // chi2-compatible) ends on the last candidate of minimal distance among the
  // qualifying ones -- unless a candidate with a NaN distance qualifies: from
  // then on every denser, chi2-compatible candidate is taken, so the result
  // is the last of those.  The warp evaluates both, the first as the minimum
  // of (distance, reversed position).
  for (uint32_t pi = wFirst + (threadIdx.x >> 5); pi < nt; pi += wStride) {
    const uint32_t i = s.hbins[pi];
    const int b0 = max(0, int(s.izt[i]) - 1), b1 = min(255, int(s.izt[i]) + 1);
    const uint32_t pb = hoff[b0], pe = hoff[b1 + 1];
    const float zi = zP[pi], ei = eP[pi];
    const int32_t ni = nP[pi];
    // per-lane running results, combined once per track
    unsigned long long bestKey = ~0ull;
    bool nanLane = false;
    int32_t lastOk = -1;
    for (uint32_t p = pb + lane; p < pe; p += 32) {
      const int32_t nj = nP[p];
      const float zj = zP[p];
      const float dist = fabsf(zi - zj);
      const bool dens = !(nj < ni) && !(nj == ni && zj >= zi);
      const bool dc = dens && !(dist * dist > chi2max * (ei + eP[p]));
      nanLane |= dens && isnan(dist);
      if (dc) {
        lastOk = int32_t(p);
        if (!(dist > eps)) {
          const unsigned long long key = (uint64_t(__float_as_uint(dist)) << 32) | uint64_t(0xffffffffu - p);
          bestKey = key < bestKey ? key : bestKey;
        }
      }
    }
    const bool anyNaN = __any_sync(0xffffffffu, nanLane);
    lastOk = __reduce_max_sync(0xffffffffu, lastOk);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, bestKey, o);
      bestKey = other < bestKey ? other : bestKey;
    }
    int32_t best = int32_t(i);
    if (anyNaN)
      best = int32_t(s.hbins[lastOk]);
    else if (bestKey != ~0ull)
      best = int32_t(s.hbins[0xffffffffu - uint32_t(bestKey & 0xffffffffu)]);
    if (remote ? lane < P : lane == 0) *(remote ? cl.map_shared_rank(s.iv, lane) + i : s.iv + i) = best;
  }
  }
  // every CTA holds every closest denser neighbour; only rank 0 goes on,
  // and no CTA reads another CTA's shared memory after this point
  cl.sync();
  if (rank != 0) return;
  // percolate to the seed
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
    int32_t m = s.iv[i];
    while (m != s.iv[m]) m = s.iv[m];
    s.root[i] = m;
  }
  __syncthreads();
  // number the seeds with nn >= minT in ascending track order
  {
    uint32_t carry = 0;
    for (uint32_t i0 = 0; i0 < nt; i0 += blockDim.x) {
      uint32_t i = i0 + threadIdx.x;
      uint32_t seed = (i < nt && s.root[i] == int32_t(i) && s.nn[i] >= 2) ? 1u : 0u;
      uint32_t tot;
      uint32_t pre = blockExclusiveScan(seed, scanSh, &tot);
      if (seed) s.iv[i] = int32_t(carry + pre);  // rank of the seed
      carry += tot;
    }
    if (threadIdx.x == 0) sFound = carry;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
    int32_t r = s.root[i];
    // seeds hold their rank in iv[r]; noise seeds end as 9997 (= -(-9998) - 1)
    s.zz[i] = 0;
    s.newV[i] = 0;
    int32_t v = (s.nn[r] >= 2) ? s.iv[r] : 9997;
    s.root[i] = v;  // staged: iv of a seed is still read by other threads in this loop
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) s.iv[i] = s.root[i];
  __syncthreads();
  uint32_t found = sFound;
  if (found >= kMaxVtx) {
    if (threadIdx.x == 0) atomicOr(&c->flags, kFlagVtxOverflow);
    found = kMaxVtx - 1;
  }

  // ---- fitVertices(50)
  fitVertices(s, nt, found, 50.f, zv, wv, vchi2, ndof, vOff, vCur, scanSh);

  // ---- splitVertices(9): tracks of each vertex are the list built by the fit
  //      minus the ones rejected there (iv = 9999)
  if (threadIdx.x == 0) sNv = found;
  __syncthreads();
  for (uint32_t kv = threadIdx.x >> 5; kv < found; kv += nw) {
    if (lane == 0) vCur[kv] = 0;  // split flag
    if (ndof[kv] < 4) continue;
    if (vchi2[kv] < 9.f * float(ndof[kv])) continue;
    if (ndof[kv] >= 512) {
      if (lane == 0) atomicOr(&c->flags, kFlagVtxOverflow);
      continue;
    }
    const uint32_t b = vOff[kv], n = vOff[kv + 1] - b;
    for (uint32_t k = lane; k < n; k += 32) {
      const uint32_t i = s.list[b + k];
      if (s.iv[i] != int32_t(kv)) continue;
      s.zz[i] = s.zt[i] - zv[kv];
      s.newV[i] = s.zz[i] < 0 ? 0 : 1;
    }
    __syncwarp();
    float znew[2], wnew[2];
    int maxiter = 20;
    bool more = true;
    while (more) {
      more = false;
      znew[0] = znew[1] = 0;
      wnew[0] = wnew[1] = 0;
      for (uint32_t k0 = 0; k0 < n; k0 += 32) {
        const uint32_t k = k0 + lane;
        float z0 = 0.f, w0 = 0.f, z1 = 0.f, w1 = 0.f;
        if (k < n) {
          const uint32_t i = s.list[b + k];
          if (s.iv[i] == int32_t(kv)) {
            const float ww = 1.f / s.ezt2[i];
            const float p = s.zz[i] * ww;
            if (s.newV[i]) {
              z1 = p;
              w1 = ww;
            } else {
              z0 = p;
              w0 = ww;
            }
          }
        }
        znew[0] = laneOrderSum(znew[0], z0);
        wnew[0] = laneOrderSum(wnew[0], w0);
        znew[1] = laneOrderSum(znew[1], z1);
        wnew[1] = laneOrderSum(wnew[1], w1);
      }
      znew[0] /= wnew[0];
      znew[1] /= wnew[1];
      bool changed = false;
      for (uint32_t k = lane; k < n; k += 32) {
        const uint32_t i = s.list[b + k];
        if (s.iv[i] != int32_t(kv)) continue;
        const float d0 = fabsf(s.zz[i] - znew[0]);
        const float d1 = fabsf(s.zz[i] - znew[1]);
        const uint8_t newer = d0 < d1 ? 0 : 1;
        changed |= newer != s.newV[i];
        s.newV[i] = newer;
      }
      more = __any_sync(0xffffffffu, changed);
      __syncwarp();
      --maxiter;
      if (maxiter <= 0) more = false;
    }
    if (0 == wnew[0] || 0 == wnew[1]) continue;
    const float dist2 = (znew[0] - znew[1]) * (znew[0] - znew[1]);
    const float chi2Dist = dist2 / (1.f / wnew[0] + 1.f / wnew[1]);
    if (chi2Dist < 4) continue;
    if (lane == 0) vCur[kv] = 1;
  }
  __syncthreads();
  // new vertex numbers in ascending order of the vertex that was split
  {
    uint32_t carry = 0;
    for (uint32_t k0 = 0; k0 < found; k0 += blockDim.x) {
      uint32_t kv = k0 + threadIdx.x;
      uint32_t f = kv < found ? vCur[kv] : 0u;
      uint32_t tot;
      uint32_t pre = blockExclusiveScan(f, scanSh, &tot);
      if (kv < found) vCur[kv] = f ? (found + carry + pre + 1) : 0u;  // 0: no split, else igv+1
      carry += tot;
    }
    if (threadIdx.x == 0) sNv = found + carry;
  }
  __syncthreads();
  // tracks of the split-off halves to their new vertices (warp per vertex)
  for (uint32_t kv = threadIdx.x >> 5; kv < found; kv += nw) {
    if (vCur[kv] == 0) continue;
    const uint32_t igv = vCur[kv] - 1;
    const uint32_t b = vOff[kv], n = vOff[kv + 1] - b;
    for (uint32_t k = lane; k < n; k += 32) {
      const uint32_t i = s.list[b + k];
      if (s.iv[i] == int32_t(kv) && s.newV[i] == 1) s.iv[i] = int32_t(igv);
    }
  }
  __syncthreads();
  uint32_t nv = sNv;
  if (nv >= kMaxVtx) {
    if (threadIdx.x == 0) atomicOr(&c->flags, kFlagVtxOverflow);
    nv = kMaxVtx - 1;
  }

  // ---- fitVertices(5000)
  fitVertices(s, nt, nv, 5000.f, zv, wv, vchi2, ndof, vOff, vCur, scanSh);

  // ---- sortByPt2
  if (threadIdx.x == 0) c->nVertices = nv;
  if (nv < 1) return;
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) idv[s.itrk[i]] = int16_t(s.iv[i]);
  // the fit above left every vertex's accepted tracks in vOff/list order
  for (uint32_t v = threadIdx.x >> 5; v < nv; v += nw) {
    const uint32_t b = vOff[v], n = vOff[v + 1] - b;
    float p2 = 0;
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
      const uint32_t k = k0 + lane;
      float t = 0.f;
      if (k < n) {
        const uint32_t i = s.list[b + k];
        if (s.iv[i] <= 9990) t = s.ptt2[i];
      }
      p2 = laneOrderSum(p2, t);
    }
    if (lane == 0) ptv2[v] = p2;
  }
  __syncthreads();
  if (nv == 1) {
    if (threadIdx.x == 0) sortInd[0] = 0;
    return;
  }
  for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) {
    float p = ptv2[v];
    uint32_t r = 0;
    for (uint32_t u = 0; u < nv; ++u) {
      float o = ptv2[u];
      r += (o < p || (o == p && u < v)) ? 1u : 0u;
    }
    sortInd[r] = uint16_t(v);
  }
  if (threadIdx.x == 0) c->nVtxTracks = nt;
}

}  // namespace

cudaError_t runVertices(Workspace& ws, uint32_t nEvents, cudaStream_t stream, int algo) {
  // opt in to the large shared-memory carve-out, once per device
  static std::atomic<uint64_t> configured{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = uint64_t(1) << (dev & 63);
  if (!(configured.load() & bit)) {
    cudaError_t e = cudaFuncSetAttribute(kVertices, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kVtxSmemBytes));
    if (e != cudaSuccess) return e;
    configured.fetch_or(bit);
  }
  // small batches: a cluster of kVtxCtas CTAs per event shortens the event's
  // latency; large batches: pairs of CTAs (measured at 64 PU50 events: 0.52 ->
  // 0.39 ms per batch and +2 % throughput with three batches in flight).  Only
  // the density clusterer splits its work across the cluster; the others run
  // on one CTA.
  const uint32_t P = algo != 0 ? 1u : (nEvents <= kClusterMaxEvents ? kVtxCtas : 2u);
  cudaError_t le = cudaSuccess;
  PG_PROBED("kVertices", stream,
            le = launchClustered(kVertices, P, nEvents, kVtxThreads, kVtxSmemBytes, stream, ws, algo));
  if (le != cudaSuccess) return le;
  return cudaGetLastError();
}

}  // namespace pixgpu
