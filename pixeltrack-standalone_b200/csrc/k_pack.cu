// Result packing and small batch-setup kernels.
//
// kPackResults writes, per event, the compact result that a consumer of the
// chain needs (the role of the PixelTrackSoAFromCUDA / PixelVertexSoAFromCUDA
// transfer modules of the CUDA program): counts, the loose tracks (quality >=
// loose, in tuple order) with their fit state, covariance, hits and vertex
// assignment, and the vertices.  The destination is mapped pinned host memory,
// so the transfer is exact-sized and needs no host synchronisation.
#include "device_utils.cuh"
#include "pixgpu_internal.cuh"
#include "pixgpu_results.h"

namespace pixgpu {

namespace {

__global__ void kSetInput(BatchInput* in, const uint32_t* words, const uint8_t* fedIds) {
  in->words = words;
  in->fedIds = fedIds;
}

__global__ void kPackResults(Workspace ws, uint8_t* out) {
  __shared__ uint32_t scanSh[33];
  __shared__ uint32_t sGuard;
  const uint32_t e = blockIdx.x;
  const EventCounters* c = ws.ev + e;
  uint8_t* base = out + size_t(e) * kResultStride;
  ResultHeader* hdr = reinterpret_cast<ResultHeader*>(base);
  ResultTracks trk = resultTracks(base);
  ResultVertices vtx = resultVertices(base);
  const uint32_t* toff = ws.tupleOff + size_t(e) * (kTupleBins + 1);
  const uint16_t* th = ws.tupleHits + size_t(e) * kTupleHitCap;
  const uint8_t* q = ws.quality + size_t(e) * kTupleBins;
  const size_t tb = size_t(e) * kTupleBins;
  if (threadIdx.x == 0) {
    uint32_t g = c->nTuples;
    if (c->apcM >= kTupleBins) g = kTupleBins - 1;
    sGuard = g;
  }
  __syncthreads();
  const uint32_t guard = sGuard;
  uint32_t carry = 0;
  for (uint32_t t0 = 0; t0 < guard; t0 += blockDim.x) {
    uint32_t t = t0 + threadIdx.x;
    uint32_t loose = (t < guard && q[t] >= 2) ? 1u : 0u;
    uint32_t tot;
    uint32_t pre = blockExclusiveScan(loose, scanSh, &tot);
    uint32_t p = carry + pre;
    if (loose && p < kResultTracks) {
      uint32_t nh = toff[t + 1] - toff[t];
      trk.tupleIndex[p] = t;
      trk.nHits[p] = uint8_t(nh);
      trk.quality[p] = q[t];
      for (int k = 0; k < 5; ++k) trk.state[5 * p + k] = ws.state[tb * 5 + size_t(t) * 5 + k];
      for (int k = 0; k < 15; ++k) trk.cov[15 * p + k] = ws.cov[tb * 15 + size_t(t) * 15 + k];
      trk.pt[p] = ws.pt[tb + t];
      trk.eta[p] = ws.eta[tb + t];
      trk.chi2[p] = ws.chi2[tb + t];
      for (uint32_t k = 0; k < 5; ++k) trk.hits[5 * p + k] = k < nh ? th[toff[t] + k] : uint16_t(0xffff);
      trk.vertex[p] = c->nVertices > 0 ? ws.idv[tb + t] : int16_t(-1);
    }
    carry += tot;
  }
  const uint32_t nv = min(c->nVertices, uint32_t(kMaxVtx));
  const size_t vb = size_t(e) * kMaxVtx;
  for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) {
    vtx.zv[v] = ws.zv[vb + v];
    vtx.wv[v] = ws.wv[vb + v];
    vtx.chi2[v] = ws.vchi2[vb + v];
    vtx.ptv2[v] = ws.ptv2[vb + v];
    vtx.ndof[v] = ws.ndof[vb + v];
    vtx.sortInd[v] = ws.sortInd[vb + v];
  }
  if (threadIdx.x == 0) {
    hdr->nTracks = min(carry, kResultTracks);
    hdr->nLooseAll = carry;
    hdr->nVertices = nv;
    hdr->nHits = c->nHits;
    hdr->nTuples = guard;
    hdr->nDigis = c->nWords;
    hdr->nCells = c->nCells;
    hdr->flags = c->flags | (carry > kResultTracks ? kFlagResultOverflow : 0u);
    hdr->nEdges = c->nEdges;
    hdr->nTupleHits = toff[guard];
    hdr->nModules = c->nModules;
  }
}

}  // namespace

void launchSetInput(Workspace& ws, const uint32_t* words, const uint8_t* fedIds, cudaStream_t s) {
  PG_PROBED("kSetInput", s, kSetInput<<<1, 1, 0, s>>>(ws.input, words, fedIds));
}

void launchPack(Workspace& ws, uint32_t nEvents, uint8_t* out, cudaStream_t s) {
  PG_PROBED("kPackResults", s, kPackResults<<<nEvents, 256, 0, s>>>(ws, out));
}

}  // namespace pixgpu
