// Layout of the compact per-event result region (shared by the packing
// kernel and the host API).
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace pixgpu {

constexpr uint32_t kResultTracks = 16384;  // loose tracks kept per event (PU 250: ~11k)
constexpr uint32_t kResultVertices = 1024;
constexpr uint32_t kFlagResultOverflow = 1u << 16;

struct ResultHeader {
  uint32_t nTracks, nLooseAll, nVertices, nHits, nTuples, nDigis, nCells, flags;
  uint32_t nEdges, nTupleHits, nModules;
  uint32_t nearDoublet, nearCA, nearQuality;  // cut decisions on their float boundary
  uint32_t pad[2];
};
constexpr size_t kResultTrackBytes = 4 + 1 + 1 + 20 + 60 + 4 + 4 + 4 + 20 + 2;  // per stored track
constexpr size_t kResultVertexBytes = 4 + 4 + 4 + 4 + 4 + 2;                   // per stored vertex

struct ResultTracks {
  uint32_t* tupleIndex;
  uint8_t* nHits;
  uint8_t* quality;
  float* state;   // [n][5]
  float* cov;     // [n][15]
  float *pt, *eta, *chi2;
  uint32_t* hits;  // [n][5]
  int16_t* vertex;
};

struct ResultVertices {
  float *zv, *wv, *chi2, *ptv2;
  int32_t* ndof;
  uint16_t* sortInd;
};

constexpr size_t kResOffTupleIndex = 64;
constexpr size_t kResOffNHits = kResOffTupleIndex + 4 * size_t(kResultTracks);
constexpr size_t kResOffQuality = kResOffNHits + kResultTracks;
constexpr size_t kResOffState = kResOffQuality + kResultTracks;
constexpr size_t kResOffCov = kResOffState + 4 * 5 * size_t(kResultTracks);
constexpr size_t kResOffPt = kResOffCov + 4 * 15 * size_t(kResultTracks);
constexpr size_t kResOffEta = kResOffPt + 4 * size_t(kResultTracks);
constexpr size_t kResOffChi2 = kResOffEta + 4 * size_t(kResultTracks);
constexpr size_t kResOffHits = kResOffChi2 + 4 * size_t(kResultTracks);
constexpr size_t kResOffVertex = kResOffHits + 4 * 5 * size_t(kResultTracks);
constexpr size_t kResOffZv = kResOffVertex + 2 * size_t(kResultTracks);
constexpr size_t kResOffWv = kResOffZv + 4 * size_t(kResultVertices);
constexpr size_t kResOffVchi2 = kResOffWv + 4 * size_t(kResultVertices);
constexpr size_t kResOffPtv2 = kResOffVchi2 + 4 * size_t(kResultVertices);
constexpr size_t kResOffNdof = kResOffPtv2 + 4 * size_t(kResultVertices);
constexpr size_t kResOffSortInd = kResOffNdof + 4 * size_t(kResultVertices);
constexpr size_t kResultStride = ((kResOffSortInd + 2 * size_t(kResultVertices)) + 4095) & ~size_t(4095);

#ifdef __CUDACC__
#define PG_HD __host__ __device__
#else
#define PG_HD
#endif

PG_HD inline ResultTracks resultTracks(uint8_t* base) {
  ResultTracks t;
  t.tupleIndex = reinterpret_cast<uint32_t*>(base + kResOffTupleIndex);
  t.nHits = base + kResOffNHits;
  t.quality = base + kResOffQuality;
  t.state = reinterpret_cast<float*>(base + kResOffState);
  t.cov = reinterpret_cast<float*>(base + kResOffCov);
  t.pt = reinterpret_cast<float*>(base + kResOffPt);
  t.eta = reinterpret_cast<float*>(base + kResOffEta);
  t.chi2 = reinterpret_cast<float*>(base + kResOffChi2);
  t.hits = reinterpret_cast<uint32_t*>(base + kResOffHits);
  t.vertex = reinterpret_cast<int16_t*>(base + kResOffVertex);
  return t;
}

PG_HD inline ResultVertices resultVertices(uint8_t* base) {
  ResultVertices v;
  v.zv = reinterpret_cast<float*>(base + kResOffZv);
  v.wv = reinterpret_cast<float*>(base + kResOffWv);
  v.chi2 = reinterpret_cast<float*>(base + kResOffVchi2);
  v.ptv2 = reinterpret_cast<float*>(base + kResOffPtv2);
  v.ndof = reinterpret_cast<int32_t*>(base + kResOffNdof);
  v.sortInd = reinterpret_cast<uint16_t*>(base + kResOffSortInd);
  return v;
}

}  // namespace pixgpu
