// Oracle (checker only): pixel vertexing, restating
// plugin-PixelVertexFinding/gpuVertexFinderImpl.h:10-43 (loadTracks),
// gpuClusterTracksByDensity.h:20-207 (or, configured,
// gpuClusterTracksDBSCAN.h:16-227 / gpuClusterTracksIterative.h:16-201; the
// choice of gpuVertexFinderImpl.h:96-102), gpuFitVertices.h:15-98,
// gpuSplitVertices.h:15-125 and gpuSortByPt2.h:15-55 with the
// PixelVertexProducerCUDA configuration (PixelVertexProducerCUDA.cc:16-26):
// minT=2, eps=0.07, errmax=0.01, chi2max=9, ptMin=0.5.  See oracle.h.
#include <stdexcept>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>

#include "oracle.h"

namespace oracle {

void makeVertices(const CA& ca, Vertices& v, int algo) {
  // the TrackSoA stride (32768 in the reference, ZVertexSoA.h:11)
  const uint32_t MAXTRACKS = ca.tupleBins;
  constexpr uint32_t MAXVTX = PF_MAX_VTX;
  const int minT = 2;
  const float eps = 0.07f, errmax = 0.01f, chi2max = 9.f, ptMin = 0.5f;
  v.nvFinal = 0;
  v.zv.assign(MAXVTX, 0.f);
  v.wv.assign(MAXVTX, 0.f);
  v.chi2.assign(MAXVTX, 0.f);
  v.ptv2.assign(MAXVTX, 0.f);
  v.ndof.assign(MAXTRACKS, 0);
  v.sortInd.assign(MAXVTX, 0);
  v.idv.assign(MAXTRACKS, 0);

  // ---- loadTracks (quality loose, nHits >= 4, pt >= ptMin)
  std::vector<uint32_t> itrk;
  std::vector<float> zt, ezt2, ptt2;
  for (uint32_t idx = 0; idx < MAXTRACKS; ++idx) {
    uint32_t nHits = ca.size(idx);
    if (nHits == 0) break;
    v.idv[idx] = -1;
    if (nHits < 4) continue;
    if (ca.quality[idx] != 2) continue;
    float pt = ca.pt[idx];
    if (pt < ptMin) continue;
    itrk.push_back(idx);
    zt.push_back(ca.state[size_t(idx) * 5 + 4]);
    ezt2.push_back(ca.cov[size_t(idx) * 15 + 14]);
    ptt2.push_back(pt * pt);
  }
  const uint32_t nt = uint32_t(itrk.size());
  // ZVertexSoA::MAXTRACKS (ZVertexSoA.h:11): the reference writes past its arrays beyond it
  if (nt > 32 * 1024) throw std::runtime_error("undefined in the reference: more than 32768 vertex tracks");
  std::vector<int32_t> iv(nt);
  int32_t* nn = v.ndof.data();
  uint32_t nvIntermediate = 0;

  // ---- clustering: histogram common to the three algorithms
  {
    float er2mx = errmax * errmax;
    std::vector<uint8_t> izt(nt);
    std::vector<uint32_t> off(257, 0);
    for (uint32_t i = 0; i < nt; ++i) {
      int iz = int(zt[i] * 10.);
      iz = std::min(std::max(iz, INT8_MIN), INT8_MAX);
      izt[i] = uint8_t(iz - INT8_MIN);
      off[izt[i]]++;
      iv[i] = int32_t(i);
      nn[i] = 0;
    }
    for (int b = 1; b < 257; ++b) off[b] += off[b - 1];
    std::vector<uint32_t> bins(nt);
    for (uint32_t i = 0; i < nt; ++i) {
      uint32_t w = off[izt[i]]--;
      bins[w - 1] = i;
    }
    // forEachInBins(hist, izt[i], 1, f): bins izt-1 .. izt+1, in storage order
    auto forEach = [&](uint32_t i, auto&& f) {
      int bs = izt[i];
      int be = std::min(255, bs + 1);
      bs = std::max(0, bs - 1);
      for (uint32_t p = off[bs]; p < off[be + 1]; ++p) f(uint32_t(bins[p]));
    };
    // neighbour counts (DBSCAN: no chi2 compatibility)
    for (uint32_t i = 0; i < nt; ++i) {
      if (ezt2[i] > er2mx) continue;
      forEach(i, [&](uint32_t j) {
        if (i == j) return;
        float dist = std::abs(zt[i] - zt[j]);
        if (dist > eps) return;
        if (algo != 1 && dist * dist > chi2max * (ezt2[i] + ezt2[j])) return;
        nn[i]++;
      });
    }
    auto percolate = [&]() {
      for (uint32_t i = 0; i < nt; ++i) {
        int32_t m = iv[i];
        while (m != iv[m]) m = iv[m];
        iv[i] = m;
      }
    };
    // DBSCAN/Iterative edge rule: a non-core track joins its closest
    // chi2-compatible core neighbour
    auto edges = [&]() {
      for (uint32_t i = 0; i < nt; ++i) {
        if (nn[i] >= minT) continue;
        float mdist = eps;
        forEach(i, [&](uint32_t j) {
          if (nn[j] < minT) return;
          float dist = std::abs(zt[i] - zt[j]);
          if (dist > mdist) return;
          if (dist * dist > chi2max * (ezt2[i] + ezt2[j])) return;
          mdist = dist;
          iv[i] = iv[j];
        });
      }
    };
    if (algo == 0) {  // gpuClusterTracksByDensity.h:20-207: closest denser neighbour
      for (uint32_t i = 0; i < nt; ++i) {
        float mdist = eps;
        forEach(i, [&](uint32_t j) {
          if (nn[j] < nn[i]) return;
          if (nn[j] == nn[i] && zt[j] >= zt[i]) return;
          float dist = std::abs(zt[i] - zt[j]);
          if (dist > mdist) return;
          if (dist * dist > chi2max * (ezt2[i] + ezt2[j])) return;
          mdist = dist;
          iv[i] = int32_t(j);
        });
      }
      percolate();
    } else if (algo == 1) {  // gpuClusterTracksDBSCAN.h:16-227: core links to the lowest-z core neighbour
      for (uint32_t i = 0; i < nt; ++i) {
        if (nn[i] < minT) continue;
        float mz = zt[i];
        forEach(i, [&](uint32_t j) {
          if (zt[j] >= mz) return;
          if (nn[j] < minT) return;
          float dist = std::abs(zt[i] - zt[j]);
          if (dist > eps) return;
          mz = zt[j];
          iv[i] = int32_t(j);
        });
      }
      percolate();
      edges();
    } else {  // gpuClusterTracksIterative.h:16-201: min-label propagation over compatible cores
      int nloops = 0;
      bool more = true;
      while (more) {
        if (1 == nloops % 2) {
          percolate();
        } else {
          more = false;
          for (uint32_t k = 0; k < nt; ++k) {
            const uint32_t i = bins[k];
            const int be = std::min(int(izt[i]) + 1, 255);
            if (nn[i] < minT) continue;
            for (uint32_t p = k + 1; p < off[be + 1]; ++p) {
              const uint32_t j = bins[p];
              if (nn[j] < minT) continue;
              float dist = std::abs(zt[i] - zt[j]);
              if (dist > eps) continue;
              if (dist * dist > chi2max * (ezt2[i] + ezt2[j])) continue;
              const int32_t old = iv[j];  // the serial atomicMin
              if (iv[i] < old) iv[j] = iv[i];
              if (old != iv[i]) more = true;
              if (old < iv[i]) iv[i] = old;
            }
          }
        }
        ++nloops;
      }
      edges();
    }
    uint32_t found = 0;
    for (uint32_t i = 0; i < nt; ++i) {
      if (iv[i] == int32_t(i)) {
        if (nn[i] >= minT)
          iv[i] = -int32_t(found++ + 1);
        else
          iv[i] = -9998;
      }
    }
    for (uint32_t i = 0; i < nt; ++i)
      if (iv[i] >= 0) iv[i] = iv[iv[i]];
    for (uint32_t i = 0; i < nt; ++i) iv[i] = -iv[i] - 1;
    nvIntermediate = v.nvFinal = found;
  }

  // ---- fitVertices
  auto fit = [&](float chi2Max) {
    v.nvFinal = nvIntermediate;
    uint32_t found = v.nvFinal;
    for (uint32_t i = 0; i < found; ++i) {
      v.zv[i] = 0;
      v.wv[i] = 0;
      v.chi2[i] = 0;
    }
    for (uint32_t i = 0; i < nt; ++i) {
      if (iv[i] > 9990) continue;
      float w = 1.f / ezt2[i];
      v.zv[iv[i]] += zt[i] * w;
      v.wv[iv[i]] += w;
    }
    for (uint32_t i = 0; i < found; ++i) {
      v.zv[i] /= v.wv[i];
      nn[i] = -1;
    }
    for (uint32_t i = 0; i < nt; ++i) {
      if (iv[i] > 9990) continue;
      float c2 = v.zv[iv[i]] - zt[i];
      c2 *= c2 / ezt2[i];
      if (c2 > chi2Max) {
        iv[i] = 9999;
        continue;
      }
      v.chi2[iv[i]] += c2;
      nn[iv[i]]++;
    }
    for (uint32_t i = 0; i < found; ++i)
      if (nn[i] > 0) v.wv[i] *= float(nn[i]) / v.chi2[i];
  };
  fit(50.f);

  // ---- splitVertices (maxChi2 = 9)
  {
    const float maxChi2 = 9.f;
    constexpr int MAXTK = 512;
    std::vector<uint32_t> it(MAXTK);
    std::vector<float> zz(MAXTK), ww(MAXTK);
    std::vector<uint8_t> newV(MAXTK);
    for (uint32_t kv = 0; kv < v.nvFinal; ++kv) {
      if (nn[kv] < 4) continue;
      if (v.chi2[kv] < maxChi2 * float(nn[kv])) continue;
      if (nn[kv] >= MAXTK) continue;
      uint32_t nq = 0;
      for (uint32_t k = 0; k < nt; ++k) {
        if (iv[k] == int32_t(kv)) {
          uint32_t old = nq;
          if (nq < uint32_t(MAXTK)) ++nq;
          zz[old] = zt[k] - v.zv[kv];
          newV[old] = zz[old] < 0 ? 0 : 1;
          ww[old] = 1.f / ezt2[k];
          it[old] = k;
        }
      }
      float znew[2], wnew[2];
      int maxiter = 20;
      bool more = true;
      while (more) {
        more = false;
        znew[0] = znew[1] = 0;
        wnew[0] = wnew[1] = 0;
        for (uint32_t k = 0; k < nq; ++k) {
          int i = newV[k];
          znew[i] += zz[k] * ww[k];
          wnew[i] += ww[k];
        }
        znew[0] /= wnew[0];
        znew[1] /= wnew[1];
        for (uint32_t k = 0; k < nq; ++k) {
          float d0 = std::abs(zz[k] - znew[0]);
          float d1 = std::abs(zz[k] - znew[1]);
          int newer = d0 < d1 ? 0 : 1;
          more |= newer != newV[k];
          newV[k] = uint8_t(newer);
        }
        --maxiter;
        if (maxiter <= 0) more = false;
      }
      if (0 == wnew[0] || 0 == wnew[1]) continue;
      float dist2 = (znew[0] - znew[1]) * (znew[0] - znew[1]);
      float chi2Dist = dist2 / (1.f / wnew[0] + 1.f / wnew[1]);
      if (chi2Dist < 4) continue;
      uint32_t igv = nvIntermediate++;
      for (uint32_t k = 0; k < nq; ++k)
        if (1 == newV[k]) iv[it[k]] = int32_t(igv);
    }
  }
  fit(5000.f);

  // ---- sortByPt2 (stable for equal pt^2; the reference uses std::sort)
  if (v.nvFinal < 1) return;
  for (uint32_t i = 0; i < nt; ++i) v.idv[itrk[i]] = int16_t(iv[i]);
  for (uint32_t i = 0; i < v.nvFinal; ++i) v.ptv2[i] = 0;
  for (uint32_t i = 0; i < nt; ++i) {
    if (iv[i] > 9990) continue;
    v.ptv2[iv[i]] += ptt2[i];
  }
  if (1 == v.nvFinal) {
    v.sortInd[0] = 0;
    return;
  }
  for (uint16_t i = 0; i < v.nvFinal; ++i) v.sortInd[i] = i;
  std::stable_sort(v.sortInd.begin(), v.sortInd.begin() + v.nvFinal,
                   [&](uint16_t a, uint16_t b) { return v.ptv2[a] < v.ptv2[b]; });
}

}  // namespace oracle
