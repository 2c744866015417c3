// Oracle (checker only): doublets, CA connect, fishbone, n-tuplet search,
// duplicate removal, fits and classification (plugin-PixelTriplets/*).
// See oracle.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <stdexcept>

#include "oracle.h"

namespace oracle {

namespace {

// gpuPixelDoublets.h:14-66 (19 layer pairs and their cuts)
constexpr int kNPairs = 19;
constexpr uint8_t kLayerPairs[2 * kNPairs] = {0, 1, 0, 4, 0, 7, 1, 2, 1, 4, 1, 7, 4, 5, 7, 8, 2, 3, 2, 4,
                                             2, 7, 5, 6, 8, 9, 0, 2, 1, 3, 0, 5, 0, 8, 4, 6, 7, 9};
constexpr int16_t kPhi0p05 = 522, kPhi0p06 = 626, kPhi0p07 = 730;
constexpr int16_t kPhiCuts[kNPairs] = {kPhi0p05, kPhi0p07, kPhi0p07, kPhi0p05, kPhi0p06, kPhi0p06, kPhi0p05,
                                       kPhi0p05, kPhi0p06, kPhi0p06, kPhi0p06, kPhi0p05, kPhi0p05, kPhi0p05,
                                       kPhi0p05, kPhi0p05, kPhi0p05, kPhi0p05, kPhi0p05};
constexpr float kMinZ[kNPairs] = {-20., 0., -30., -22., 10., -30., -70., -70., -22., 15.,
                                  -30,  -70., -70., -20., -22., 0,   -30., -70., -70.};
constexpr float kMaxZ[kNPairs] = {20., 30., 0., 22., 30., -10., 70., 70., 22., 30.,
                                  -15., 70., 70., 20., 22., 30., 0., 70., 70.};
constexpr float kMaxR[kNPairs] = {20., 9., 9., 20., 7., 7., 5., 5., 20., 6., 6., 5., 5., 20., 20., 9., 9., 9., 9.};

// CAHitNtupletGeneratorOnGPU.cc:45-65 (module configuration; the switches are
// CAParams, the container capacities CAParams::caps)
constexpr float kPtMin = 0.899999976158f;
constexpr float kThetaCutBarrel = 0.00200000009499f;
constexpr float kThetaCutForward = 0.00300000002608f;
constexpr float kHardCurvCut = 0.0328407224959f;
constexpr float kDcaCutInner = 0.15000000596f;
constexpr float kDcaCutOuter = 0.25f;

constexpr uint8_t kBad = 0, kDup = 1, kLoose = 2;

// DataFormats/approx_atan2.h:459-462 short2phi
inline float short2phi(short x) {
  constexpr float i2p = M_PI / (int(std::numeric_limits<short>::max()) + 1);
  return float(x) * i2p;
}

inline uint32_t phiBin(int16_t t) { return uint32_t((int(t) >> 9) & 127); }

// GPUCACell.h:175-185; fabs(float) resolves to the double overload in the serial build
bool areAlignedRZ(float r1, float z1, float ri, float zi, float ro, float zo, float ptmin, float thetaCut,
                  uint32_t* near) {
  float radius_diff = std::abs(r1 - ro);
  float distance_13_squared = radius_diff * radius_diff + (z1 - zo) * (z1 - zo);
  float pMin = ptmin * std::sqrt(distance_13_squared);
  double tan_12_13_half_mul_distance_13_squared = ::fabs(double(z1 * (ri - ro) + zi * (ro - r1) + zo * (r1 - ri)));
  const double lhs = tan_12_13_half_mul_distance_13_squared * pMin;
  const double rhs = double(thetaCut * distance_13_squared * radius_diff);
  *near += cutNear(lhs, rhs);
  return lhs <= rhs;
}

// CircleEq.h:23-107 (float), dca0 and curvature
struct Circle {
  float xp, yp, c, alpha, beta;
};
Circle circleEq(float x1, float y1, float x2, float y2, float x3, float y3) {
  bool noflip = std::abs(x3 - x1) < std::abs(y3 - y1);
  float x1p = noflip ? x1 - x2 : y1 - y2;
  float y1p = noflip ? y1 - y2 : x1 - x2;
  float d12 = x1p * x1p + y1p * y1p;
  float x3p = noflip ? x3 - x2 : y3 - y2;
  float y3p = noflip ? y3 - y2 : x3 - x2;
  float d32 = x3p * x3p + y3p * y3p;
  float num = x1p * y3p - y1p * x3p;
  float det = d12 * y3p - d32 * y1p;
  float st2 = (d12 * x3p - d32 * x1p);
  float seq = det * det + st2 * st2;
  float al2 = 1.f / std::sqrt(seq);
  float be2 = -st2 * al2;
  float ct = 2.f * num * al2;
  al2 *= det;
  Circle e;
  e.xp = x2;
  e.yp = y2;
  e.c = noflip ? ct : -ct;
  e.alpha = noflip ? al2 : -be2;
  e.beta = noflip ? be2 : -al2;
  return e;
}
inline float dca0(const Circle& e) {
  float x = e.c * e.xp + e.alpha;
  float y = e.c * e.yp + e.beta;
  return std::sqrt(x * x + y * y) - 1.f;
}

}  // namespace

void makeTuples(const ES& es, const Hits& hh, CA& ca, const CAParams& prm) {
  const bool useRiemannFit = prm.useRiemannFit;
  const Caps& caps = prm.caps;
  const uint32_t kTupleBins = caps.tuples;
  // "no tuple" in the duplicate removers (the reference's 60000 lies above
  // every tuple index of its 32768 bins; 32-bit indices need a larger one)
  constexpr uint32_t kNoTuple = 0xffffffffu;
  const int nPairs = prm.nPairs();
  const uint32_t nHits = hh.nHits;
  // ---- allocateOnGPU / launchZero (CAHitNtupletGeneratorKernelsAlloc.h:4-25) and tuples zero
  ca.nCells = 0;
  ca.inner.clear();
  ca.outer.clear();
  ca.used.clear();
  ca.layerPair.clear();
  ca.doubletId.clear();
  ca.innerZ.clear();
  ca.innerR.clear();
  ca.outerHitCells.assign(std::max(1u, nHits), {});
  ca.nbr.clear();
  ca.trk.clear();
  ca.nbrPool = 1;
  ca.trkPool = 1;
  ca.apcM = ca.apcN = 0;
  ca.nearDoublet = ca.nearCA = ca.nearQuality = 0;
  ca.tupleBins = kTupleBins;
  ca.tupleOff.assign(kTupleBins + 1, 0);
  ca.tupleHits.assign(5 * kTupleBins, 0);
  ca.tupleDet.assign(5 * kTupleBins, 0);
  ca.quality.assign(kTupleBins, 0);
  ca.tmOff.assign(9, 0);
  ca.tmBins.assign(caps.multiplicity, 0);
  ca.state.assign(size_t(kTupleBins) * 5, 0.f);
  ca.cov.assign(size_t(kTupleBins) * 15, 0.f);
  ca.pt.assign(kTupleBins, 0.f);
  ca.eta.assign(kTupleBins, 0.f);
  ca.chi2.assign(kTupleBins, 0.f);

  // ---- buildDoublets: doubletsFromHisto (gpuPixelDoubletsAlgos.h:25-238)
  if (nHits) {
    const uint32_t* offsets = hh.layerStart;
    auto layerSize = [&](uint8_t li) { return offsets[li + 1] - offsets[li]; };
    uint32_t cum[kNPairs];
    cum[0] = layerSize(kLayerPairs[0]);
    for (int i = 1; i < nPairs; ++i) cum[i] = cum[i - 1] + layerSize(kLayerPairs[2 * i]);
    const uint32_t ntot = cum[nPairs - 1];
    constexpr int minYsizeB1 = 36, minYsizeB2 = 28, maxDYsize12 = 28, maxDYsize = 20, maxDYPred = 20;
    constexpr float dzdrFact = 8 * 0.0285 / 0.015;
    constexpr float z0cut = 12.f;
    constexpr float hardPtCut = 0.5f;
    constexpr float minRadius = hardPtCut * 87.78f;
    constexpr float minRadius2T4 = 4.f * minRadius * minRadius;
    uint32_t pairLayerId = 0;
    for (uint32_t j = 0; j < ntot; ++j) {
      while (j >= cum[pairLayerId++])
        ;
      --pairLayerId;
      uint8_t inner = kLayerPairs[2 * pairLayerId], outer = kLayerPairs[2 * pairLayerId + 1];
      uint32_t i = (0 == pairLayerId) ? j : j - cum[pairLayerId - 1];
      i += offsets[inner];
      uint16_t mi = hh.detInd[i];
      if (mi > 2000) continue;
      float mez = hh.zg[i];
      ca.nearDoublet += cutNear(mez, kMinZ[pairLayerId]) + cutNear(mez, kMaxZ[pairLayerId]);
      if (mez < kMinZ[pairLayerId] || mez > kMaxZ[pairLayerId]) continue;
      int16_t mes = -1;
      if (prm.doClusterCut) {
        // gpuPixelDoubletsAlgos.h:120-135: with ideal conditions every ladder counts as outer
        const bool isOuterLadder = prm.idealConditions ? true : 0 == (mi / 8) % 2;
        mes = inner > 0 || isOuterLadder ? hh.ysize[i] : int16_t(-1);
        if (inner == 0 && outer > 3)
          if (mes > 0 && mes < minYsizeB1) continue;
        if (inner == 1 && outer > 3)
          if (mes > 0 && mes < minYsizeB2) continue;
      }
      int16_t mep = hh.iphi[i];
      float mer = hh.rg[i];
      int16_t iphicut = kPhiCuts[pairLayerId];
      uint32_t kl = phiBin(int16_t(mep - iphicut)), kh = phiBin(int16_t(mep + iphicut));
      uint32_t hoff = 128 * outer;
      uint32_t khh = (kh + 1) % 128;
      for (uint32_t kk = kl; kk != khh; kk = (kk + 1) % 128) {
        uint32_t b = kk + hoff;
        for (uint32_t p = hh.phiOff[b]; p < hh.phiOff[b + 1]; ++p) {
          uint32_t oi = hh.phiBins[p];
          uint16_t mo = hh.detInd[oi];
          if (mo > 2000) continue;
          // z0cutoff
          if (prm.doZ0Cut) {
            float zo = hh.zg[oi], ro = hh.rg[oi];
            float dr = ro - mer;
            ca.nearDoublet += cutNear(dr, kMaxR[pairLayerId]);
            if (dr > kMaxR[pairLayerId] || dr < 0) continue;
            ca.nearDoublet += cutNear(std::abs((mez * ro - mer * zo)), z0cut * dr);
            if (std::abs((mez * ro - mer * zo)) > z0cut * dr) continue;
          }
          int16_t mop = hh.iphi[oi];
          uint16_t idphi = uint16_t(std::min(std::abs(int16_t(mop - mep)), std::abs(int16_t(mep - mop))));
          if (idphi > iphicut) continue;
          // zsizeCut
          if (prm.doClusterCut) {
            bool onlyBarrel = outer < 4;
            int16_t so = hh.ysize[oi];
            int dy = inner == 0 ? maxDYsize12 : maxDYsize;
            float zo = hh.zg[oi], ro = hh.rg[oi];
            bool cut = onlyBarrel ? (mes > 0 && so > 0 && std::abs(so - mes) > dy)
                                  : ((inner < 4) && mes > 0 &&
                                     std::abs(mes - int(std::abs((mez - zo) / (mer - ro)) * dzdrFact + 0.5f)) > maxDYPred);
            if (cut) continue;
          }
          // ptcut
          if (prm.doPtCut) {
            float ri = mer, ro = hh.rg[oi];
            float dphi = short2phi(short(idphi));
            ca.nearDoublet += cutNear(dphi * dphi * (minRadius2T4 - ri * ro), (ro - ri) * (ro - ri));
            if (dphi * dphi * (minRadius2T4 - ri * ro) > (ro - ri) * (ro - ri)) continue;
          }
          uint32_t ind = ca.nCells;
          // full container: the reference leaves the bin (break), storing
          // nothing more; the candidates are still tested here so that the
          // cut-margin count covers every candidate of the windows (the
          // stored doublets are the same)
          if (ind >= caps.doublets) continue;
          ca.nCells++;
          ca.inner.push_back(i);
          ca.outer.push_back(oi);
          ca.layerPair.push_back(int16_t(pairLayerId));
          ca.doubletId.push_back(int32_t(ind));
          ca.used.push_back(0);
          ca.innerZ.push_back(hh.zg[i]);
          ca.innerR.push_back(hh.rg[i]);
          if (ca.outerHitCells[oi].size() < PF_MAX_CELLS_PER_HIT) ca.outerHitCells[oi].push_back(ind);
        }
      }
    }
  }
  const uint32_t nCells = ca.nCells;
  ca.nbr.assign(nCells, {});
  ca.trk.assign(nCells, {});
  std::vector<uint8_t> hasNbrList(nCells, 0), hasTrkList(nCells, 0);

  // ---- kernel_connect (CAHitNtupletGeneratorKernelsImpl.h:191-262)
  for (uint32_t idx = 0; idx < nCells; ++idx) {
    uint32_t innerHit = ca.inner[idx];
    const auto& vi = ca.outerHitCells[innerHit];
    float ri = ca.innerR[idx], zi = ca.innerZ[idx];
    float ro = hh.rg[ca.outer[idx]], zo = hh.zg[ca.outer[idx]];
    bool isBarrel = float(hh.detInd[innerHit]) < 1184;
    for (uint32_t oc : vi) {
      float r1 = ca.innerR[oc], z1 = ca.innerZ[oc];
      bool aligned =
          areAlignedRZ(r1, z1, ri, zi, ro, zo, kPtMin, isBarrel ? kThetaCutBarrel : kThetaCutForward, &ca.nearCA);
      if (!aligned) continue;
      // GPUCACell::dcaCut (GPUCACell.h:187-206)
      float x1 = hh.xg[ca.inner[oc]], y1 = hh.yg[ca.inner[oc]];
      float x2 = hh.xg[innerHit], y2 = hh.yg[innerHit];
      float x3 = hh.xg[ca.outer[idx]], y3 = hh.yg[ca.outer[idx]];
      float region = float(hh.detInd[ca.inner[oc]]) < 96 ? kDcaCutInner : kDcaCutOuter;
      Circle eq = circleEq(x1, y1, x2, y2, x3, y3);
      ca.nearCA += cutNear(eq.c, kHardCurvCut);
      if (eq.c > kHardCurvCut) continue;
      ca.nearCA += cutNear(std::abs(dca0(eq)), region * std::abs(eq.c));
      if (!(std::abs(dca0(eq)) < region * std::abs(eq.c))) continue;
      // GPUCACell::addOuterNeighbor (GPUCACell.h:67-86): pool of maxNumOfActiveDoublets lists
      if (ca.nbr[oc].empty() && !hasNbrList[oc]) {
        if (ca.nbrPool < int32_t(caps.lists)) {
          ca.nbrPool++;
          hasNbrList[oc] = 1;
        }
      }
      if (hasNbrList[oc] && ca.nbr[oc].size() < PF_MAX_CELL_NEIGHBORS) ca.nbr[oc].push_back(idx);
      ca.used[idx] |= 1;
      ca.used[oc] |= 1;
    }
  }

  // ---- fishbone (gpuFishbone.h:21-90): early (after connect) with checkTrack
  //      false, late (after the multiplicity fill) with checkTrack true, which
  //      skips cells that are on no n-tuplet (CAHitNtupletGeneratorKernels.cc:101-134)
  auto fishbone = [&](bool checkTrack) {
    std::vector<float> x, y, z, n;
    std::vector<uint16_t> d;
    std::vector<uint32_t> cc;
    for (uint32_t idy = 0; idy < nHits; ++idy) {
      const auto& vc = ca.outerHitCells[idy];
      uint32_t s = uint32_t(vc.size());
      if (s < 2) continue;
      float xo = hh.xg[ca.outer[vc[0]]], yo = hh.yg[ca.outer[vc[0]]], zo = hh.zg[ca.outer[vc[0]]];
      x.clear(); y.clear(); z.clear(); n.clear(); d.clear(); cc.clear();
      for (uint32_t ic = 0; ic < s; ++ic) {
        uint32_t c = vc[ic];
        if (0 == ca.used[c]) continue;
        if (checkTrack && ca.trk[c].empty()) continue;
        cc.push_back(c);
        d.push_back(uint16_t(float(hh.detInd[ca.inner[c]])));
        float xx = hh.xg[ca.inner[c]] - xo, yy = hh.yg[ca.inner[c]] - yo, zz = ca.innerZ[c] - zo;
        x.push_back(xx);
        y.push_back(yy);
        z.push_back(zz);
        n.push_back(xx * xx + yy * yy + zz * zz);
      }
      uint32_t sg = uint32_t(cc.size());
      if (sg < 2) continue;
      for (uint32_t ic = 0; ic + 1 < sg; ++ic) {
        for (uint32_t jc = ic + 1; jc < sg; ++jc) {
          float cos12 = x[ic] * x[jc] + y[ic] * y[jc] + z[ic] * z[jc];
          if (d[ic] != d[jc] && cos12 * cos12 >= 0.99999f * n[ic] * n[jc]) {
            if (n[ic] > n[jc]) {
              ca.doubletId[cc[ic]] = -1;
              break;
            } else {
              ca.doubletId[cc[jc]] = -1;
            }
          }
        }
      }
    }
  };
  if (nHits > 1 && prm.earlyFishbone) fishbone(false);

  // ---- kernel_find_ntuplets (CAHitNtupletGeneratorKernelsImpl.h:264-292) with
  //      GPUCACell::find_ntuplets<6> (GPUCACell.h:278-331) and bulkFill (HistoContainer.h:181-190)
  uint32_t tmp[6];
  int depth = 0;
  auto addTrack = [&](uint32_t c, uint32_t it) {
    if (ca.trk[c].empty() && !hasTrkList[c]) {
      if (ca.trkPool < int32_t(caps.lists)) {
        ca.trkPool++;
        hasTrkList[c] = 1;
      } else
        return;
    }
    if (hasTrkList[c] && ca.trk[c].size() < PF_MAX_CELL_TRACKS) ca.trk[c].push_back(it);
  };
  std::function<void(uint32_t)> dfs = [&](uint32_t cell) {
    tmp[depth++] = uint32_t(ca.doubletId[cell]);
    if (depth > 4) throw std::runtime_error("find_ntuplets: tuple longer than 5 hits");
    bool last = true;
    for (uint32_t other : ca.nbr[cell]) {
      if (ca.doubletId[other] < 0) continue;
      last = false;
      dfs(other);
    }
    if (last && uint32_t(depth) >= prm.minHitsPerNtuplet - 1) {
      uint32_t hits[6];
      uint32_t nh = 0;
      for (int k = 0; k < depth; ++k) hits[nh++] = ca.inner[tmp[k]];
      hits[nh] = ca.outer[cell];
      uint32_t n = uint32_t(depth) + 1;
      uint32_t m = ca.apcM, off = ca.apcN;
      ca.apcM += 1;
      ca.apcN += n;
      if (m < kTupleBins) {
        ca.tupleOff[m] = off;
        for (uint32_t k = 0; k < n; ++k) ca.tupleHits[off + k] = hits[k];
        for (int k = 0; k < depth; ++k) addTrack(tmp[k], m);
        ca.quality[m] = kBad;
      }
    }
    --depth;
  };
  for (uint32_t idx = 0; idx < nCells; ++idx) {
    if (ca.doubletId[idx] < 0) continue;
    int pid = ca.layerPair[idx];
    bool doit = prm.minHitsPerNtuplet > 3 ? pid < 3 : pid < 8 || pid > 12;
    if (doit) {
      depth = 0;
      dfs(idx);
    }
  }
  // finalizeBulk / bulkFinalizeFill (HistoContainer.h:193-204)
  if (ca.apcM >= kTupleBins) {
    ca.tupleOff[kTupleBins] = ca.tupleOff[kTupleBins - 1];
  } else {
    for (uint32_t i = ca.apcM; i < kTupleBins + 1; ++i) ca.tupleOff[i] = ca.apcN;
  }

  // ---- kernel_earlyDuplicateRemover (Impl.h:118-149)
  for (uint32_t idx = 0; idx < nCells; ++idx) {
    const auto& tr = ca.trk[idx];
    if (tr.size() < 2) continue;
    uint32_t maxNh = 0;
    for (auto it : tr) maxNh = std::max(ca.size(it), maxNh);
    for (auto it : tr)
      if (ca.size(it) != maxNh) ca.quality[it] = kDup;
  }

  // ---- TupleMultiplicity (Impl.h:304-338): counts, scan, fill (descending within a bin)
  for (uint32_t it = 0; it < kTupleBins; ++it) {
    uint32_t nh = ca.size(it);
    if (nh < 3) continue;
    if (ca.quality[it] == kDup) continue;
    ca.tmOff[nh]++;
  }
  for (int b = 1; b < 9; ++b) ca.tmOff[b] += ca.tmOff[b - 1];
  // beyond this capacity the reference writes past TupleMultiplicity::bins
  if (ca.tmOff[8] > caps.multiplicity)
    throw std::runtime_error("undefined in the reference: TupleMultiplicity overflow");
  for (uint32_t it = 0; it < kTupleBins; ++it) {
    uint32_t nh = ca.size(it);
    if (nh < 3) continue;
    if (ca.quality[it] == kDup) continue;
    uint32_t w = ca.tmOff[nh]--;
    ca.tmBins[w - 1] = it;
  }

  if (nHits > 1 && prm.lateFishbone) fishbone(true);

  // ---- fillHitDetIndices (Impl.h:449-464)
  for (uint32_t k = 0; k < ca.tupleOff[kTupleBins]; ++k) ca.tupleDet[k] = hh.detInd[ca.tupleHits[k]];

  if (0 == nHits) return;

  // ---- broken-line fits (BrokenLineFitOnGPU.cc:3-68), or with useRiemannFit
  // the Riemann fits (RiemannFitOnGPU.cc:3-110): N=3, 4, and 5 fitted as 4
  const double B = double(float(0.0114256972711507));
  auto fitBin = [&](uint32_t nHitsBin, int N) {
    uint32_t sz = ca.tmOff[nHitsBin + 1] - ca.tmOff[nHitsBin];
    for (uint32_t local = 0; local < caps.multiplicity; ++local) {
      if (local >= sz) break;
      uint32_t tkid = ca.tmBins[ca.tmOff[nHitsBin] + local];
      double hits[3 * 5];
      float ge[6 * 5];
      const uint32_t* hitId = &ca.tupleHits[ca.tupleOff[tkid]];
      for (int i = 0; i < N; ++i) {
        uint32_t hit = hitId[i];
        const PfFrame& f = es.det[hh.detInd[hit]].frame;
        // SOAFrame::toGlobal(cxx, cxy, cyy, gl) (DataFormats/SOARotation.h:511-519)
        float cxx = hh.xerr[hit], cxy = 0, cyy = hh.yerr[hit];
        float* gl = ge + 6 * i;
        gl[0] = f.R11 * (f.R11 * cxx + f.R21 * cxy) + f.R21 * (f.R11 * cxy + f.R21 * cyy);
        gl[1] = f.R11 * (f.R12 * cxx + f.R22 * cxy) + f.R21 * (f.R12 * cxy + f.R22 * cyy);
        gl[2] = f.R12 * (f.R12 * cxx + f.R22 * cxy) + f.R22 * (f.R12 * cxy + f.R22 * cyy);
        gl[3] = f.R11 * (f.R13 * cxx + f.R23 * cxy) + f.R21 * (f.R13 * cxy + f.R23 * cyy);
        gl[4] = f.R12 * (f.R13 * cxx + f.R23 * cxy) + f.R22 * (f.R13 * cxy + f.R23 * cyy);
        gl[5] = f.R13 * (f.R13 * cxx + f.R23 * cxy) + f.R23 * (f.R13 * cxy + f.R23 * cyy);
        hits[3 * i + 0] = hh.xg[hit];
        hits[3 * i + 1] = hh.yg[hit];
        hits[3 * i + 2] = hh.zg[hit];
      }
      if (useRiemannFit)
        riemannFit(N, hits, ge, B, &ca.state[size_t(tkid) * 5], &ca.cov[size_t(tkid) * 15], &ca.pt[tkid],
                   &ca.eta[tkid], &ca.chi2[tkid]);
      else
        brokenLineFit(N, hits, ge, B, &ca.state[size_t(tkid) * 5], &ca.cov[size_t(tkid) * 15], &ca.pt[tkid],
                      &ca.eta[tkid], &ca.chi2[tkid]);
    }
  };
  fitBin(3, 3);
  fitBin(4, 4);
  fitBin(5, 4);

  // ---- kernel_classifyTracks (Impl.h:340-406) with makeQualityCuts (CAHitNtupletGeneratorOnGPU.cc:21-41)
  const float chi2Coeff[4] = {float(0.68177776), float(0.74609577), float(-0.08035491), float(0.00315399)};
  const float chi2MaxPt = 10.f, chi2Scale = 30.f;
  for (uint32_t it = 0; it < kTupleBins; ++it) {
    uint32_t nh = ca.size(it);
    if (nh == 0) break;
    if (ca.quality[it] == kDup) continue;
    if (nh < 3) continue;
    bool isNaN = false;
    for (int i = 0; i < 5; ++i) isNaN |= std::isnan(ca.state[size_t(it) * 5 + i]);
    if (isNaN) continue;
    float pt = std::min<float>(ca.pt[it], chi2MaxPt);
    float chi2Cut = chi2Scale * (chi2Coeff[0] + pt * (chi2Coeff[1] + pt * (chi2Coeff[2] + pt * chi2Coeff[3])));
    ca.nearQuality += cutNear(3.f * ca.chi2[it], chi2Cut);
    if (3.f * ca.chi2[it] >= chi2Cut) continue;
    float maxTip = nh > 3 ? 0.5f : 0.3f, minPt = nh > 3 ? 0.3f : 0.5f, maxZip = 12.f;
    float tip = ca.state[size_t(it) * 5 + 1], zip = ca.state[size_t(it) * 5 + 4];
    // the three region cuts are all evaluated (their margins counted), then combined
    ca.nearQuality += cutNear(std::abs(tip), maxTip) + cutNear(ca.pt[it], minPt) + cutNear(std::abs(zip), maxZip);
    bool isOk = (std::abs(tip) < maxTip) and (ca.pt[it] > minPt) and (std::abs(zip) < maxZip);
    if (isOk) ca.quality[it] = kLoose;
  }

  // ---- kernel_fishboneCleaner (Impl.h:104-116), with lateFishbone only
  if (prm.lateFishbone)
    for (uint32_t idx = 0; idx < nCells; ++idx)
      if (ca.doubletId[idx] < 0)
        for (auto it : ca.trk[idx]) ca.quality[it] = kBad;

  // ---- kernel_fastDuplicateRemover (Impl.h:151-189): sequential over cells
  for (uint32_t idx = 0; idx < nCells; ++idx) {
    const auto& tr = ca.trk[idx];
    if (tr.size() < 2) continue;
    float mc = 10000.f;
    uint32_t im = kNoTuple;
    for (auto it : tr) {
      float score = std::abs(ca.state[size_t(it) * 5 + 1]);
      if (ca.quality[it] == kLoose && score < mc) {
        mc = score;
        im = it;
      }
    }
    for (auto it : tr)
      if (ca.quality[it] != kBad && it != im) ca.quality[it] = kDup;
  }

  // ---- hit -> tuple map (Impl.h:421-447) and kernel_tripletCleaner (:479-534)
  std::vector<uint32_t> h2tOff(caps.hits + 1, 0);
  std::vector<uint32_t> h2t(caps.hitToTuple, 0);
  for (uint32_t idx = 0; idx < kTupleBins; ++idx) {
    if (ca.size(idx) == 0) break;
    if (ca.quality[idx] != kLoose) continue;
    for (uint32_t k = ca.tupleOff[idx]; k < ca.tupleOff[idx + 1]; ++k) h2tOff[ca.tupleHits[k]]++;
  }
  for (uint32_t b = 1; b < h2tOff.size(); ++b) h2tOff[b] += h2tOff[b - 1];
  if (h2tOff.back() > h2t.size()) throw std::runtime_error("undefined in the reference: HitToTuple overflow");
  for (uint32_t idx = 0; idx < kTupleBins; ++idx) {
    if (ca.size(idx) == 0) break;
    if (ca.quality[idx] != kLoose) continue;
    for (uint32_t k = ca.tupleOff[idx]; k < ca.tupleOff[idx + 1]; ++k) {
      uint32_t w = h2tOff[ca.tupleHits[k]]--;
      h2t[w - 1] = idx;
    }
  }
  for (uint32_t idx = 0; idx < caps.hits; ++idx) {
    uint32_t b = h2tOff[idx], e = h2tOff[idx + 1];
    if (e - b < 2) continue;
    uint32_t maxNh = 0;
    for (uint32_t p = b; p < e; ++p) maxNh = std::max(ca.size(h2t[p]), maxNh);
    for (uint32_t p = b; p < e; ++p)
      if (ca.size(h2t[p]) != maxNh) ca.quality[h2t[p]] = kDup;
    if (maxNh > 3) continue;
    float mc = 10000.f;
    uint32_t im = kNoTuple;
    for (uint32_t p = b; p < e; ++p) {
      uint32_t it = h2t[p];
      float tip = std::abs(ca.state[size_t(it) * 5 + 1]);
      if (ca.quality[it] != kBad && tip < mc) {
        mc = tip;
        im = it;
      }
    }
    for (uint32_t p = b; p < e; ++p) {
      uint32_t it = h2t[p];
      if (ca.quality[it] != kBad && it != im) ca.quality[it] = kDup;
    }
  }
}

}  // namespace oracle
