// Seeded synthetic Phase-1 pixel detector and events (see include/pixsynth.h).
//
// Geometry conventions follow the reference's topology and decoding code so
// that its raw-to-digi, CPE and CA code reconstruct the generated tracks:
//  * module indices and layer boundaries: Geometry/phase1PixelTopology.h:26-36
//    (barrel module = layerStart + 8*ladder + zslot, zslot<4 at z<0, as read by
//    gpuPixelDoubletsAlgos.h:94 and GPUCACell.h hole checks);
//  * raw ids: layer/module/panel bit fields decoded in
//    plugin-SiPixelClusterizer/SiPixelRawToClusterGPUKernel.cc:404-418;
//  * ROC-to-module pixel mapping: the inverse of frameConversion (:72-138);
//  * FED word formats: SiPixelRawToClusterGPUKernel.h:35-72 (layer-1 row/col
//    and DCOL/PXID encodings); S-Link header/trailer: DataFormats/fed_header.h,
//    fed_trailer.h, FEDHeader.cc:25-36, FEDTrailer.cc:29-40;
//  * gain payload addressing: CondFormats/SiPixelGainForHLTonGPU.h:22-45;
//  * pixel pitch/big-pixel local coordinates: phase1PixelTopology.h:142-158.
#include "pixsynth.h"
#include "pixfmt.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;
// 1/(0.3 * 3.8 T) in GeV/cm: the reference's bField (CAHitNtupletCUDA.cc:31)
constexpr double kBField = 0.0114256972711507;
constexpr double kPitchX = 0.01, kPitchY = 0.015;
constexpr double kThickB = 0.0285, kThickE = 0.029;
constexpr double kHalfX = 0.81, kHalfY = 3.24;  // 162 x 432 pitch units
constexpr double kTanLABarrel = 0.1;
constexpr uint32_t kLayerStart[11] = {0, 96, 320, 672, 1184, 1296, 1408, 1520, 1632, 1744, 1856};
constexpr double kBarrelR[4] = {2.9, 6.8, 10.9, 16.0};
constexpr int kLadders[4] = {12, 28, 44, 64};
constexpr double kDiskZ[3] = {32.0, 39.5, 48.5};
constexpr double kRingR[2] = {7.6, 12.8};
constexpr int kRingN[2] = {44, 68};
constexpr int kNFeds = 108;

struct Module {
  int layer;    // 0..9
  bool barrel;
  bool posZ;
  int ladder;   // barrel ladder or endcap module-in-ring
  int zslot;    // barrel 0..7
  int ring;     // endcap 0/1
  int panel;    // endcap 1/2
  double p[3];  // centre
  double ex[3], ey[3], ez[3];
  uint32_t rawId;
  bool frameAB;  // frameConversion branch with ROC<8 at rows 0..79
  int fedIdx, linkA;
  double thick, tanLA;
};

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

}  // namespace

struct ps_detector {
  std::vector<Module> modules;
  std::vector<uint8_t> cabling, gain, cpe, beamspot, fedids;
  std::vector<uint8_t> gainPayload;  // {gain, ped} pairs
  PfGainHeader gainHdr;
  std::vector<uint8_t> badRoc;  // per cabling index
  PfBeamSpot bs;
  std::vector<std::vector<int>> fedModules;
};

struct ps_event {
  std::vector<uint8_t> raw;
  std::vector<float> vz, tpt, teta, tphi;
  std::vector<int32_t> tq, tv;
  std::vector<uint8_t> tnh;
  uint32_t nSimHits = 0, nDigis = 0;
};

namespace {

void buildModules(ps_detector& d) {
  d.modules.resize(PF_N_MODULES);
  for (int L = 0; L < 4; ++L) {
    int nl = kLadders[L];
    for (int l = 0; l < nl; ++l) {
      double phi = 2 * kPi * (l + 0.5) / nl;
      double R = kBarrelR[L] + ((l % 2) ? 0.16 : -0.16);
      for (int k = 0; k < 8; ++k) {
        int idx = kLayerStart[L] + 8 * l + k;
        Module& m = d.modules[idx];
        m.layer = L;
        m.barrel = true;
        m.ladder = l;
        m.zslot = k;
        m.posZ = k >= 4;
        m.ring = 0;
        m.panel = 0;
        double zc = (k - 3.5) * 6.7;
        m.p[0] = R * std::cos(phi);
        m.p[1] = R * std::sin(phi);
        m.p[2] = zc;
        m.ex[0] = -std::sin(phi); m.ex[1] = std::cos(phi); m.ex[2] = 0;
        m.ey[0] = 0; m.ey[1] = 0; m.ey[2] = 1;
        m.ez[0] = std::cos(phi); m.ez[1] = std::sin(phi); m.ez[2] = 0;
        int moduleNum = k + 1;  // 1..8, side = module<5 ? -1 : +1
        m.rawId = (1u << 28) | (1u << 25) | (uint32_t(L + 1) << 20) | (uint32_t(l + 1) << 12) | (uint32_t(moduleNum) << 2);
        int side = moduleNum < 5 ? -1 : 1;
        m.frameAB = (side == -1 && L + 1 != 1);
        m.thick = kThickB;
        m.tanLA = kTanLABarrel;
      }
    }
  }
  for (int e = 0; e < 6; ++e) {
    bool pos = e < 3;
    int disk = e % 3;
    int base = kLayerStart[4 + e];
    int j = 0;
    for (int g = 0; g < 2; ++g) {
      for (int q = 0; q < kRingN[g]; ++q, ++j) {
        Module& m = d.modules[base + j];
        m.layer = 4 + e;
        m.barrel = false;
        m.posZ = pos;
        m.ladder = q;
        m.zslot = 0;
        m.ring = g;
        m.panel = 1 + (q % 2);
        double phi = 2 * kPi * (q + 0.5) / kRingN[g];
        double az = kDiskZ[disk] + (m.panel == 1 ? -0.25 : 0.25) + (g == 1 ? 0.8 : 0.0);
        m.p[0] = kRingR[g] * std::cos(phi);
        m.p[1] = kRingR[g] * std::sin(phi);
        m.p[2] = pos ? az : -az;
        m.ey[0] = std::cos(phi); m.ey[1] = std::sin(phi); m.ey[2] = 0;
        if (pos) {
          m.ex[0] = std::sin(phi); m.ex[1] = -std::cos(phi); m.ex[2] = 0;
          m.ez[0] = 0; m.ez[1] = 0; m.ez[2] = 1;
        } else {
          m.ex[0] = -std::sin(phi); m.ex[1] = std::cos(phi); m.ex[2] = 0;
          m.ez[0] = 0; m.ez[1] = 0; m.ez[2] = -1;
        }
        uint32_t side = pos ? 2 : 1;
        uint32_t blade = g * 40 + q / 2 + 1;
        m.rawId = (1u << 28) | (2u << 25) | (side << 23) | (uint32_t(disk + 1) << 18) | (blade << 12) |
                  (uint32_t(m.panel) << 10) | (1u << 2);
        m.frameAB = true;  // both fpix panels decode with the same branch
        m.thick = kThickE;
        m.tanLA = 0.0;
      }
    }
  }
  // FED assignment: contiguous blocks of modules, two links per module
  d.fedModules.assign(kNFeds, {});
  for (int i = 0; i < PF_N_MODULES; ++i) {
    int f = int((int64_t(i) * kNFeds) / PF_N_MODULES);
    Module& m = d.modules[i];
    m.fedIdx = f;
    m.linkA = 1 + 2 * int(d.fedModules[f].size());
    d.fedModules[f].push_back(i);
  }
}

template <typename T>
void appendPod(std::vector<uint8_t>& v, const T& x) {
  const uint8_t* p = reinterpret_cast<const uint8_t*>(&x);
  v.insert(v.end(), p, p + sizeof(T));
}

void buildES(ps_detector& d, const ps_detector_config& cfg) {
  std::mt19937_64 rng(cfg.seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  // ---- cabling
  auto cab = std::make_unique<PfCablingMap>();
  std::memset(cab.get(), 0, sizeof(PfCablingMap));
  for (int i = 0; i < PF_MAX_SIZE; ++i) {
    cab->rawId[i] = 9999;
    cab->moduleId[i] = 9999;
    cab->rocInDet[i] = 9999;
  }
  uint32_t maxIndex = 0;
  d.badRoc.assign(PF_MAX_SIZE, 0);
  for (int i = 0; i < PF_N_MODULES; ++i) {
    const Module& m = d.modules[i];
    for (int r = 0; r < 16; ++r) {
      uint32_t link = m.linkA + r / 8;
      uint32_t roc = 1 + r % 8;
      uint32_t index = m.fedIdx * PF_MAX_LINK * PF_MAX_ROC + (link - 1) * PF_MAX_ROC + roc;
      cab->fed[index] = 1200 + m.fedIdx;
      cab->link[index] = link;
      cab->roc[index] = roc;
      cab->rawId[index] = m.rawId;
      cab->rocInDet[index] = r;
      cab->moduleId[index] = i;
      uint8_t bad = (cfg.bad_roc_frac > 0 && U(rng) < cfg.bad_roc_frac) ? 1 : 0;
      cab->badRocs[index] = bad;
      d.badRoc[index] = bad;
      maxIndex = std::max(maxIndex, index);
    }
  }
  cab->size = maxIndex + 1;
  d.cabling.clear();
  appendPod(d.cabling, *cab);
  uint32_t nUnp = PF_MAX_SIZE;
  appendPod(d.cabling, nUnp);
  d.cabling.insert(d.cabling.end(), PF_MAX_SIZE, uint8_t(0));

  // ---- gains: per module 416 columns x 2 row blocks x {gain, ped}
  PfGainHeader& g = d.gainHdr;
  std::memset(&g, 0, sizeof(g));
  g.minPed = 10.f;
  g.maxPed = 40.f;
  g.minGain = 2.f;
  g.maxGain = 4.f;
  g.nBinsToUseForEncoding = 253;
  g.pedPrecision = (g.maxPed - g.minPed) / float(g.nBinsToUseForEncoding);
  g.gainPrecision = (g.maxGain - g.minGain) / float(g.nBinsToUseForEncoding);
  g.numberOfRowsAveragedOver = 80;
  g.deadFlag = 255;
  g.noisyFlag = 254;
  const uint32_t perModule = 416 * 4;
  d.gainPayload.assign(size_t(PF_N_MODULES) * perModule, 0);
  std::normal_distribution<double> N(0.0, 1.0);
  for (int i = 0; i < PF_MAX_MODULES; ++i) {
    if (i < PF_N_MODULES) {
      g.rangeAndCols[i].first = i * perModule;
      g.rangeAndCols[i].second = (i + 1) * perModule;
      g.rangeAndCols[i].nCols = 416;
    } else {
      g.rangeAndCols[i].first = g.rangeAndCols[i].second = 0;
      g.rangeAndCols[i].nCols = 416;
    }
  }
  for (size_t k = 0; k < d.gainPayload.size() / 2; ++k) {
    int gb = int(std::lround(126.5 + 20.0 * N(rng)));
    int pb = int(std::lround(126.5 + 15.0 * N(rng)));
    gb = std::min(253, std::max(0, gb));
    pb = std::min(253, std::max(0, pb));
    if (cfg.dead_column_frac > 0 && U(rng) < cfg.dead_column_frac)
      pb = int(g.deadFlag);
    d.gainPayload[2 * k] = uint8_t(gb);
    d.gainPayload[2 * k + 1] = uint8_t(pb);
  }
  d.gain.clear();
  appendPod(d.gain, g);
  uint32_t nbytes = uint32_t(d.gainPayload.size());
  appendPod(d.gain, nbytes);
  d.gain.insert(d.gain.end(), d.gainPayload.begin(), d.gainPayload.end());

  // ---- CPE
  PfCommonParams cp{float(kThickB), float(kThickE), float(kPitchX), float(kPitchY)};
  d.cpe.clear();
  appendPod(d.cpe, cp);
  uint32_t ndet = PF_N_MODULES;
  appendPod(d.cpe, ndet);
  for (int i = 0; i < PF_N_MODULES; ++i) {
    const Module& m = d.modules[i];
    PfDetParams dp;
    std::memset(&dp, 0, sizeof(dp));
    dp.isBarrel = m.barrel;
    dp.isPosZ = m.posZ;
    dp.layer = m.barrel ? uint16_t(m.layer + 1) : uint16_t(m.layer - 3);
    dp.index = uint16_t(i);
    dp.rawId = m.rawId;
    dp.shiftX = float(-m.tanLA * m.thick / 2);
    dp.shiftY = 0.f;
    dp.chargeWidthX = float(-m.tanLA * m.thick);
    dp.chargeWidthY = 0.f;
    double o[3] = {-m.p[0], -m.p[1], -m.p[2]};
    dp.x0 = float(dot3(m.ex, o));
    dp.y0 = float(dot3(m.ey, o));
    dp.z0 = float(dot3(m.ez, o));
    const float sx[3] = {0.0015f, 0.0029f, 0.0058f};
    const float sy[3] = {0.0022f, 0.0043f, 0.0087f};
    for (int k = 0; k < 3; ++k) {
      dp.sx[k] = sx[k];
      dp.sy[k] = sy[k];
    }
    dp.frame.px = float(m.p[0]);
    dp.frame.py = float(m.p[1]);
    dp.frame.pz = float(m.p[2]);
    dp.frame.R11 = float(m.ex[0]); dp.frame.R12 = float(m.ex[1]); dp.frame.R13 = float(m.ex[2]);
    dp.frame.R21 = float(m.ey[0]); dp.frame.R22 = float(m.ey[1]); dp.frame.R23 = float(m.ey[2]);
    dp.frame.R31 = float(m.ez[0]); dp.frame.R32 = float(m.ez[1]); dp.frame.R33 = float(m.ez[2]);
    appendPod(d.cpe, dp);
  }
  PfAverageGeometry ag;
  std::memset(&ag, 0, sizeof(ag));
  for (int il = 0; il < PF_N_LADDERS_BARREL; ++il) {
    double sx = 0, sy = 0, sz = 0, mnz = 1e9, mxz = -1e9;
    for (int k = 0; k < 8; ++k) {
      const Module& m = d.modules[il * 8 + k];
      sx += m.p[0];
      sy += m.p[1];
      sz += m.p[2];
      mnz = std::min(mnz, m.p[2] - kHalfY);
      mxz = std::max(mxz, m.p[2] + kHalfY);
    }
    ag.ladderX[il] = float(sx / 8);
    ag.ladderY[il] = float(sy / 8);
    ag.ladderZ[il] = float(sz / 8);
    ag.ladderR[il] = float(std::sqrt(sx * sx + sy * sy) / 8);
    ag.ladderMinZ[il] = float(mnz);
    ag.ladderMaxZ[il] = float(mxz);
  }
  ag.endCapZ[0] = float(d.modules[kLayerStart[4]].p[2]);
  ag.endCapZ[1] = float(d.modules[kLayerStart[7]].p[2]);
  appendPod(d.cpe, ag);
  PfLayerGeometry lg;
  std::memset(&lg, 0, sizeof(lg));
  for (int i = 0; i < 11; ++i)
    lg.layerStart[i] = kLayerStart[i];
  for (int i = 0; i < PF_LAYER_INDEX_SIZE; ++i) {
    uint32_t det = i * 16;
    uint8_t l = 11;
    for (uint8_t k = 0; k < 11; ++k)
      if (det < kLayerStart[k + 1]) {
        l = k;
        break;
      }
    lg.layer[i] = l;
  }
  appendPod(d.cpe, lg);

  // ---- beam spot
  PfBeamSpot bs{0.05f, -0.03f, 0.3f, 3.5f, 0.0015f, 0.0015f, 0.f, 0.f, 0.f, 0.f, 0.f};
  d.bs = bs;
  d.beamspot.clear();
  appendPod(d.beamspot, bs);

  // ---- fed ids
  d.fedids.clear();
  uint32_t nf = kNFeds;
  appendPod(d.fedids, nf);
  for (uint32_t f = 0; f < uint32_t(kNFeds); ++f) {
    uint32_t id = 1200 + f;
    appendPod(d.fedids, id);
  }
}

// ---- pixel/ROC geometry -------------------------------------------------

// local pitch-unit coordinate -> module row (inverse of phase1PixelTopology::localX)
int rowFromUnits(double u) {
  if (u < 0 || u >= 162) return -1;
  if (u < 79) return int(u);
  if (u < 81) return 79;
  if (u < 83) return 80;
  return int(u) - 2;
}
// inverse of phase1PixelTopology::localY
int colFromUnits(double u) {
  if (u < 0 || u >= 432) return -1;
  int roc = int(u / 54);
  double w = u - 54.0 * roc;
  int yin;
  if (w < 2) yin = 0;
  else if (w >= 52) yin = 51;
  else yin = int(w) - 1;
  return 52 * roc + yin;
}

// module pixel -> (rocInDet, row in ROC, col in ROC); inverse of frameConversion
void moduleToRoc(bool frameAB, int R, int C, int& roc, int& row, int& col) {
  if (frameAB) {
    if (R < 80) {
      roc = 7 - C / 52;
      col = (8 - roc) * 52 - 1 - C;
      row = R;
    } else {
      roc = 8 + C / 52;
      col = C % 52;
      row = 159 - R;
    }
  } else {
    if (R >= 80) {
      roc = C / 52;
      col = C % 52;
      row = 159 - R;
    } else {
      roc = 15 - C / 52;
      col = (16 - roc) * 52 - 1 - C;
      row = R;
    }
  }
}

// ---- helix -----------------------------------------------------------------

struct Helix {
  double x, y, z, psi, cot, kappa;  // kappa = q / R, dpsi/ds = -kappa
  void at(double s, double* P) const {
    double ps = psi - kappa * s;
    P[0] = x + (std::sin(psi) - std::sin(ps)) / kappa;
    P[1] = y + (std::cos(ps) - std::cos(psi)) / kappa;
    P[2] = z + s * cot;
  }
  void tangent(double s, double* T) const {
    double ps = psi - kappa * s;
    T[0] = std::cos(ps);
    T[1] = std::sin(ps);
    T[2] = cot;
  }
  // smallest s > eps where x^2+y^2 = r^2 ; <0 if none
  double cylinder(double r) const {
    double cx = x + std::sin(psi) / kappa, cy = y - std::cos(psi) / kappa;
    double rho = 1.0 / std::fabs(kappa);
    double dd = std::sqrt(cx * cx + cy * cy);
    if (dd > r + rho || dd < std::fabs(r - rho) || dd == 0) return -1;
    double a = (r * r - rho * rho + dd * dd) / (2 * dd);
    double h2 = r * r - a * a;
    double h = h2 > 0 ? std::sqrt(h2) : 0;
    double best = -1;
    for (int sgn = -1; sgn <= 1; sgn += 2) {
      double px = a * cx / dd + sgn * h * (-cy) / dd;
      double py = a * cy / dd + sgn * h * (cx) / dd;
      // psi at that point: (x-cx, y-cy) = (-sin psi, cos psi)/kappa
      double ps = std::atan2(-(px - cx) * kappa, (py - cy) * kappa);
      double ds = (psi - ps) / kappa;
      double period = 2 * kPi / std::fabs(kappa);
      ds = std::fmod(ds, period);
      if (ds < 0) ds += period;
      if (ds > 1e-6 && (best < 0 || ds < best)) best = ds;
    }
    return best;
  }
  // Newton: n.(P(s)-p) = 0 starting near s0
  bool plane(const double* n, const double* p, double s0, double& s) const {
    s = s0;
    for (int it = 0; it < 12; ++it) {
      double P[3], T[3];
      at(s, P);
      tangent(s, T);
      double f = n[0] * (P[0] - p[0]) + n[1] * (P[1] - p[1]) + n[2] * (P[2] - p[2]);
      double fp = dot3(n, T);
      if (std::fabs(fp) < 1e-9) return false;
      double ds = f / fp;
      s -= ds;
      if (std::fabs(ds) < 1e-10) break;
    }
    double P[3];
    at(s, P);
    double f = n[0] * (P[0] - p[0]) + n[1] * (P[1] - p[1]) + n[2] * (P[2] - p[2]);
    return std::fabs(f) < 1e-7 && s > 1e-6;
  }
};

struct SimHit {
  int module;
  double s;
  double P[3];
  double T[3];  // tangent (unnormalised)
};

// Moyal variate (analytic approximation of the Landau shape), mode 0
double moyal(std::mt19937_64& rng) {
  std::normal_distribution<double> N(0.0, 1.0);
  double z = N(rng);
  double x = -std::log(z * z + 1e-300);
  return std::min(x, 12.0);
}

struct Deposit {
  uint32_t key;  // module << 17 | row << 9 | col
  float q;
};

void depositHit(const ps_detector& d, const SimHit& h, double qtot, std::mt19937_64& rng,
                std::vector<Deposit>& out) {
  const Module& m = d.modules[h.module];
  double tn = std::sqrt(dot3(h.T, h.T));
  double dir[3] = {h.T[0] / tn, h.T[1] / tn, h.T[2] / tn};
  double dl[3] = {dot3(m.ex, dir), dot3(m.ey, dir), dot3(m.ez, dir)};
  if (std::fabs(dl[2]) < 0.05) dl[2] = dl[2] < 0 ? -0.05 : 0.05;
  double rel[3] = {h.P[0] - m.p[0], h.P[1] - m.p[1], h.P[2] - m.p[2]};
  double lx = dot3(m.ex, rel), ly = dot3(m.ey, rel);
  const int nseg = 24;
  std::normal_distribution<double> N(0.0, 1.0);
  // per-hit map of small size
  std::vector<Deposit> local;
  for (int i = 0; i < nseg; ++i) {
    double f = (i + 0.5) / nseg;
    double zl = -m.thick / 2 + f * m.thick;
    double xs = lx + dl[0] / dl[2] * zl + m.tanLA * (zl + m.thick / 2) + 0.0004 * N(rng);
    double ys = ly + dl[1] / dl[2] * zl + 0.0004 * N(rng);
    int row = rowFromUnits(xs / kPitchX + 81.0);
    int col = colFromUnits(ys / kPitchY + 216.0);
    if (row < 0 || col < 0) continue;
    double q = qtot / nseg * (1.0 + 0.2 * N(rng));
    if (q < 0) q = 0;
    uint32_t key = (uint32_t(h.module) << 17) | (uint32_t(row) << 9) | uint32_t(col);
    bool found = false;
    for (auto& dd : local)
      if (dd.key == key) {
        dd.q += float(q);
        found = true;
        break;
      }
    if (!found) local.push_back({key, float(q)});
  }
  out.insert(out.end(), local.begin(), local.end());
}

// electrons -> ADC through the module's gain/pedestal (inverse of gpuCalibPixel.h:46-63)
int electronsToAdc(const ps_detector& d, int module, int row, int col, double e) {
  const Module& m = d.modules[module];
  bool l1 = module < 96;
  double conv = l1 ? 50.0 : 47.0;
  double off = l1 ? -670.0 : -60.0;
  const PfGainHeader& g = d.gainHdr;
  uint32_t offset = g.rangeAndCols[module].first + col * 4 + 2 * (row / 80);
  uint8_t gb = d.gainPayload[offset], pb = d.gainPayload[offset + 1];
  (void)m;
  double gain = gb * g.gainPrecision + g.minGain;
  double ped = pb * g.pedPrecision + g.minPed;
  double vcal = (e - off) / conv;
  long adc = std::lround(vcal / gain + ped);
  return int(std::min(255L, std::max(1L, adc)));
}

uint32_t packWord(bool layer1, uint32_t link, uint32_t roc, uint32_t row, uint32_t col, uint32_t adc) {
  if (layer1)
    return (link << 26) | (roc << 21) | (col << 15) | (row << 8) | adc;
  uint32_t dcol = col / 2;
  uint32_t pxid = 2 * (80 - row) + (col % 2);
  return (link << 26) | (roc << 21) | (dcol << 16) | (pxid << 8) | adc;
}

void fedHeader(std::vector<uint8_t>& v, uint32_t fedId, uint32_t lvl1) {
  uint32_t sourceid = ((0u << 20) & 0xfff00000u) | ((fedId << 8) & 0x000fff00u) | ((1u << 4) & 0xf0u);
  uint32_t eventid = (0x5u << 28) | ((1u << 24) & 0x0f000000u) | (lvl1 & 0x00ffffffu);
  appendPod(v, sourceid);
  appendPod(v, eventid);
}
void fedTrailer(std::vector<uint8_t>& v, uint32_t len64) {
  uint32_t conscheck = 0;  // crc 0, no CRC-modified bit, no more trailers
  uint32_t eventsize = (0xau << 28) | (len64 & 0x00ffffffu);
  appendPod(v, conscheck);
  appendPod(v, eventsize);
}

}  // namespace

extern "C" {

void ps_default_detector_config(ps_detector_config* cfg) {
  cfg->seed = 20261203ull;
  cfg->dead_column_frac = 0.0;
  cfg->bad_roc_frac = 0.0;
}

void ps_default_event_config(ps_event_config* cfg) {
  cfg->tracks_per_vertex = 82.0;
  cfg->pt_min = 0.5;
  cfg->pt_index = 3.0;
  cfg->eta_max = 2.5;
  cfg->noise_frac = 0.001;
  cfg->inject_errors = 0;
  cfg->fixed_pu = 1;
  cfg->soft_per_vertex = 0.0;
  cfg->soft_pt_min = 0.05;
  cfg->soft_pt_mean = 0.25;
  cfg->secondary_frac = 0.0;
}

void ps_calibrated_event_config(ps_event_config* cfg) {
  ps_default_event_config(cfg);
  cfg->tracks_per_vertex = 28.0;
  cfg->pt_index = 3.5;
  cfg->soft_per_vertex = 50.0;
  cfg->soft_pt_mean = 0.25;
  cfg->secondary_frac = 0.8;
}

int ps_detector_create(const ps_detector_config* cfg, ps_detector** out) {
  if (!out) return -1;
  ps_detector_config c;
  if (cfg)
    c = *cfg;
  else
    ps_default_detector_config(&c);
  auto d = std::make_unique<ps_detector>();
  buildModules(*d);
  buildES(*d, c);
  *out = d.release();
  return 0;
}

void ps_detector_destroy(ps_detector* det) { delete det; }

int ps_detector_es(const ps_detector* det, int kind, const uint8_t** data, size_t* size) {
  if (!det || !data || !size) return -1;
  const std::vector<uint8_t>* v = nullptr;
  switch (kind) {
    case PS_ES_CABLING: v = &det->cabling; break;
    case PS_ES_GAIN: v = &det->gain; break;
    case PS_ES_CPE: v = &det->cpe; break;
    case PS_ES_BEAMSPOT: v = &det->beamspot; break;
    case PS_ES_FEDIDS: v = &det->fedids; break;
    default: return -2;
  }
  *data = v->data();
  *size = v->size();
  return 0;
}

int ps_detector_write(const ps_detector* det, const char* dir) {
  if (!det || !dir) return -1;
  const char* names[5] = {"cablingMap.bin", "gain.bin", "cpefast.bin", "beamspot.bin", "fedIds.bin"};
  for (int k = 0; k < 5; ++k) {
    const uint8_t* p;
    size_t n;
    ps_detector_es(det, k, &p, &n);
    std::string path = std::string(dir) + "/" + names[k];
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return -3;
    size_t w = std::fwrite(p, 1, n, f);
    std::fclose(f);
    if (w != n) return -4;
  }
  return 0;
}

int ps_event_generate(const ps_detector* det, uint64_t seed, double pu, const ps_event_config* cfgp,
                      ps_event** out) {
  if (!det || !out) return -1;
  ps_event_config cfg;
  if (cfgp)
    cfg = *cfgp;
  else
    ps_default_event_config(&cfg);
  const ps_detector& d = *det;
  auto ev = std::make_unique<ps_event>();
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  std::normal_distribution<double> N(0.0, 1.0);

  int nvtx = cfg.fixed_pu ? int(std::lround(pu)) : int(std::poisson_distribution<int>(pu)(rng));
  std::vector<Deposit> deposits;
  deposits.reserve(size_t(nvtx * cfg.tracks_per_vertex * 5 * 4) + 16);

  // One charged track from (vx, vy, vz): helix steps from surface to
  // surface, charge deposits on every module crossed, multiple scattering at
  // each layer.  `start` > 0 moves the origin that far along the initial
  // direction in the transverse plane (a displaced secondary).
  auto propagate = [&](double vx, double vy, double vz, double pt, double eta, double phi, int q, int iv,
                       double start) {
    double cot = std::sinh(eta);
    double R = pt / kBField;
    Helix hx{vx, vy, vz, phi, cot, q / R};
    if (start > 0) {
      double P0[3];
      hx.at(start, P0);
      double T0[3];
      hx.tangent(start, T0);
      hx.x = P0[0];
      hx.y = P0[1];
      hx.z = P0[2];
      hx.psi = std::atan2(T0[1], T0[0]);
    }
    double p = pt * std::sqrt(1 + cot * cot);
    uint8_t nh = 0;
    bool crossedB[4] = {false, false, false, false};
    bool crossedD[6][4] = {};
    for (int step = 0; step < 30; ++step) {
      // next surface
      double bestS = -1;
      int bestKind = -1, bestA = 0, bestB = 0;
      for (int L = 0; L < 4; ++L) {
        if (crossedB[L]) continue;
        double s = hx.cylinder(kBarrelR[L]);
        if (s > 0 && (bestS < 0 || s < bestS)) {
          bestS = s; bestKind = 0; bestA = L;
        }
      }
      if (hx.cot != 0) {
        for (int e = 0; e < 6; ++e)
          for (int pl = 0; pl < 4; ++pl) {
            if (crossedD[e][pl]) continue;
            int disk = e % 3;
            int g = pl / 2, pan = 1 + pl % 2;
            double az = kDiskZ[disk] + (pan == 1 ? -0.25 : 0.25) + (g == 1 ? 0.8 : 0.0);
            double zp = e < 3 ? az : -az;
            double s = (zp - hx.z) / hx.cot;
            if (s > 1e-6 && (bestS < 0 || s < bestS)) {
              bestS = s; bestKind = 1; bestA = e; bestB = pl;
            }
          }
      }
      if (bestS < 0) break;
      double Pc[3];
      hx.at(bestS, Pc);
      if (std::fabs(Pc[2]) > 55.0 || std::hypot(Pc[0], Pc[1]) > 17.5) break;
      std::vector<SimHit> hits;
      if (bestKind == 0) {
        int L = bestA;
        crossedB[L] = true;
        int nl = kLadders[L];
        double phic = std::atan2(Pc[1], Pc[0]);
        if (phic < 0) phic += 2 * kPi;
        int l0 = int(std::floor(phic * nl / (2 * kPi)));
        for (int dlad = -1; dlad <= 1; ++dlad) {
          int l = ((l0 + dlad) % nl + nl) % nl;
          const Module& ref = d.modules[kLayerStart[L] + 8 * l];
          double lp[3] = {ref.p[0], ref.p[1], 0.0};
          double s;
          if (!hx.plane(ref.ez, lp, bestS, s)) continue;
          double P[3];
          hx.at(s, P);
          double rel[3] = {P[0] - lp[0], P[1] - lp[1], P[2]};
          double lx = dot3(ref.ex, rel);
          if (std::fabs(lx) >= kHalfX) continue;
          int k = int(std::floor((P[2] + 26.8) / 6.7));
          if (k < 0 || k > 7) continue;
          double ly = P[2] - (k - 3.5) * 6.7;
          if (std::fabs(ly) >= kHalfY) continue;
          SimHit h;
          h.module = kLayerStart[L] + 8 * l + k;
          h.s = s;
          std::memcpy(h.P, P, sizeof(P));
          hx.tangent(s, h.T);
          hits.push_back(h);
        }
      } else {
        int e = bestA, pl = bestB;
        crossedD[e][pl] = true;
        int g = pl / 2, pan = 1 + pl % 2;
        double r = std::hypot(Pc[0], Pc[1]);
        if (std::fabs(r - kRingR[g]) < kHalfY + 0.01) {
          int n = kRingN[g];
          double phic = std::atan2(Pc[1], Pc[0]);
          if (phic < 0) phic += 2 * kPi;
          int j0 = int(std::floor(phic * n / (2 * kPi)));
          int base = kLayerStart[4 + e] + (g == 1 ? kRingN[0] : 0);
          for (int dj = -2; dj <= 2; ++dj) {
            int j = ((j0 + dj) % n + n) % n;
            if (1 + j % 2 != pan) continue;
            const Module& m = d.modules[base + j];
            double rel[3] = {Pc[0] - m.p[0], Pc[1] - m.p[1], Pc[2] - m.p[2]};
            double lx = dot3(m.ex, rel), ly = dot3(m.ey, rel);
            if (std::fabs(lx) >= kHalfX || std::fabs(ly) >= kHalfY) continue;
            SimHit h;
            h.module = base + j;
            h.s = bestS;
            std::memcpy(h.P, Pc, sizeof(Pc));
            hx.tangent(bestS, h.T);
            hits.push_back(h);
          }
        }
      }
      if (hits.empty()) continue;
      std::sort(hits.begin(), hits.end(), [](const SimHit& a, const SimHit& b) { return a.s < b.s; });
      for (auto& h : hits) {
        double path = 1.0;
        {
          const Module& m = d.modules[h.module];
          double tn = std::sqrt(dot3(h.T, h.T));
          double cz = std::fabs(dot3(m.ez, h.T)) / tn;
          path = 1.0 / std::max(cz, 0.05);
        }
        double qtot = (21000.0 + 1400.0 * moyal(rng)) * std::min(path, 8.0);
        depositHit(d, h, qtot, rng, deposits);
        ++nh;
        ++ev->nSimHits;
      }
      // multiple scattering at the last hit, restart the helix there
      const SimHit& last = hits.back();
      double tn = std::sqrt(dot3(last.T, last.T));
      double dir[3] = {last.T[0] / tn, last.T[1] / tn, last.T[2] / tn};
      double x0 = (bestKind == 0 ? 0.025 : 0.03) * hits.size();
      double th0 = 0.0136 / p * std::sqrt(x0) * (1 + 0.038 * std::log(x0));
      double u1[3] = {-dir[1], dir[0], 0};
      double nu = std::sqrt(u1[0] * u1[0] + u1[1] * u1[1]);
      if (nu < 1e-9) {
        u1[0] = 1; u1[1] = 0; nu = 1;
      }
      u1[0] /= nu; u1[1] /= nu;
      double u2[3] = {dir[1] * u1[2] - dir[2] * u1[1], dir[2] * u1[0] - dir[0] * u1[2], dir[0] * u1[1] - dir[1] * u1[0]};
      double a1 = th0 * N(rng), a2 = th0 * N(rng);
      double nd[3];
      for (int k = 0; k < 3; ++k) nd[k] = dir[k] + a1 * u1[k] + a2 * u2[k];
      double nn = std::sqrt(dot3(nd, nd));
      for (int k = 0; k < 3; ++k) nd[k] /= nn;
      double ptn = p * std::sqrt(nd[0] * nd[0] + nd[1] * nd[1]);
      if (ptn < 1e-3) break;
      hx.x = last.P[0];
      hx.y = last.P[1];
      hx.z = last.P[2];
      hx.psi = std::atan2(nd[1], nd[0]);
      hx.cot = nd[2] / std::sqrt(nd[0] * nd[0] + nd[1] * nd[1]);
      hx.kappa = q * kBField / ptn;
    }
    ev->tpt.push_back(float(pt));
    ev->teta.push_back(float(eta));
    ev->tphi.push_back(float(phi));
    ev->tq.push_back(q);
    ev->tv.push_back(iv);
    ev->tnh.push_back(nh);
  };

  for (int iv = 0; iv < nvtx; ++iv) {
    double vz = d.bs.z + 3.5 * N(rng);
    double vx = d.bs.x + 0.0015 * N(rng), vy = d.bs.y + 0.0015 * N(rng);
    ev->vz.push_back(float(vz));
    int ntk = std::poisson_distribution<int>(cfg.tracks_per_vertex)(rng);
    for (int it = 0; it < ntk; ++it) {
      double u = U(rng);
      double pt = cfg.pt_min * std::pow(1.0 - u, -1.0 / (cfg.pt_index - 1.0));
      pt = std::min(pt, 100.0);
      double eta = (2 * U(rng) - 1) * cfg.eta_max;
      double phi = (2 * U(rng) - 1) * kPi;
      int q = U(rng) < 0.5 ? -1 : 1;
      propagate(vx, vy, vz, pt, eta, phi, q, iv, 0.0);
    }
    // soft component: exponential pT above soft_pt_min (loopers below
    // ~0.3 GeV curl inside the pixel volume), a share of it produced
    // displaced (conversions and decays: outside the CA's z0/dca cuts).
    // No random numbers are drawn when it is off, so events without it are
    // those of earlier versions of this generator.
    if (cfg.soft_per_vertex > 0) {
      int nsoft = std::poisson_distribution<int>(cfg.soft_per_vertex)(rng);
      std::exponential_distribution<double> Ex(1.0 / std::max(cfg.soft_pt_mean, 1e-3));
      for (int it = 0; it < nsoft; ++it) {
        double pt = cfg.soft_pt_min + Ex(rng);
        double eta = (2 * U(rng) - 1) * cfg.eta_max;
        double phi = (2 * U(rng) - 1) * kPi;
        int q = U(rng) < 0.5 ? -1 : 1;
        double start = U(rng) < cfg.secondary_frac ? 2.0 + 10.0 * U(rng) : 0.0;
        propagate(vx, vy, vz, pt, eta, phi, q, iv, start);
      }
    }
  }
  // merge deposits per pixel
  std::sort(deposits.begin(), deposits.end(), [](const Deposit& a, const Deposit& b) { return a.key < b.key; });
  std::vector<Deposit> pix;
  for (auto& dd : deposits) {
    if (!pix.empty() && pix.back().key == dd.key)
      pix.back().q += dd.q;
    else
      pix.push_back(dd);
  }
  size_t nSignal = 0;
  for (auto& px : pix)
    if (px.q >= 1000.f) ++nSignal;
  // noise digis
  size_t nNoise = size_t(std::lround(cfg.noise_frac * double(nSignal)));
  for (size_t k = 0; k < nNoise; ++k) {
    uint32_t m = uint32_t(U(rng) * PF_N_MODULES) % PF_N_MODULES;
    uint32_t row = uint32_t(U(rng) * 160) % 160, col = uint32_t(U(rng) * 416) % 416;
    pix.push_back({(m << 17) | (row << 9) | col, float(1500.0 + 4500.0 * U(rng))});
  }
  std::sort(pix.begin(), pix.end(), [](const Deposit& a, const Deposit& b) { return a.key < b.key; });
  // per module, per ROC lists of encoded words
  struct W {
    uint32_t sortKey;
    uint32_t word;
  };
  std::vector<std::vector<W>> rocWords(size_t(PF_N_MODULES) * 16);
  uint32_t ndig = 0;
  for (size_t k = 0; k < pix.size(); ++k) {
    if (k + 1 < pix.size() && pix[k + 1].key == pix[k].key) {  // noise on a signal pixel: merge
      pix[k + 1].q += pix[k].q;
      continue;
    }
    if (pix[k].q < 1000.f) continue;
    int m = int(pix[k].key >> 17), row = int((pix[k].key >> 9) & 0xff), col = int(pix[k].key & 0x1ff);
    const Module& mod = d.modules[m];
    int roc, rrow, rcol;
    moduleToRoc(mod.frameAB, row, col, roc, rrow, rcol);
    uint32_t link = mod.linkA + roc / 8;
    uint32_t rocInLink = 1 + roc % 8;
    uint32_t index = mod.fedIdx * PF_MAX_LINK * PF_MAX_ROC + (link - 1) * PF_MAX_ROC + rocInLink;
    (void)index;
    int adc = electronsToAdc(d, m, row, col, pix[k].q);
    bool l1 = m < 96;
    uint32_t w = packWord(l1, link, rocInLink, rrow, rcol, adc);
    uint32_t sk = l1 ? ((uint32_t(rcol) << 8) | uint32_t(rrow)) : (w & 0x1fff00u);
    rocWords[size_t(m) * 16 + roc].push_back({sk, w});
    ++ndig;
  }
  ev->nDigis = ndig;
  // error words: appended at the end of a random FED payload
  std::vector<std::vector<uint32_t>> extra(kNFeds);
  for (int k = 0; k < cfg.inject_errors; ++k) {
    int f = int(U(rng) * kNFeds) % kNFeds;
    if (d.fedModules[f].empty()) continue;
    int m = d.fedModules[f][int(U(rng) * d.fedModules[f].size()) % d.fedModules[f].size()];
    uint32_t link = d.modules[m].linkA;
    static const uint32_t types[] = {26, 27, 28, 29, 30, 31, 37};
    uint32_t t = types[k % 7];
    uint32_t w;
    if (t == 37) {
      bool l1 = m < 96;
      w = l1 ? ((link << 26) | (1u << 21) | (3u << 15) | (100u << 8) | 50u)
             : ((link << 26) | (1u << 21) | (3u << 16) | (0u << 8) | 50u);
    } else if (t == 29) {
      w = (link << 26) | (29u << 21) | (1u << 8) | 0x3u;  // block 1, channels 1+2
    } else if (t == 30) {
      w = (link << 26) | (30u << 21) | ((k % 2 ? 1u : 8u) << 8);
    } else {
      w = (link << 26) | (t << 21) | uint32_t(k & 0xff);
    }
    extra[f].push_back(w);
  }
  // FED framing
  std::vector<uint8_t>& raw = ev->raw;
  uint32_t nfeds = kNFeds;
  appendPod(raw, nfeds);
  uint32_t lvl1 = uint32_t(seed & 0xffffff);
  for (int f = 0; f < kNFeds; ++f) {
    std::vector<uint32_t> words;
    for (int m : d.fedModules[f])
      for (int r8 = 0; r8 < 16; ++r8) {
        auto& v = rocWords[size_t(m) * 16 + r8];
        std::sort(v.begin(), v.end(), [](const W& a, const W& b) { return a.sortKey < b.sortKey; });
        for (auto& w : v) words.push_back(w.word);
      }
    for (auto w : extra[f]) words.push_back(w);
    if (words.size() % 2) words.push_back(0u);
    uint32_t fedId = 1200 + f;
    uint32_t len64 = uint32_t(words.size() / 2 + 2);
    uint32_t size = len64 * 8;
    appendPod(raw, fedId);
    appendPod(raw, size);
    fedHeader(raw, fedId, lvl1);
    for (auto w : words) appendPod(raw, w);
    fedTrailer(raw, len64);
  }
  *out = ev.release();
  return 0;
}

void ps_event_destroy(ps_event* ev) { delete ev; }

int ps_event_raw(const ps_event* ev, const uint8_t** data, size_t* size) {
  if (!ev || !data || !size) return -1;
  *data = ev->raw.data();
  *size = ev->raw.size();
  return 0;
}

int ps_event_truth(const ps_event* ev, ps_truth* out) {
  if (!ev || !out) return -1;
  out->n_vertices = uint32_t(ev->vz.size());
  out->n_tracks = uint32_t(ev->tpt.size());
  out->n_sim_hits = ev->nSimHits;
  out->n_digis = ev->nDigis;
  out->vertex_z = ev->vz.data();
  out->track_pt = ev->tpt.data();
  out->track_eta = ev->teta.data();
  out->track_phi = ev->tphi.data();
  out->track_q = ev->tq.data();
  out->track_vertex = ev->tv.data();
  out->track_nhits = ev->tnh.data();
  return 0;
}

int ps_fit_tuples(uint64_t seed, uint32_t n, uint32_t nhits, double* hits, float* hits_ge, double* truth) {
  if (nhits < 3 || nhits > 5 || !hits || !hits_ge || !truth) return -1;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  std::normal_distribution<double> N(0.0, 1.0);
  const double radii[5] = {2.9, 6.8, 10.9, 16.0, 19.0};
  for (uint32_t t = 0; t < n; ++t) {
    double pt = std::min(0.5 * std::pow(1.0 - U(rng), -0.5), 50.0);
    double eta = (2 * U(rng) - 1) * 1.3;
    double phi = (2 * U(rng) - 1) * kPi;
    int q = U(rng) < 0.5 ? -1 : 1;
    double tip = 0.01 * N(rng), zip = 3.0 * N(rng);
    double cot = std::sinh(eta);
    double x0 = -tip * std::sin(phi), y0 = tip * std::cos(phi);
    Helix hx{x0, y0, zip, phi, cot, q * kBField / pt};
    double p = pt * std::sqrt(1 + cot * cot);
    truth[t * 5 + 0] = phi;
    truth[t * 5 + 1] = tip;
    truth[t * 5 + 2] = pt;
    truth[t * 5 + 3] = cot;
    truth[t * 5 + 4] = zip;
    for (uint32_t i = 0; i < nhits; ++i) {
      double s = hx.cylinder(radii[i]);
      if (s < 0) s = 1.0;
      double P[3], T[3];
      hx.at(s, P);
      hx.tangent(s, T);
      double ph = std::atan2(P[1], P[0]);
      double st = 0.0020, sz = 0.0030;
      double et = st * N(rng), ez = sz * N(rng);
      double* hp = hits + (size_t(t) * nhits + i) * 3;
      hp[0] = P[0] - et * std::sin(ph);
      hp[1] = P[1] + et * std::cos(ph);
      hp[2] = P[2] + ez;
      float* ge = hits_ge + (size_t(t) * nhits + i) * 6;
      ge[0] = float(st * st * std::sin(ph) * std::sin(ph));
      ge[1] = float(-st * st * std::sin(ph) * std::cos(ph));
      ge[2] = float(st * st * std::cos(ph) * std::cos(ph));
      ge[3] = 0.f;
      ge[4] = 0.f;
      ge[5] = float(sz * sz);
      // scatter
      double tn = std::sqrt(dot3(T, T));
      double dir[3] = {T[0] / tn, T[1] / tn, T[2] / tn};
      double x0l = 0.025;
      double th0 = 0.0136 / p * std::sqrt(x0l) * (1 + 0.038 * std::log(x0l));
      double nd[3] = {dir[0] - dir[1] * th0 * N(rng), dir[1] + dir[0] * th0 * N(rng), dir[2] + th0 * N(rng)};
      double ptn = p * std::sqrt(nd[0] * nd[0] + nd[1] * nd[1]) / std::sqrt(dot3(nd, nd));
      hx.x = P[0];
      hx.y = P[1];
      hx.z = P[2];
      hx.psi = std::atan2(nd[1], nd[0]);
      hx.cot = nd[2] / std::sqrt(nd[0] * nd[0] + nd[1] * nd[1]);
      hx.kappa = q * kBField / ptn;
    }
  }
  return 0;
}

}  // extern "C"
