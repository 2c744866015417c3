// Oracle (checker only): ES parsing, FED loop, raw-to-digi, calibration,
// clustering, charge cut, hit-module starts and rechits.  See oracle.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>

#include "oracle.h"

namespace oracle {

namespace {

struct Reader {
  const uint8_t* p;
  size_t n, off = 0;
  template <typename T>
  void get(T& x) {
    if (off + sizeof(T) > n) throw std::runtime_error("ES image truncated");
    std::memcpy(&x, p + off, sizeof(T));
    off += sizeof(T);
  }
  void bytes(void* dst, size_t k) {
    if (off + k > n) throw std::runtime_error("ES image truncated");
    std::memcpy(dst, p + off, k);
    off += k;
  }
};

constexpr uint16_t kInvId = PF_INV_ID;

// ---- raw-to-digi helpers: SiPixelRawToClusterGPUKernel.cc:51-339 -----------

struct DetIdGPU {
  uint32_t rawId, rocInDet, moduleId;
};

inline uint32_t cablingIndex(uint32_t fed, uint32_t link, uint32_t roc) {
  return fed * PF_MAX_LINK * PF_MAX_ROC + (link - 1) * PF_MAX_ROC + roc;
}

// :59-67
DetIdGPU getRawId(const PfCablingMap& cab, uint8_t fed, uint32_t link, uint32_t roc) {
  uint32_t index = cablingIndex(fed, link, roc);
  if (link == 0 || index >= uint32_t(PF_MAX_SIZE))
    throw std::runtime_error("undefined in the reference: a word outside the cabling tables");
  return {cab.rawId[index], cab.rocInDet[index], cab.moduleId[index]};
}

// :72-138
void frameConversion(bool bpix, int side, uint32_t layer, uint32_t rocIdInDetUnit, uint32_t row, uint32_t col,
                     uint32_t& gRow, uint32_t& gCol) {
  int slopeRow = 0, slopeCol = 0, rowOffset = 0, colOffset = 0;
  const int nr = 80, nc = 52;
  bool minusSide = bpix ? (side == -1 && layer != 1) : true;  // fpix: both panels use the same mapping
  if (minusSide) {
    if (rocIdInDetUnit < 8) {
      slopeRow = 1;
      slopeCol = -1;
      rowOffset = 0;
      colOffset = (8 - rocIdInDetUnit) * nc - 1;
    } else {
      slopeRow = -1;
      slopeCol = 1;
      rowOffset = 2 * nr - 1;
      colOffset = (rocIdInDetUnit - 8) * nc;
    }
  } else {
    if (rocIdInDetUnit < 8) {
      slopeRow = -1;
      slopeCol = 1;
      rowOffset = 2 * nr - 1;
      colOffset = rocIdInDetUnit * nc;
    } else {
      slopeRow = 1;
      slopeCol = -1;
      rowOffset = 0;
      colOffset = (16 - rocIdInDetUnit) * nc - 1;
    }
  }
  gRow = rowOffset + slopeRow * row;
  gCol = colOffset + slopeCol * col;
}

// :188-262
uint8_t checkROC(uint32_t errorWord, uint8_t fedId, uint32_t link, const PfCablingMap& cab) {
  uint8_t errorType = (errorWord >> 21) & 0x1f;
  if (errorType < 25) return 0;
  bool errorFound = false;
  switch (errorType) {
    case 25: {
      errorFound = true;
      uint32_t index = cablingIndex(fedId, link, 1);
      if (index > 1 && index <= cab.size) {
        if (!(link == cab.link[index] && 1 == cab.roc[index])) errorFound = false;
      }
      break;
    }
    case 26:
    case 27:
    case 28:
    case 29:
    case 31:
      errorFound = true;
      break;
    case 30: {
      int stateMatch = (errorWord >> 8) & 0xf;
      if (stateMatch == 1) errorType = 40;
      errorFound = true;
      break;
    }
    default:
      errorFound = false;
  }
  return errorFound ? errorType : 0;
}

// :264-339
uint32_t getErrRawID(uint8_t fedId, uint32_t errWord, uint32_t errorType, const PfCablingMap& cab) {
  uint32_t rID = 0xffffffff;
  switch (errorType) {
    case 25:
    case 30:
    case 31:
    case 36:
    case 40: {
      uint32_t link = (errWord >> 26) & 0x3f;
      uint32_t t = getRawId(cab, fedId, link, 1).rawId;
      if (t != 9999) rID = t;
      break;
    }
    case 29: {
      int ch[5];
      for (int k = 0; k < 5; ++k) ch[k] = (errWord >> k) & 1;
      int block = (errWord >> 8) & 0x7;
      int localCH = 1 * ch[0] + 2 * ch[1] + 3 * ch[2] + 4 * ch[3] + 5 * ch[4];
      int chanNmbr = (block % 2 == 0) ? (block / 2) * 9 + localCH : ((block - 1) / 2) * 9 + 4 + localCH;
      if (chanNmbr < 1 || chanNmbr > 36) break;
      uint32_t t = getRawId(cab, fedId, uint32_t(chanNmbr), 1).rawId;
      if (t != 9999) rID = t;
      break;
    }
    case 37:
    case 38: {
      uint32_t roc = (errWord >> 21) & 0x1f;
      uint32_t link = (errWord >> 26) & 0x3f;
      uint32_t t = getRawId(cab, fedId, link, roc).rawId;
      if (t != 9999) rID = t;
      break;
    }
    default:
      break;
  }
  return rID;
}

// ---- rechit helpers ----------------------------------------------------------

// Geometry/phase1PixelTopology.h:115-158
inline uint16_t divu52(uint16_t n) {
  n = n >> 2;
  uint16_t q = (n >> 1) + (n >> 4);
  q = q + (q >> 4) + (q >> 5);
  q = q >> 3;
  uint16_t r = n - q * 13;
  return q + ((r + 3) >> 4);
}
inline bool isBigPixX(uint16_t px) { return (px == 79) | (px == 80); }
inline bool isBigPixY(uint16_t py) {
  uint16_t ly = py - 52 * divu52(py);
  return (ly == 0) | (ly == 51);
}
inline uint16_t localX(uint16_t px) {
  int shift = 0;
  if (px > 79) shift += 1;
  if (px > 80) shift += 1;
  return px + shift;
}
inline uint16_t localY(uint16_t py) {
  uint16_t roc = divu52(py);
  int shift = 2 * roc;
  int yInRoc = py - 52 * roc;
  if (yInRoc > 0) shift += 1;
  return py + shift;
}

// CondFormats/pixelCPEforGPU.h:118-174
float correction(int sizeM1, int Q_f, int Q_l, uint16_t upper_edge_first_pix, uint16_t lower_edge_last_pix,
                 float lorentz_shift, float theThickness, float cot_angle, float pitch, bool first_is_big,
                 bool last_is_big) {
  if (0 == sizeM1) return 0;
  float W_eff = 0;
  bool simple = true;
  if (1 == sizeM1) {
    float W_inner = pitch * float(lower_edge_last_pix - upper_edge_first_pix);
    float W_pred = theThickness * cot_angle - lorentz_shift;
    W_eff = std::abs(W_pred) - W_inner;
    simple = (W_eff < 0.0f) | (W_eff > pitch);
  }
  if (simple) {
    float sum_of_edge = 2.0f;
    if (first_is_big) sum_of_edge += 1.0f;
    if (last_is_big) sum_of_edge += 1.0f;
    W_eff = pitch * 0.5f * sum_of_edge;
  }
  float Qdiff = Q_l - Q_f;
  float Qsum = Q_l + Q_f;
  if (Qsum == 0) Qsum = 1.0f;
  return 0.5f * (Qdiff / Qsum) * W_eff;
}

// DataFormats/approx_atan2.h:245-263 (degree-7 polynomial, coefficients of the reference)
inline float atan2sPoly7(float x) {
  float z = x * x;
  return x * ((-10422.177734375f) + z * (3349.97412109375f + z * ((-1525.589599609375f) + z * 406.64190673828125f)));
}
inline int16_t unsafeAtan2s7(float y, float x) {
  constexpr int maxshort = 32768;
  constexpr short pi4 = short(maxshort / 4);
  constexpr short pi34 = short(3 * maxshort / 4);
  float r = (std::abs(x) - std::abs(y)) / (std::abs(x) + std::abs(y));
  if (x < 0) r = -r;
  short angle = (x >= 0) ? pi4 : pi34;
  angle += short(atan2sPoly7(r));
  return (y < 0) ? short(-angle) : angle;
}

}  // namespace

void loadES(ES& es, const uint8_t* cabling, size_t ncab, const uint8_t* gain, size_t ngain, const uint8_t* cpe,
            size_t ncpe, const uint8_t* bs, size_t nbs, const uint8_t* fedids, size_t nfed) {
  {
    Reader r{cabling, ncab};
    es.cab = std::make_unique<PfCablingMap>();
    r.bytes(es.cab.get(), sizeof(PfCablingMap));
    uint32_t n;
    r.get(n);
    es.modToUnp.resize(n);
    r.bytes(es.modToUnp.data(), n);
  }
  {
    Reader r{gain, ngain};
    r.get(es.gain);
    uint32_t nb;
    r.get(nb);
    es.gainPayload.resize(nb);
    r.bytes(es.gainPayload.data(), nb);
  }
  {
    Reader r{cpe, ncpe};
    r.get(es.common);
    uint32_t nd;
    r.get(nd);
    es.det.resize(nd);
    r.bytes(es.det.data(), nd * sizeof(PfDetParams));
    r.get(es.ag);
    r.get(es.lg);
  }
  {
    Reader r{bs, nbs};
    r.get(es.bs);
  }
  {
    Reader r{fedids, nfed};
    uint32_t n;
    r.get(n);
    es.fedIds.resize(n);
    r.bytes(es.fedIds.data(), n * 4);
  }
}

// SiPixelRawToClusterCUDA.cc:78-138 with ErrorChecker.cc:36-91.  The
// reference's ErrorChecker records no errors (includeErrors = false in its
// constructor, :36); formatterErrors turns that recording on.
void fedLoop(const ES& es, const uint8_t* raw, size_t n, Words& w, bool formatterErrors, const Caps& caps) {
  // Source.cc:9-21 record layout
  std::vector<std::pair<const uint8_t*, uint32_t>> fedData(4096, {nullptr, 0});
  size_t off = 0;
  auto rd32 = [&](uint32_t& x) {
    if (off + 4 > n) throw std::runtime_error("raw record truncated");
    std::memcpy(&x, raw + off, 4);
    off += 4;
  };
  uint32_t nfeds;
  rd32(nfeds);
  for (uint32_t i = 0; i < nfeds; ++i) {
    uint32_t fedId, size;
    rd32(fedId);
    rd32(size);
    if (off + size > n || fedId >= 4096) throw std::runtime_error("raw record malformed");
    fedData[fedId] = {raw + off, size};
    off += size;
  }
  w.word.assign(caps.fedWords, 0);
  w.fedId.assign(caps.fedWords, 0);
  w.formatterErrors.clear();
  auto record = [&](uint64_t word64, uint32_t type, uint32_t fedId) {
    if (formatterErrors) w.formatterErrors.push_back({word64, type, fedId});
  };
  uint32_t wordCounter = 0;
  for (uint32_t fedId : es.fedIds) {
    if (fedId == 40) continue;
    const uint8_t* data = fedData[fedId].first;
    uint32_t size = fedData[fedId].second;
    int nWords = int(size / 8);
    if (nWords == 0) continue;
    auto word64 = [&](int k) {
      uint64_t v;
      std::memcpy(&v, data + 8 * size_t(k), 8);
      return v;
    };
    // checkCRC (:38-48): the CRC-modified bit of the last word drops the FED
    if ((word64(nWords - 1) >> 2) & 1) {
      record(word64(nWords - 1), 39, fedId);
      continue;
    }
    // checkHeader (:50-65): FEDHeader::check (start marker 0x5), sourceID,
    // moreHeaders; a word that fails the check ends the headers unrecorded
    int h = -1;
    bool more = true;
    while (more) {
      ++h;
      if (h >= nWords) throw std::runtime_error("undefined in the reference: headers run past the FED");
      uint64_t v = word64(h);
      uint32_t sourceid = uint32_t(v), eventid = uint32_t(v >> 32);
      if (((eventid >> 28) & 0xf) != 0x5) {
        more = false;
      } else {
        if (((sourceid >> 8) & 0xfff) != fedId) record(v, 32, fedId);
        more = ((sourceid >> 3) & 1) != 0;
      }
    }
    // checkTrailer (:67-91): FEDTrailer::check (end marker 0xa),
    // fragmentLength against the FED's 64-bit word count, moreTrailers
    int t = nWords;
    more = true;
    while (more) {
      --t;
      if (t < 0) throw std::runtime_error("undefined in the reference: trailers run past the FED");
      uint64_t v = word64(t);
      uint32_t conscheck = uint32_t(v), eventsize = uint32_t(v >> 32);
      if (((eventsize >> 28) & 0xf) != 0xa) {
        record(v, 33, fedId);
        more = false;
      } else {
        if ((eventsize & 0x00ffffffu) != uint32_t(nWords)) record(v, 34, fedId);
        more = ((conscheck >> 3) & 1) != 0;
      }
    }
    if (t < h + 1) throw std::runtime_error("undefined in the reference: header and trailer overlap");
    const uint8_t* bw = data + 8 * size_t(h + 1);
    const uint8_t* ew = data + 8 * size_t(t);
    uint32_t length = uint32_t((ew - bw) / 4);
    if (wordCounter + length > caps.fedWords)
      throw std::runtime_error("undefined in the reference: more than MAX_FED_WORDS words");
    // WordFedAppender::initializeWordFed (SiPixelRawToClusterGPUKernel.cc:41-47)
    std::memcpy(w.word.data() + wordCounter, bw, 4 * size_t(length));
    std::memset(w.fedId.data() + wordCounter / 2, int(fedId - 1200), length / 2);
    wordCounter += length;
  }
  w.nWords = wordCounter;
}

void makeClusters(const ES& es, const Words& w, Digis& d, Clusters& c, const Caps& caps) {
  const PfCablingMap& cab = *es.cab;
  const uint32_t nW = w.nWords;
  d.nDigis = nW;
  d.xx.assign(nW, 0);
  d.yy.assign(nW, 0);
  d.adc.assign(nW, 0);
  d.moduleInd.assign(nW, 0);
  d.clus.assign(nW, 0);
  d.pdigi.assign(nW, 0);
  d.rawIdArr.assign(nW, 0);
  d.errors.clear();


  // ---- RawToDigi_kernel (:342-462), useQualityInfo = includeErrors = true
  for (uint32_t i = 0; i < nW; ++i) {
    d.xx[i] = d.yy[i] = d.adc[i] = 0;
    uint8_t fedId = w.fedId[i / 2];
    d.pdigi[i] = 0;
    d.rawIdArr[i] = 0;
    d.moduleInd[i] = 9999;
    uint32_t ww = w.word[i];
    if (ww == 0) continue;
    uint32_t link = (ww >> 26) & 0x3f;
    uint32_t roc = (ww >> 21) & 0x1f;
    DetIdGPU det = getRawId(cab, fedId, link, roc);
    uint8_t errorType = checkROC(ww, fedId, link, cab);
    bool skipROC = (roc < 8) ? false : (errorType != 0);
    if (skipROC) {
      d.errors.push_back({getErrRawID(fedId, ww, errorType, cab), ww, errorType, fedId});
      continue;
    }
    uint32_t rawId = det.rawId;
    bool barrel = 1 == ((rawId >> 25) & 0x7);
    uint32_t index = cablingIndex(fedId, link, roc);
    if (cab.badRocs[index]) continue;
    if (es.modToUnp[index]) continue;
    uint32_t layer = 0;
    int side = 0;
    if (barrel) {
      layer = (rawId >> 20) & 0xf;
      int module = (rawId >> 2) & 0x3ff;
      side = (module < 5) ? -1 : 1;
    } else {
      int panel = (rawId >> 10) & 0x3;
      side = (panel == 1) ? -1 : 1;
    }
    uint32_t row, col;
    if (layer == 1) {
      col = (ww >> 15) & 0x3f;
      row = (ww >> 8) & 0x7f;
      if (!((row < 80) & (col < 52))) {
        d.errors.push_back({rawId, ww, 37, fedId});
        continue;
      }
    } else {
      uint32_t dcol = (ww >> 16) & 0x1f;
      uint32_t pxid = (ww >> 8) & 0xff;
      row = 80 - pxid / 2;
      col = dcol * 2 + pxid % 2;
      if (!((dcol < 26) & (2 <= pxid) & (pxid < 162))) {
        d.errors.push_back({rawId, ww, 37, fedId});
        continue;
      }
    }
    uint32_t gRow, gCol;
    frameConversion(barrel, side, layer, det.rocInDet, row, col, gRow, gCol);
    d.xx[i] = uint16_t(gRow);
    d.yy[i] = uint16_t(gCol);
    d.adc[i] = uint16_t(ww & 0xff);
    // pack(row, col, adc): Packing(11, 11, 0, 10) (SiPixelRawToClusterGPUKernel.h:130-137)
    uint32_t a = std::min<uint32_t>(d.adc[i], 1023u);
    d.pdigi[i] = (gRow << 0) | (gCol << 11) | (a << 22);
    d.moduleInd[i] = uint16_t(det.moduleId);
    d.rawIdArr[i] = rawId;
  }

  // ---- calibDigis (gpuCalibPixel.h:22-66), isRun2 = true
  const PfGainHeader& g = es.gain;
  for (uint32_t i = 0; i < nW; ++i) {
    uint16_t id = d.moduleInd[i];
    if (kInvId == id) continue;
    float conversionFactor = id < 96 ? 50.f : 47.f;
    float offset = id < 96 ? -670.f : -60.f;
    int row = d.xx[i], col = d.yy[i];
    // SiPixelGainForHLTonGPU::getPedAndGain (SiPixelGainForHLTonGPU.h:22-45)
    uint32_t first = g.rangeAndCols[id].first, second = g.rangeAndCols[id].second;
    int nCols = g.rangeAndCols[id].nCols;
    unsigned int lengthOfColumnData = (second - first) / nCols;
    unsigned int blocks = row / g.numberOfRowsAveragedOver;
    uint32_t o = first + col * lengthOfColumnData + 2 * blocks;
    uint8_t gb = es.gainPayload[o], pb = es.gainPayload[o + 1];
    bool isDead = pb == g.deadFlag, isNoisy = pb == g.noisyFlag;
    float pedestal = float(unsigned(pb)) * g.pedPrecision + g.minPed;
    float gain = float(unsigned(gb)) * g.gainPrecision + g.minGain;
    if (isDead | isNoisy) {
      d.moduleInd[i] = kInvId;
      d.adc[i] = 0;
    } else {
      float vcal = float(int(d.adc[i])) * gain - pedestal * gain;
      d.adc[i] = uint16_t(std::max(100, int(vcal * conversionFactor + offset)));
    }
  }

  clusterDigis(d, c, caps);
}

void clusterDigis(Digis& d, Clusters& c, const Caps& caps) {
  const uint32_t nW = d.nDigis;
  c.moduleStart.assign(PF_MAX_MODULES + 1, 0);
  c.clusInModule.assign(PF_MAX_MODULES, 0);
  c.moduleId.assign(PF_MAX_MODULES, 0);
  c.clusModuleStart.assign(PF_MAX_MODULES + 1, 0);
  // ---- countModules (gpuClustering.h:19-37)
  std::vector<uint32_t>& ms = c.moduleStart;
  for (uint32_t i = 0; i < nW; ++i) {
    d.clus[i] = int32_t(i);
    if (kInvId == d.moduleInd[i]) continue;
    int j = int(i) - 1;
    while (j >= 0 && d.moduleInd[j] == kInvId) --j;
    if (j < 0 || d.moduleInd[j] != d.moduleInd[i]) {
      uint32_t loc = ms[0];
      if (ms[0] < PF_MAX_MODULES) ms[0]++;
      ms[loc + 1] = i;
    }
  }
  d.nModules = ms[0];
  // a module in two runs: findClus and the rechits then overwrite its cluster
  // count and hit slots in loop order (and race in the reference's CUDA build)
  {
    std::vector<uint8_t> seen(PF_MAX_MODULES, 0);
    for (uint32_t module = 0; module < ms[0]; ++module) {
      uint16_t id = d.moduleInd[ms[1 + module]];
      if (id < PF_MAX_MODULES && seen[id]++)
        throw std::runtime_error("undefined in the reference: a module's digis in two separate runs");
    }
  }

  // ---- findClus (gpuClustering.h:40-273): connected components (|dx|<=1, |dy|<=1)
  // labelled by the lowest pixel index, numbered in ascending order of that index
  std::vector<int32_t> parent;
  for (uint32_t module = 0; module < ms[0]; ++module) {
    uint32_t firstPixel = ms[1 + module];
    uint16_t thisModuleId = d.moduleInd[firstPixel];
    uint32_t msize = nW;
    for (uint32_t i = firstPixel; i < nW; ++i) {
      if (d.moduleInd[i] == kInvId) continue;
      if (d.moduleInd[i] != thisModuleId) {
        msize = i;
        break;
      }
    }
    if (msize - firstPixel > PF_MAX_PIX_IN_MODULE) {
      std::printf("too many pixels in module %d: %d > %d\n", thisModuleId, msize - firstPixel, PF_MAX_PIX_IN_MODULE);
      msize = PF_MAX_PIX_IN_MODULE + firstPixel;
    }
    uint32_t np = msize - firstPixel;
    parent.assign(np, 0);
    for (uint32_t k = 0; k < np; ++k) parent[k] = int32_t(k);
    auto find = [&](int32_t k) {
      while (parent[k] != k) {
        parent[k] = parent[parent[k]];
        k = parent[k];
      }
      return k;
    };
    // column buckets
    std::vector<std::vector<uint32_t>> colPix(418);
    for (uint32_t k = 0; k < np; ++k) {
      uint32_t i = firstPixel + k;
      if (d.moduleInd[i] == kInvId) continue;
      colPix[d.yy[i] & 511].push_back(k);
    }
    for (uint32_t y = 0; y < 417; ++y) {
      auto& a = colPix[y];
      for (size_t p = 0; p < a.size(); ++p) {
        uint32_t ki = a[p];
        int xi = d.xx[firstPixel + ki];
        auto link = [&](uint32_t kj) {
          if (std::abs(int(d.xx[firstPixel + kj]) - xi) > 1) return;
          int32_t ri = find(int32_t(ki)), rj = find(int32_t(kj));
          if (ri == rj) return;
          if (ri < rj)
            parent[rj] = ri;
          else
            parent[ri] = rj;
        };
        for (size_t q = p + 1; q < a.size(); ++q) link(a[q]);
        if (y + 1 < 418)
          for (uint32_t kj : colPix[y + 1]) link(kj);
      }
    }
    uint32_t found = 0;
    std::vector<int32_t> number(np, -1);
    for (uint32_t k = 0; k < np; ++k) {
      uint32_t i = firstPixel + k;
      if (d.moduleInd[i] == kInvId) continue;
      if (find(int32_t(k)) == int32_t(k)) number[k] = int32_t(found++);
    }
    for (uint32_t k = 0; k < np; ++k) {
      uint32_t i = firstPixel + k;
      if (d.moduleInd[i] == kInvId) {
        d.clus[i] = -9999;
        continue;
      }
      d.clus[i] = number[find(int32_t(k))];
    }
    c.clusInModule[thisModuleId] = found;
    c.moduleId[module] = thisModuleId;
  }

  // ---- clusterChargeCut (gpuClusterChargeCut.h:14-114)
  std::vector<int32_t> charge(PF_MAX_CLUS_PER_MODULE);
  std::vector<uint16_t> newclusId(PF_MAX_CLUS_PER_MODULE);
  std::vector<uint8_t> ok(PF_MAX_CLUS_PER_MODULE);
  for (uint32_t module = 0; module < ms[0]; ++module) {
    uint32_t firstPixel = ms[1 + module];
    uint16_t thisModuleId = d.moduleInd[firstPixel];
    uint32_t nclus = c.clusInModule[thisModuleId];
    if (nclus == 0) continue;
    if (nclus > uint32_t(PF_MAX_CLUS_PER_MODULE)) {
      std::printf("Warning too many clusters in module %d in block %d: %d > %d\n", thisModuleId, 0, nclus,
                  PF_MAX_CLUS_PER_MODULE);
      for (uint32_t i = firstPixel; i < nW; ++i) {
        if (d.moduleInd[i] == kInvId) continue;
        if (d.moduleInd[i] != thisModuleId) break;
        if (d.clus[i] >= PF_MAX_CLUS_PER_MODULE) {
          d.moduleInd[i] = kInvId;
          d.clus[i] = kInvId;
        }
      }
      nclus = PF_MAX_CLUS_PER_MODULE;
    }
    for (uint32_t k = 0; k < nclus; ++k) charge[k] = 0;
    for (uint32_t i = firstPixel; i < nW; ++i) {
      if (d.moduleInd[i] == kInvId) continue;
      if (d.moduleInd[i] != thisModuleId) break;
      // a pixel past the 4000-pixel cap of a module of at most 1024 clusters
      // still holds its initial index: the reference sums past its array
      if (uint32_t(d.clus[i]) >= nclus)
        throw std::runtime_error("undefined in the reference: a pixel beyond a module's 4000-pixel cap");
      charge[d.clus[i]] += d.adc[i];
    }
    int chargeCut = thisModuleId < 96 ? 2000 : 4000;
    for (uint32_t k = 0; k < nclus; ++k) newclusId[k] = ok[k] = charge[k] > chargeCut ? 1 : 0;
    for (uint32_t k = 1; k < nclus; ++k) newclusId[k] += newclusId[k - 1];
    if (nclus == newclusId[nclus - 1]) continue;
    c.clusInModule[thisModuleId] = newclusId[nclus - 1];
    for (uint32_t k = 0; k < nclus; ++k)
      if (0 == ok[k]) newclusId[k] = kInvId + 1;
    for (uint32_t i = firstPixel; i < nW; ++i) {
      if (d.moduleInd[i] == kInvId) continue;
      if (d.moduleInd[i] != thisModuleId) break;
      d.clus[i] = newclusId[d.clus[i]] - 1;
      if (d.clus[i] == kInvId) d.moduleInd[i] = kInvId;
    }
  }

  // ---- fillHitsModuleStart (SiPixelRawToClusterGPUKernel.cc:464-506)
  std::vector<uint32_t>& cms = c.clusModuleStart;
  cms[0] = 0;
  for (uint32_t i = 0; i < PF_MAX_MODULES; ++i) cms[i + 1] = std::min<uint32_t>(PF_MAX_CLUS_PER_MODULE, c.clusInModule[i]);
  for (uint32_t i = 1; i < PF_MAX_MODULES + 1; ++i) cms[i] += cms[i - 1];
  for (uint32_t i = 0; i < PF_MAX_MODULES + 1; ++i)
    if (cms[i] > caps.hits) cms[i] = caps.hits;
  c.nClusters = cms[PF_MAX_MODULES];
}

void makeHits(const ES& es, const Digis& d, const Clusters& c, Hits& h, const Caps& caps) {
  const uint32_t nHits = c.nClusters;
  h.nHits = nHits;
  h.xl.assign(nHits, 0);
  h.yl.assign(nHits, 0);
  h.xerr.assign(nHits, 0);
  h.yerr.assign(nHits, 0);
  h.xg.assign(nHits, 0);
  h.yg.assign(nHits, 0);
  h.zg.assign(nHits, 0);
  h.rg.assign(nHits, 0);
  h.charge.assign(nHits, 0);
  h.iphi.assign(nHits, 0);
  h.xsize.assign(nHits, 0);
  h.ysize.assign(nHits, 0);
  h.detInd.assign(nHits, 0);
  const PfBeamSpot& bs = es.bs;
  const PfCommonParams& cp = es.common;

  // average geometry corrected by the beam spot (gpuPixelRecHits.h:35-48)
  for (int il = 0; il < PF_N_LADDERS_BARREL; ++il) {
    h.agc.ladderZ[il] = es.ag.ladderZ[il] - bs.z;
    h.agc.ladderX[il] = es.ag.ladderX[il] - bs.x;
    h.agc.ladderY[il] = es.ag.ladderY[il] - bs.y;
    // unqualified sqrt(float) binds to sqrt(double) there; rounding to float equals sqrtf
    h.agc.ladderR[il] = float(std::sqrt(double(h.agc.ladderX[il] * h.agc.ladderX[il] + h.agc.ladderY[il] * h.agc.ladderY[il])));
    h.agc.ladderMinZ[il] = es.ag.ladderMinZ[il] - bs.z;
    h.agc.ladderMaxZ[il] = es.ag.ladderMaxZ[il] - bs.z;
  }
  h.agc.endCapZ[0] = es.ag.endCapZ[0] - bs.z;
  h.agc.endCapZ[1] = es.ag.endCapZ[1] - bs.z;

  // ---- getHits (gpuPixelRecHits.h:16-207)
  if (d.nModules) {
    const uint32_t nW = d.nDigis;
    for (uint32_t module = 0; module < c.moduleStart[0]; ++module) {
      uint32_t me = c.moduleId[module];
      int nclus = int(c.clusInModule[me]);
      if (0 == nclus) continue;
      const PfDetParams& dp = es.det[me];
      for (int startClus = 0; startClus < nclus; startClus += PF_MAX_HITS_IN_ITER) {
        uint32_t first = c.moduleStart[1 + module];
        int nIn = std::min(int(PF_MAX_HITS_IN_ITER), nclus - startClus);
        int lastClus = startClus + nIn;
        uint32_t minRow[PF_MAX_HITS_IN_ITER], maxRow[PF_MAX_HITS_IN_ITER], minCol[PF_MAX_HITS_IN_ITER],
            maxCol[PF_MAX_HITS_IN_ITER];
        int32_t Qfx[PF_MAX_HITS_IN_ITER], Qlx[PF_MAX_HITS_IN_ITER], Qfy[PF_MAX_HITS_IN_ITER],
            Qly[PF_MAX_HITS_IN_ITER], chg[PF_MAX_HITS_IN_ITER];
        for (int k = 0; k < nIn; ++k) {
          minRow[k] = minCol[k] = std::numeric_limits<uint32_t>::max();
          maxRow[k] = maxCol[k] = 0;
          chg[k] = Qfx[k] = Qlx[k] = Qfy[k] = Qly[k] = 0;
        }
        for (uint32_t i = first; i < nW; ++i) {
          uint16_t id = d.moduleInd[i];
          if (id == kInvId) continue;
          if (id != me) break;
          int cl = d.clus[i];
          if (cl < startClus || cl >= lastClus) continue;
          cl -= startClus;
          minRow[cl] = std::min<uint32_t>(minRow[cl], d.xx[i]);
          maxRow[cl] = std::max<uint32_t>(maxRow[cl], d.xx[i]);
          minCol[cl] = std::min<uint32_t>(minCol[cl], d.yy[i]);
          maxCol[cl] = std::max<uint32_t>(maxCol[cl], d.yy[i]);
        }
        for (uint32_t i = first; i < nW; ++i) {
          uint16_t id = d.moduleInd[i];
          if (id == kInvId) continue;
          if (id != me) break;
          int cl = d.clus[i];
          if (cl < startClus || cl >= lastClus) continue;
          cl -= startClus;
          int32_t ch = d.adc[i];  // min(adc, 65535)
          uint32_t x = d.xx[i], y = d.yy[i];
          chg[cl] += ch;
          if (minRow[cl] == x) Qfx[cl] += ch;
          if (maxRow[cl] == x) Qlx[cl] += ch;
          if (minCol[cl] == y) Qfy[cl] += ch;
          if (maxCol[cl] == y) Qly[cl] += ch;
        }
        uint32_t firstHit = c.clusModuleStart[me] + startClus;
        for (int ic = 0; ic < nIn; ++ic) {
          uint32_t hidx = firstHit + ic;
          if (hidx >= caps.hits) break;
          // pixelCPEforGPU::position (pixelCPEforGPU.h:176-259)
          uint16_t llx = uint16_t(minRow[ic] + 1), lly = uint16_t(minCol[ic] + 1);
          uint16_t urx = uint16_t(maxRow[ic]), ury = uint16_t(maxCol[ic]);
          uint16_t llxl = localX(llx), llyl = localY(lly), urxl = localX(urx), uryl = localY(ury);
          int mx = llxl + urxl, my = llyl + uryl;
          int xsize = int(urxl) + 2 - int(llxl);
          int ysize = int(uryl) + 2 - int(llyl);
          if (isBigPixX(uint16_t(minRow[ic]))) ++xsize;
          if (isBigPixX(uint16_t(maxRow[ic]))) ++xsize;
          if (isBigPixY(uint16_t(minCol[ic]))) ++ysize;
          if (isBigPixY(uint16_t(maxCol[ic]))) ++ysize;
          int unbalanceX = int(8. * std::abs(float(Qfx[ic] - Qlx[ic])) / float(Qfx[ic] + Qlx[ic]));
          int unbalanceY = int(8. * std::abs(float(Qfy[ic] - Qly[ic])) / float(Qfy[ic] + Qly[ic]));
          xsize = 8 * xsize - unbalanceX;
          ysize = 8 * ysize - unbalanceY;
          int16_t sxv = int16_t(std::min(xsize, 1023)), syv = int16_t(std::min(ysize, 1023));
          if (minRow[ic] == 0 || maxRow[ic] == 159) sxv = int16_t(-sxv);
          if (minCol[ic] == 0 || maxCol[ic] == 415) syv = int16_t(-syv);
          float xPos = dp.shiftX + cp.pitchX * (0.5f * float(mx) + float(-81));
          float yPos = dp.shiftY + cp.pitchY * (0.5f * float(my) + float(-54 * 4));
          float gvx = xPos - dp.x0, gvy = yPos - dp.y0, gvz = -1.f / dp.z0;
          float cotalpha = gvx * gvz, cotbeta = gvy * gvz;
          float thickness = dp.isBarrel ? cp.thicknessB : cp.thicknessE;
          float xcorr = correction(int(maxRow[ic] - minRow[ic]), Qfx[ic], Qlx[ic], llxl, urxl, dp.chargeWidthX,
                                   thickness, cotalpha, cp.pitchX, isBigPixX(uint16_t(minRow[ic])),
                                   isBigPixX(uint16_t(maxRow[ic])));
          float ycorr = correction(int(maxCol[ic] - minCol[ic]), Qfy[ic], Qly[ic], llyl, uryl, dp.chargeWidthY,
                                   thickness, cotbeta, cp.pitchY, isBigPixY(uint16_t(minCol[ic])),
                                   isBigPixY(uint16_t(maxCol[ic])));
          float xpos = xPos + xcorr, ypos = yPos + ycorr;
          // errorFromDB (pixelCPEforGPU.h:316-340)
          float xerr = 0.0050f, yerr = 0.0085f;
          uint32_t sx = maxRow[ic] - minRow[ic], sy = maxCol[ic] - minCol[ic];
          bool isEdgeX = minRow[ic] == 0 or maxRow[ic] == 159;
          bool isEdgeY = minCol[ic] == 0 or maxCol[ic] == 415;
          uint32_t ix = (0 == sx), iy = (0 == sy);
          ix += (0 == sx) && isBigPixX(uint16_t(minRow[ic]));
          iy += (0 == sy) && isBigPixY(uint16_t(minCol[ic]));
          if (!isEdgeX) xerr = dp.sx[ix];
          if (!isEdgeY) yerr = dp.sy[iy];
          h.charge[hidx] = chg[ic];
          h.detInd[hidx] = uint16_t(me);
          h.xl[hidx] = xpos;
          h.yl[hidx] = ypos;
          h.xsize[hidx] = sxv;
          h.ysize[hidx] = syv;
          h.xerr[hidx] = xerr * xerr;
          h.yerr[hidx] = yerr * yerr;
          // SOAFrame::toGlobal(x, y) (DataFormats/SOARotation.h:504-509)
          const PfFrame& f = dp.frame;
          float xg = f.R11 * xpos + f.R21 * ypos;
          float yg = f.R12 * xpos + f.R22 * ypos;
          float zg = f.R13 * xpos + f.R23 * ypos;
          xg += f.px;
          yg += f.py;
          zg += f.pz;
          xg -= bs.x;
          yg -= bs.y;
          zg -= bs.z;
          h.xg[hidx] = xg;
          h.yg[hidx] = yg;
          h.zg[hidx] = zg;
          h.rg[hidx] = std::sqrt(xg * xg + yg * yg);
          h.iphi[hidx] = unsafeAtan2s7(yg, xg);
        }
      }
    }
  }

  // ---- setHitsLayerStart (PixelRecHits.cc:15-28) and phi histogram (HistoContainer.h:18-73)
  h.phiOff.assign(10 * PF_PHI_BINS + 1, 0);
  h.phiBins.assign(nHits, 0);
  if (nHits) {
    for (int i = 0; i < 11; ++i) h.layerStart[i] = c.clusModuleStart[es.lg.layerStart[i]];
    auto layerOf = [&](uint32_t i) {
      int ih = int(std::upper_bound(h.layerStart, h.layerStart + 11, i) - h.layerStart) - 1;
      return ih;
    };
    auto bin = [](int16_t t) { return uint32_t((int(t) >> 9) & 127); };
    uint32_t nt = h.layerStart[10];
    for (uint32_t i = 0; i < nt; ++i) h.phiOff[bin(h.iphi[i]) + 128 * layerOf(i)]++;
    for (uint32_t b = 1; b < h.phiOff.size(); ++b) h.phiOff[b] += h.phiOff[b - 1];
    for (uint32_t i = 0; i < nt; ++i) {
      uint32_t b = bin(h.iphi[i]) + 128 * layerOf(i);
      uint32_t w = h.phiOff[b]--;
      h.phiBins[w - 1] = i;
    }
  }
}

}  // namespace oracle
