// FED scan on the device: the S-Link header/trailer checks of the FED loop
// (SiPixelRawToClusterCUDA.cc:87-136 with ErrorChecker.cc:38-91) and the
// word concatenation of WordFedAppender (SiPixelRawToClusterGPUKernel.cc:36-47),
// from the whole FED buffers of a batch.
//
// The host only walks each record's FED directory (Source.cc:9-21) and
// copies every FED block, header to trailer, to an 8-byte-aligned place in
// the pinned raw buffer; its table gives, for each event and each FED of the
// ES list (in that order), the block's first 64-bit word and length.  Then:
//   kFedScan  one CTA per event: each thread walks the header and trailer
//             words of its FEDs (CRC-modified bit, start/end markers, source
//             id, fragment length, more-headers/trailers bits), the CTA scans
//             the payload lengths in FED order and writes the event's word
//             count; the framing errors go to a per-event list in FED order.
//   kFedCopy  (FED groups x events): each CTA adds up the counts of the
//             events before its own (the event's first word), one CTA per
//             event writes wordOffsets, and each warp copies one FED payload
//             as 64-bit word pairs (four loads in flight per lane) with their
//             one-byte FED index per pair.
#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kCopyThreads = 256;

struct FedWalk {
  uint32_t first, len;  // payload: first 64-bit word (within the block), 32-bit word count
  uint32_t nErr;
};

// header/trailer walk of one FED block (n64 > 0); emit(word64, type) for each
// framing error in the serial loop's order
template <typename Emit>
__device__ __forceinline__ FedWalk walkFed(const uint64_t* p, uint32_t n64, uint32_t fedId, Emit&& emit) {
  FedWalk r{0, 0, 0};
  // checkCRC: the CRC-modified bit of the last word drops the FED
  if ((p[n64 - 1] >> 2) & 1) {
    emit(p[n64 - 1], 39u);
    r.nErr = 1;
    return r;
  }
  // checkHeader: start marker 0x5 (else the headers end, unrecorded), source
  // id, more-headers bit; bounded by the block
  int h = -1;
  bool more = true;
  while (more && h + 1 < int(n64)) {
    ++h;
    const uint64_t v = p[h];
    if (((uint32_t(v >> 32) >> 28) & 0xf) != 0x5) break;
    if (((uint32_t(v) >> 8) & 0xfff) != fedId) {
      emit(v, 32u);
      ++r.nErr;
    }
    more = (uint32_t(v) >> 3) & 1;
  }
  // checkTrailer: end marker 0xa (else type 33 and the trailers end),
  // fragment length against the block's 64-bit words, more-trailers bit
  int t = int(n64);
  more = true;
  while (more && t > 0) {
    --t;
    const uint64_t v = p[t];
    if (((uint32_t(v >> 32) >> 28) & 0xf) != 0xa) {
      emit(v, 33u);
      ++r.nErr;
      break;
    }
    if ((uint32_t(v >> 32) & 0x00ffffffu) != n64) {
      emit(v, 34u);
      ++r.nErr;
    }
    more = (uint32_t(v) >> 3) & 1;
  }
  if (t >= h + 1) {  // header and trailer overlap: no payload (undefined in the reference)
    r.first = uint32_t(h + 1);
    r.len = 2u * uint32_t(t - (h + 1));
  }
  return r;
}

__global__ void __launch_bounds__(kScanThreads) kFedScan(Workspace ws) {
  __shared__ uint32_t sh[33];
  const FedScanBuffers& fs = ws.scan;
  const uint32_t e = blockIdx.x, F = fs.nFeds;
  const uint2* tab = fs.tab + size_t(e) * F;
  uint32_t* len = fs.len + size_t(e) * F;
  uint32_t* src = fs.src + size_t(e) * F;
  uint32_t* dst = fs.dst + size_t(e) * F;
  // a contiguous run of FEDs per thread, so that the block scan keeps FED order
  const uint32_t per = (F + kScanThreads - 1) / kScanThreads;
  const uint32_t j0 = min(F, threadIdx.x * per), j1 = min(F, j0 + per);
  uint32_t sumLen = 0, sumErr = 0;
  auto none = [](uint64_t, uint32_t) {};
  for (uint32_t j = j0; j < j1; ++j) {
    const uint2 t = tab[j];
    FedWalk w{0, 0, 0};
    if (t.y > 0) w = walkFed(fs.raw64 + t.x, t.y, fs.fedIds[j], none);
    len[j] = w.len;
    src[j] = t.x + w.first;
    dst[j] = w.nErr;  // error count until the offsets replace it
    sumLen += w.len;
    sumErr += w.nErr;
  }
  uint32_t totLen, totErr;
  uint32_t offLen = blockExclusiveScan(sumLen, sh, &totLen);
  uint32_t offErr = blockExclusiveScan(sumErr, sh, &totErr);
  PfFormatterError* fmt = fs.fmt + size_t(e) * kFmtErrCap;
  for (uint32_t j = j0; j < j1; ++j) {
    const uint32_t nErr = dst[j];
    if (nErr && fs.recordErrors) {
      const uint2 t = tab[j];
      uint32_t k = offErr;
      walkFed(fs.raw64 + t.x, t.y, fs.fedIds[j], [&](uint64_t v, uint32_t type) {
        if (k < kFmtErrCap) fmt[k] = PfFormatterError{v, type, fs.fedIds[j]};
        ++k;
      });
    }
    offErr += nErr;
    dst[j] = offLen;
    offLen += len[j];
  }
  if (threadIdx.x == 0) {
    fs.evWords[e] = totLen;
    fs.fmtCount[e] = fs.recordErrors ? totErr : 0u;
  }
}

__global__ void __launch_bounds__(kCopyThreads) kFedCopy(Workspace ws, uint32_t nEvents) {
  __shared__ uint32_t sBase;
  const FedScanBuffers& fs = ws.scan;
  const uint32_t e = blockIdx.y, F = fs.nFeds;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp == 0) {
    uint32_t s = 0;
    for (uint32_t k = lane; k < e; k += 32) s += fs.evWords[k];
    s = __reduce_add_sync(0xffffffffu, s);
    if (lane == 0) sBase = s;
  }
  __syncthreads();
  const uint32_t base = sBase;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ws.wordOffsets[e] = base;
    if (e == nEvents - 1) ws.wordOffsets[nEvents] = base + fs.evWords[e];
  }
  const uint32_t* len = fs.len + size_t(e) * F;
  const uint32_t* src = fs.src + size_t(e) * F;
  const uint32_t* dst = fs.dst + size_t(e) * F;
  uint64_t* words64 = reinterpret_cast<uint64_t*>(ws.words);
  uint8_t* fed = ws.fedIds;
  const uint32_t warps = kCopyThreads / 32;
  for (uint32_t j = blockIdx.x * warps + warp; j < F; j += gridDim.x * warps) {
    const uint32_t pairs = len[j] / 2;
    const uint64_t* s = fs.raw64 + src[j];
    const uint32_t d = (base + dst[j]) / 2;  // word pairs; every payload length is even
    const uint8_t idx = uint8_t(fs.fedIds[j] - 1200u);
    // four independent loads in flight per lane
    for (uint32_t i0 = 0; i0 < pairs; i0 += 128) {
      uint64_t v[4];
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t i = i0 + u * 32 + lane;
        v[u] = i < pairs ? s[i] : 0ull;
      }
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t i = i0 + u * 32 + lane;
        if (i < pairs) {
          words64[d + i] = v[u];
          fed[d + i] = idx;
        }
      }
    }
  }
}

}  // namespace

void launchFedScan(Workspace& ws, uint32_t nEvents, cudaStream_t stream) {
  PG_PROBED("kFedScan", stream, kFedScan<<<nEvents, kScanThreads, 0, stream>>>(ws));
  // one warp per FED (~100 FEDs of a few hundred word pairs each)
  const uint32_t sx = max(1u, (ws.scan.nFeds + kCopyThreads / 32 - 1) / (kCopyThreads / 32));
  PG_PROBED("kFedCopy", stream, kFedCopy<<<dim3(tunedGrid(ws, kTuneFedCopy, sx), nEvents), kCopyThreads, 0, stream>>>(ws, nEvents));
}

}  // namespace pixgpu
