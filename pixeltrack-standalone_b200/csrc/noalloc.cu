// Vertex finding on caller-supplied tracks without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need a
// result: a module running per event inside a multi-stream framework that
// owns all device memory through its own caching allocator (cudaFree
// synchronises the whole device, so it is banned from the event loop), or a
// latency-critical path that must not stall on the allocator.  For them this
// entry point runs the chain's vertex finder (the same kernel the chain
// launches) with every temporary it needs in one file-scope device array
// that the library holds from load to exit on each GPU that loads it.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "pixgpu.h"
#include "pixgpu_internal.cuh"

namespace pixgpu {
namespace {

// Scratch layout: the per-event counters, then the two per-track scratch
// areas the vertex kernel uses for events above its shared-memory size, with
// the sizes that kernel carves (pixgpu_internal.cuh: kVtxScratchAWords,
// kVtxScratchBWords for kMaxVtxTracks tracks).
constexpr size_t kCountersBytes = 512;
constexpr size_t kScratchABytes = kVtxScratchAWords * 4;
constexpr size_t kScratchBBytes = kVtxScratchBWords * 4;
constexpr size_t kNoAllocBytes = kCountersBytes + kScratchABytes + kScratchBBytes;  // 1.25 MiB + 512 B
static_assert(sizeof(EventCounters) <= kCountersBytes, "counters do not fit their scratch slot");
static_assert(kNoAllocBytes <= 1310720 + 512, "the documented 1.25 MB bound of the static scratch");
// the tuple limit (n_tuples < kNoAllocMaxTuples + 1) and the reference's
// TrackSoA stride the one-event workspace uses
constexpr uint32_t kNoAllocMaxTuples = PF_TRACK_STRIDE - 1;  // 32767
static_assert(PF_TRACK_STRIDE <= kMaxVtxTracks, "n_tuples limit above the vertex scratch");

static __device__ __align__(256) unsigned char gVtxScratch[kNoAllocBytes];

// the counters the vertex kernel reads and accumulates into start fresh on every call
__global__ void kNoAllocInit(EventCounters* c, uint32_t nTuples) {
  EventCounters z{};
  z.nTuples = nTuples;
  *c = z;
}

constexpr int kMaxDevices = 64;
std::mutex gSetupMu;
unsigned char* gScratchAddr[kMaxDevices] = {};

// device address of the scratch array on the current device (looked up once per device)
cudaError_t scratchAddress(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(gSetupMu);
  if (!gScratchAddr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, gVtxScratch);
    if (e != cudaSuccess) return e;
    gScratchAddr[dev] = static_cast<unsigned char*>(p);
  }
  *out = gScratchAddr[dev];
  return cudaSuccess;
}

void setMessage(char* msg, size_t cap, const char* text) {
  if (msg && cap) std::snprintf(msg, cap, "%s", text);
}

}  // namespace
}  // namespace pixgpu

using namespace pixgpu;

extern "C" int pg_vertices_noalloc(const uint32_t* tuple_off, const uint8_t* quality, const float* pt,
                                   const float* state, const float* cov, uint32_t n_tuples, int16_t* idv, float* zv,
                                   float* wv, float* chi2, float* ptv2, int32_t* ndof, uint16_t* sort_ind,
                                   uint32_t* n_vertices, uint32_t* flags, void* stream, char* msg, size_t msg_cap) {
  setMessage(msg, msg_cap, "");
  if (!tuple_off || !quality || !pt || !state || !cov || !idv || !zv || !wv || !chi2 || !ptv2 || !ndof ||
      !sort_ind || !n_vertices) {
    setMessage(msg, msg_cap, "pg_vertices_noalloc: null pointer argument");
    return PG_ERR_ARG;
  }
  if (n_tuples > kNoAllocMaxTuples) {
    setMessage(msg, msg_cap, "pg_vertices_noalloc: n_tuples above 32767, the static scratch limit");
    return PG_ERR_CAPACITY;
  }
  unsigned char* base = nullptr;
  cudaError_t e = scratchAddress(&base);
  if (e != cudaSuccess) {
    setMessage(msg, msg_cap, cudaGetErrorString(e));
    return PG_ERR_CUDA;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // a one-event workspace: the caller's arrays plus the static scratch
  Workspace ws{};
  ws.maxEvents = 1;
  // the reference's capacities: a TrackSoA stride of 32768 tuples
  ws.cap = referenceCaps();
  ws.ev = reinterpret_cast<EventCounters*>(base);
  ws.tupleOff = const_cast<uint32_t*>(tuple_off);
  ws.quality = const_cast<uint8_t*>(quality);
  ws.pt = const_cast<float*>(pt);
  ws.state = const_cast<float*>(state);
  ws.cov = const_cast<float*>(cov);
  ws.idv = idv;
  ws.zv = zv;
  ws.wv = wv;
  ws.vchi2 = chi2;
  ws.ptv2 = ptv2;
  ws.ndof = ndof;
  ws.sortInd = sort_ind;
  ws.scratchA = reinterpret_cast<uint32_t*>(base + kCountersBytes);
  ws.scratchB = reinterpret_cast<uint32_t*>(base + kCountersBytes + kScratchABytes);
  kNoAllocInit<<<1, 1, 0, s>>>(ws.ev, n_tuples);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = runVertices(ws, 1, s);
  EventCounters c{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&c, ws.ev, sizeof(c), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    setMessage(msg, msg_cap, cudaGetErrorString(e));
    return PG_ERR_CUDA;
  }
  *n_vertices = c.nVertices;
  if (flags) *flags = c.flags;
  return PG_OK;
}
