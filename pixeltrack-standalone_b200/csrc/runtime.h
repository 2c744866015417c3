// Host-side runtime of the C ABI: the context, its batch slots, the
// device-resident event pool and the helpers shared by capi.cu, pool.cu and
// serve.cu.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pixgpu.h"
#include "pixgpu_internal.cuh"
#include "pixgpu_results.h"

namespace pixgpu {

// one event of a pooled batch: where its words sit in the pool and where they
// go in the slot's batch buffer (word offsets; all even)
struct PoolRef {
  uint32_t src, n, dst, pad;
};

enum class SlotState { kFree, kBusy };

// A batch slot: one workspace, one stream, pinned staging and the mapped
// result region.  A slot carries one batch at a time.
struct Slot {
  void* dmem = nullptr;
  Workspace ws{};
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;      // end of the chain + result packing
  cudaEvent_t gathered = nullptr;  // pooled inputs copied out of the pool
  uint32_t* hWords = nullptr;      // pinned staging of unpacked words
  uint8_t* hFed = nullptr;
  uint32_t* hOffsets = nullptr;
  PoolRef* hRefs = nullptr;        // pinned
  PoolRef* dRefs = nullptr;        // device
  uint8_t* hRes = nullptr;         // mapped pinned result region [maxEvents][kResultStride]
  uint8_t* dRes = nullptr;         // its device alias
  std::map<uint32_t, cudaGraphExec_t> graphs;  // captured chain per batch size
  std::vector<uint32_t> poolHandles;           // pool entries gathered by the current batch
  KernelProbe* probe = nullptr;                // kernel timing events (when a probe is set)
  std::map<uint32_t, uint32_t> probeUsed;      // timed launches inside each captured graph
  uint32_t lastProbeUsed = 0;                  // timed launches of the current batch
  uint32_t nEvents = 0;
  bool staged = false;
  SlotState state = SlotState::kFree;
  // formatter errors of the current batch, host-scan mode: event k's are
  // [fmtOff[k], fmtOff[k + 1])
  std::vector<PfFormatterError> fmtErrors;
  std::vector<uint32_t> fmtOff;
  // device FED scan: its device buffers and the pinned FED blocks and table
  void* dScan = nullptr;
  uint64_t* hRaw = nullptr;
  uint2* hTab = nullptr;
};

// A pinned buffer that holds one unpacked event on its way into the pool.
struct Stager {
  uint32_t* hWords = nullptr;
  uint8_t* hFed = nullptr;
  cudaEvent_t copied = nullptr;
  bool used = false;
};

struct PoolEntry {
  uint32_t start = 0, nWords = 0, extent = 0;
  bool live = false;
  bool submitted = false;            // part of a batch (released once gathered)
  uint64_t seq = 0;                  // upload order
  cudaEvent_t uploaded = nullptr;
};

// Device-resident input pool: FED words of admitted events, first-fit extents.
struct Pool {
  uint32_t* dWords = nullptr;
  uint8_t* dFed = nullptr;
  uint32_t capWords = 0;
  uint64_t freeWords = 0;
  std::map<uint32_t, uint32_t> freeList;  // extent start -> length (words)
  std::vector<PoolEntry> entries;
  std::vector<uint32_t> freeHandles;
  std::vector<Stager> stagers;
  uint32_t nextStager = 0;
  uint64_t seq = 0;
  cudaStream_t upload = nullptr;
  std::mutex mu;
};

}  // namespace pixgpu

struct HostES {
  std::vector<uint32_t> fedIds;
  std::vector<uint32_t> scanFeds;  // the FEDs the loop visits, in order (fedId 40 and ids >= 4096 skipped)
};

struct pg_ctx {
  int device = 0;
  pg_config cfg{};
  pixgpu::Caps caps{};  // per-event capacities resolved from cfg
  HostES hes;
  void* esMem = nullptr;
  pixgpu::DeviceES des{};
  std::vector<pixgpu::Slot> slots;
  pixgpu::Pool pool;
  std::map<uint32_t, pixgpu::LaunchTuning> tuning;  // launch tuning per batch size (tune.cu)
  std::string probeName;  // kernel timed by the probe ("" = none)
  std::string err;
  std::mutex errMu;  // guards err: the serving loop's threads report errors concurrently
  std::mutex mu;  // slot bookkeeping (the serving loop's threads share it)
};

namespace pixgpu {

int fail(pg_ctx* c, int code, const std::string& msg);
// the capacities a configuration asks for (0 fields: the reference's); false
// when a field is below the reference's value or beyond the index widths
bool resolveCaps(const pg_config& cfg, Caps* out);
// the context's last error message (a copy taken under errMu)
std::string lastError(pg_ctx* c);
// the launch tuning for batches of n events: n's table, else the largest tuned size below n, else defaults
LaunchTuning tuningFor(const pg_ctx* c, uint32_t n);
int cudaFail(pg_ctx* c, cudaError_t e, const char* where);
// FED loop of one raw record on the host; fmt (may be null) receives the
// framing errors
int unpackRaw(const std::vector<uint32_t>& fedIds, const uint8_t* raw, size_t n, uint32_t* words, uint8_t* fed,
              uint32_t cap, uint32_t* nWordsOut, std::vector<PfFormatterError>* fmt = nullptr);
// chain + result packing for the slot's current batch (graph or plain launches)
int launchBatch(pg_ctx* c, Slot& s);
// captures the chain for n events on slot s once (no-op when present)
int captureGraphFor(pg_ctx* c, Slot& s, uint32_t n);
// a free slot index, or -1
int findFreeSlot(pg_ctx* c);
// pool set-up / teardown and reclamation of extents whose gather has finished
int poolCreate(pg_ctx* c, uint64_t words);
void poolDestroy(pg_ctx* c);
void poolReclaimSlot(pg_ctx* c, Slot& s);
void launchGather(Workspace& ws, const uint32_t* poolWords, const uint8_t* poolFed, const PoolRef* refs,
                  uint32_t nEvents, cudaStream_t stream);

}  // namespace pixgpu
