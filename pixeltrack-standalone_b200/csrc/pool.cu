// Device-resident input pool: events are unpacked on the host once, copied
// into a first-fit pool of FED words on the upload stream, and later gathered
// into a slot's batch buffer by one kernel.  The pool's capacity is the
// admission limit of the serving loop.
#include <algorithm>
#include <cstring>

#include "runtime.h"

namespace pixgpu {

namespace {

constexpr uint32_t kExtentAlign = 64;  // words (256 bytes)
constexpr uint32_t kStagers = 16;

// grid (blocks per event, events): 8-byte copies of the words, bytes of the
// FED indices, and the batch's word offsets
__global__ void kGatherPool(Workspace ws, const uint32_t* __restrict__ poolWords, const uint8_t* __restrict__ poolFed,
                            const PoolRef* __restrict__ refs, uint32_t nEvents) {
  const uint32_t e = blockIdx.y;
  const PoolRef r = refs[e];
  const uint2* src = reinterpret_cast<const uint2*>(poolWords + r.src);
  uint2* dst = reinterpret_cast<uint2*>(ws.words + r.dst);
  const uint32_t n2 = r.n / 2;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) dst[i] = src[i];
  const uint8_t* fs = poolFed + r.src / 2;
  uint8_t* fd = ws.fedIds + r.dst / 2;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) fd[i] = fs[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ws.wordOffsets[e] = r.dst;
    if (e == nEvents - 1) ws.wordOffsets[nEvents] = r.dst + r.n;
  }
}

void freeExtent(Pool& p, uint32_t start, uint32_t len) {
  auto it = p.freeList.emplace(start, len).first;
  auto next = std::next(it);
  if (next != p.freeList.end() && it->first + it->second == next->first) {
    it->second += next->second;
    p.freeList.erase(next);
  }
  if (it != p.freeList.begin()) {
    auto prev = std::prev(it);
    if (prev->first + prev->second == it->first) {
      prev->second += it->second;
      p.freeList.erase(it);
    }
  }
  p.freeWords += len;
}

bool takeExtent(Pool& p, uint32_t len, uint32_t* start) {
  for (auto it = p.freeList.begin(); it != p.freeList.end(); ++it) {
    if (it->second >= len) {
      *start = it->first;
      uint32_t rest = it->second - len, s2 = it->first + len;
      p.freeList.erase(it);
      if (rest) p.freeList.emplace(s2, rest);
      p.freeWords -= len;
      return true;
    }
  }
  return false;
}

void releaseEntry(Pool& p, uint32_t h) {
  PoolEntry& en = p.entries[h];
  freeExtent(p, en.start, en.extent);
  en.live = false;
  en.submitted = false;
  p.freeHandles.push_back(h);
}

// extents of batches whose gather has finished (caller holds p.mu)
void reclaimGathered(pg_ctx* c) {
  for (auto& s : c->slots) {
    if (s.poolHandles.empty() || cudaEventQuery(s.gathered) != cudaSuccess) continue;
    for (uint32_t h : s.poolHandles) releaseEntry(c->pool, h);
    s.poolHandles.clear();
  }
}

}  // namespace

void launchGather(Workspace& ws, const uint32_t* poolWords, const uint8_t* poolFed, const PoolRef* refs,
                  uint32_t nEvents, cudaStream_t stream) {
  PG_PROBED("kGatherPool", stream, kGatherPool<<<dim3(16, nEvents), 256, 0, stream>>>(ws, poolWords, poolFed, refs, nEvents));
}

int poolCreate(pg_ctx* c, uint64_t words) {
  Pool& p = c->pool;
  const uint32_t maxWords = c->caps.fedWords;
  if (words < maxWords || words > (uint64_t(1) << 31)) return fail(c, PG_ERR_ARG, "pool size");
  p.capWords = uint32_t(words) & ~(kExtentAlign - 1);
  if (cudaMalloc(&p.dWords, size_t(p.capWords) * 4) != cudaSuccess ||
      cudaMalloc(&p.dFed, size_t(p.capWords) / 2 + 16) != cudaSuccess)
    return fail(c, PG_ERR_NOMEM, "pool allocation");
  if (cudaStreamCreateWithFlags(&p.upload, cudaStreamNonBlocking) != cudaSuccess)
    return fail(c, PG_ERR_CUDA, "upload stream");
  p.freeList.clear();
  p.freeList.emplace(0u, p.capWords);
  p.freeWords = p.capWords;
  p.stagers.resize(kStagers);
  for (auto& st : p.stagers) {
    if (cudaMallocHost(&st.hWords, size_t(maxWords) * 4) != cudaSuccess ||
        cudaMallocHost(&st.hFed, size_t(maxWords) / 2 + 16) != cudaSuccess ||
        cudaEventCreateWithFlags(&st.copied, cudaEventDisableTiming) != cudaSuccess)
      return fail(c, PG_ERR_NOMEM, "pool staging buffers");
  }
  return PG_OK;
}

void poolDestroy(pg_ctx* c) {
  Pool& p = c->pool;
  if (p.upload) cudaStreamSynchronize(p.upload);
  for (auto& st : p.stagers) {
    if (st.hWords) cudaFreeHost(st.hWords);
    if (st.hFed) cudaFreeHost(st.hFed);
    if (st.copied) cudaEventDestroy(st.copied);
  }
  p.stagers.clear();
  for (auto& en : p.entries)
    if (en.uploaded) cudaEventDestroy(en.uploaded);
  p.entries.clear();
  if (p.dWords) cudaFree(p.dWords);
  if (p.dFed) cudaFree(p.dFed);
  if (p.upload) cudaStreamDestroy(p.upload);
  p.dWords = nullptr;
  p.dFed = nullptr;
  p.upload = nullptr;
}

void poolReclaimSlot(pg_ctx* c, Slot& s) {
  if (!c->pool.dWords) return;
  std::lock_guard<std::mutex> lk(c->pool.mu);
  for (uint32_t h : s.poolHandles) releaseEntry(c->pool, h);
  s.poolHandles.clear();
}

// Unpacks one raw record into a free stager; returns its index in *stager.
int poolStage(pg_ctx* c, const uint8_t* raw, size_t size, uint32_t* stager, uint32_t* nWords) {
  Pool& p = c->pool;
  if (!p.dWords) return fail(c, PG_ERR_ARG, "context has no pool");
  int k = -1;
  {
    std::lock_guard<std::mutex> lk(p.mu);
    for (uint32_t i = 0; i < kStagers && k < 0; ++i) {
      uint32_t j = (p.nextStager + i) % kStagers;
      Stager& st = p.stagers[j];
      if (!st.used && cudaEventQuery(st.copied) == cudaSuccess) k = int(j);
    }
    if (k < 0) return fail(c, PG_ERR_BUSY, "all pool staging buffers in flight");
    p.stagers[k].used = true;
    p.nextStager = (uint32_t(k) + 1) % kStagers;
  }
  Stager& st = p.stagers[k];
  int rc = unpackRaw(c->hes.fedIds, raw, size, st.hWords, st.hFed, c->caps.fedWords, nWords);
  if (rc != PG_OK) {
    std::lock_guard<std::mutex> lk(p.mu);
    st.used = false;
    return fail(c, rc, rc == PG_ERR_CAPACITY ? "event too large" : "malformed raw record");
  }
  *stager = uint32_t(k);
  return PG_OK;
}

// Moves a staged event into the pool (PG_ERR_NOMEM when it does not fit now).
int poolCommit(pg_ctx* c, uint32_t stager, uint32_t nWords, uint32_t* handle) {
  Pool& p = c->pool;
  std::lock_guard<std::mutex> lk(p.mu);
  Stager& st = p.stagers[stager];
  uint32_t need = std::max(kExtentAlign, (nWords + kExtentAlign - 1) & ~(kExtentAlign - 1));
  uint32_t start = 0;
  if (!takeExtent(p, need, &start)) {
    reclaimGathered(c);
    if (!takeExtent(p, need, &start)) return fail(c, PG_ERR_NOMEM, "pool full");
  }
  uint32_t h;
  if (!p.freeHandles.empty()) {
    h = p.freeHandles.back();
    p.freeHandles.pop_back();
  } else {
    h = uint32_t(p.entries.size());
    p.entries.emplace_back();
    if (cudaEventCreateWithFlags(&p.entries[h].uploaded, cudaEventDisableTiming) != cudaSuccess) {
      p.entries.pop_back();
      freeExtent(p, start, need);
      return fail(c, PG_ERR_CUDA, "pool event");
    }
  }
  PoolEntry& en = p.entries[h];
  en.start = start;
  en.nWords = nWords;
  en.extent = need;
  en.live = true;
  en.submitted = false;
  en.seq = ++p.seq;
  cudaError_t e = cudaSuccess;
  if (nWords) {
    e = cudaMemcpyAsync(p.dWords + start, st.hWords, size_t(nWords) * 4, cudaMemcpyHostToDevice, p.upload);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(p.dFed + start / 2, st.hFed, size_t(nWords) / 2, cudaMemcpyHostToDevice, p.upload);
  }
  if (e == cudaSuccess) e = cudaEventRecord(st.copied, p.upload);
  if (e == cudaSuccess) e = cudaEventRecord(en.uploaded, p.upload);
  st.used = false;
  if (e != cudaSuccess) {
    releaseEntry(p, h);
    return cudaFail(c, e, "pool upload");
  }
  *handle = h;
  return PG_OK;
}

void poolUnstage(pg_ctx* c, uint32_t stager) {
  std::lock_guard<std::mutex> lk(c->pool.mu);
  c->pool.stagers[stager].used = false;
}

}  // namespace pixgpu

using namespace pixgpu;

extern "C" {

int pg_pool_put(pg_ctx* c, const uint8_t* raw, size_t size, uint32_t* handle) {
  if (!c || !raw || !handle) return PG_ERR_ARG;
  cudaSetDevice(c->cfg.device);
  uint32_t st = 0, nw = 0;
  int rc = poolStage(c, raw, size, &st, &nw);
  if (rc != PG_OK) return rc;
  rc = poolCommit(c, st, nw, handle);
  if (rc != PG_OK) poolUnstage(c, st);
  return rc;
}

int pg_pool_release(pg_ctx* c, uint32_t handle) {
  if (!c || !c->pool.dWords) return PG_ERR_ARG;
  Pool& p = c->pool;
  std::lock_guard<std::mutex> lk(p.mu);
  if (handle >= p.entries.size() || !p.entries[handle].live) return fail(c, PG_ERR_ARG, "pool handle");
  if (p.entries[handle].submitted) return fail(c, PG_ERR_ARG, "pool handle belongs to a submitted batch");
  cudaEventSynchronize(p.entries[handle].uploaded);
  // a kept event may still be read by a gather in flight
  for (auto& s : c->slots)
    if (s.state == SlotState::kBusy) cudaEventSynchronize(s.gathered);
  releaseEntry(p, handle);
  return PG_OK;
}

int pg_pool_info(pg_ctx* c, uint64_t* capWords, uint64_t* freeWords, uint32_t* liveEvents) {
  if (!c) return PG_ERR_ARG;
  Pool& p = c->pool;
  std::lock_guard<std::mutex> lk(p.mu);
  if (p.dWords) reclaimGathered(c);
  if (capWords) *capWords = p.capWords;
  if (freeWords) *freeWords = p.freeWords;
  if (liveEvents) {
    uint32_t n = 0;
    for (auto& en : p.entries) n += en.live ? 1 : 0;
    *liveEvents = n;
  }
  return PG_OK;
}

int pg_submit_pooled(pg_ctx* c, uint32_t nEvents, const uint32_t* handles, uint32_t flags, uint32_t* slotOut) {
  const bool keep = (flags & PG_POOL_KEEP) != 0;
  if (!c || !handles || !slotOut || !c->pool.dWords) return PG_ERR_ARG;
  if (nEvents == 0 || nEvents > c->cfg.max_events) return fail(c, PG_ERR_CAPACITY, "batch size");
  cudaSetDevice(c->cfg.device);
  Pool& p = c->pool;
  int k;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    k = findFreeSlot(c);
    if (k < 0) return fail(c, PG_ERR_BUSY, "no free slot");
    c->slots[k].state = SlotState::kBusy;
  }
  Slot& s = c->slots[k];
  uint32_t total = 0, lastH = handles[0];
  cudaEvent_t lastUpload = nullptr;
  {
    std::lock_guard<std::mutex> lk(p.mu);
    int bad = 0;
    for (uint32_t i = 0; i < nEvents && !bad; ++i) {
      uint32_t h = handles[i];
      if (h >= p.entries.size() || !p.entries[h].live || p.entries[h].submitted) {
        bad = 1;
        break;
      }
      for (uint32_t j = 0; j < i; ++j)
        if (handles[j] == h) bad = 1;
      if (bad) break;
      const PoolEntry& en = p.entries[h];
      s.hRefs[i] = PoolRef{en.start, en.nWords, total, 0};
      total += en.nWords;
      if (en.seq > p.entries[lastH].seq) lastH = h;
    }
    if (!bad && total > c->cfg.max_words_per_batch) bad = 2;
    if (bad) {
      std::lock_guard<std::mutex> lk2(c->mu);
      s.state = SlotState::kFree;
      return fail(c, bad == 2 ? PG_ERR_CAPACITY : PG_ERR_ARG,
                  bad == 2 ? "batch words exceed the slot" : "pool handle invalid, repeated or already submitted");
    }
    if (!keep)
      for (uint32_t i = 0; i < nEvents; ++i) p.entries[handles[i]].submitted = true;
    lastUpload = p.entries[lastH].uploaded;
  }
  cudaError_t e = cudaMemcpyAsync(s.dRefs, s.hRefs, size_t(nEvents) * sizeof(PoolRef), cudaMemcpyHostToDevice,
                                  s.stream);
  // the upload stream is in order: the newest upload covers all earlier ones
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s.stream, lastUpload, 0);
  if (e == cudaSuccess) {
    launchGather(s.ws, p.dWords, p.dFed, s.dRefs, nEvents, s.stream);
    e = cudaEventRecord(s.gathered, s.stream);
  }
  {
    // only now may the extents be reclaimed once `gathered` has completed
    std::lock_guard<std::mutex> lk(p.mu);
    if (!keep) s.poolHandles.assign(handles, handles + nEvents);
  }
  int rc = e == cudaSuccess ? PG_OK : cudaFail(c, e, "pool gather");
  if (rc == PG_OK) {
    s.nEvents = nEvents;
    s.staged = true;
    rc = launchBatch(c, s);
  }
  if (rc != PG_OK) {
    cudaStreamSynchronize(s.stream);
    poolReclaimSlot(c, s);
    std::lock_guard<std::mutex> lk(c->mu);
    s.state = SlotState::kFree;
    return rc;
  }
  *slotOut = uint32_t(k);
  return PG_OK;
}

}  // extern "C"
