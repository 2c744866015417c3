// The process-wide B200 chain behind the framework modules: one pg_ctx per
// job (libpixgpu.so, include/pixgpu.h), built from the ESProducers' images on
// first use, and a service thread that batches the events the streams submit
// and reports each one when its batch has finished.
//
// Continuous batching: every acquire() queues its event; whenever a batch
// slot is free the service submits all queued events (up to the batch size)
// as one batch, so the events of concurrent streams share launches, and new
// events queue while earlier batches run.  The completion callback runs on the
// service thread; the framework hands it to its own task queue
// (WaitingTaskWithArenaHolder::doneWaiting).
#pragma once

#include <condition_variable>
#include <deque>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

#include "B200Products.h"
#include "pixgpu.h"

namespace edm {
  class EventSetup;
}

namespace pixelb200 {

  class ChainService;

  class Batch {
  public:
    Batch(ChainService* svc, uint32_t slot) : svc_(svc), slot_(slot) {}
    ~Batch();
    uint32_t slot() const { return slot_; }
    ChainService* service() const { return svc_; }

  private:
    ChainService* svc_;
    uint32_t slot_;
  };

  class ChainService {
  public:
    using Done = std::function<void(std::exception_ptr)>;

    // the job's chain, created from the EventSetup images on the first call
    static ChainService& get(edm::EventSetup const& es);

    ~ChainService();

    // FED ids of the cabling (the FED loop's order)
    std::vector<uint32_t> const& fedIds() const { return fedIds_; }

    // queues one raw.bin record; `ref` is filled and `done` called (on the
    // service thread) once the batch that holds it has finished
    void submit(std::vector<uint8_t> raw, std::shared_ptr<EventRef> ref, Done done);

    // serialised access to the C ABI
    std::vector<uint8_t> product(uint32_t slot, uint32_t k, const char* name, int elemBytes);
    void release(uint32_t slot);

  private:
    explicit ChainService(edm::EventSetup const& es);
    void loop();

    struct Pending {
      std::vector<uint8_t> raw;
      std::shared_ptr<EventRef> ref;
      Done done;
    };
    struct InFlight {
      std::shared_ptr<Batch> batch;
      std::vector<Pending> events;
    };

    pg_ctx* ctx_ = nullptr;
    uint32_t maxBatch_ = 0;
    std::vector<uint32_t> fedIds_;
    std::mutex abiMu_;  // every pg_* call on ctx_
    std::mutex mu_;     // pending_ and stop_
    std::condition_variable cv_;
    std::deque<Pending> pending_;
    std::vector<InFlight> inflight_;  // the service thread's own
    bool stop_ = false;
    std::thread thread_;
  };

}  // namespace pixelb200
