#include "ChainService.h"

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <string>

#include "Framework/EventSetup.h"

namespace pixelb200 {

  namespace {
    uint32_t envOr(const char* name, uint32_t def) {
      const char* v = std::getenv(name);
      return v && *v ? uint32_t(std::strtoul(v, nullptr, 10)) : def;
    }
    std::mutex gCreateMu;
    std::unique_ptr<ChainService> gService;
  }  // namespace

  Batch::~Batch() { svc_->release(slot_); }

  std::vector<uint8_t> EventRef::bytes(const char* name, int elemBytes) const {
    if (!batch) throw std::runtime_error("B200 chain: event product read before its batch finished");
    return batch->service()->product(batch->slot(), index, name, elemBytes);
  }

  uint32_t EventRef::scalar(const char* name) const {
    std::vector<uint32_t> v = product<uint32_t>(name);
    if (v.size() != 1) throw std::runtime_error(std::string("B200 chain: no scalar product ") + name);
    return v[0];
  }

  ChainService& ChainService::get(edm::EventSetup const& es) {
    std::lock_guard<std::mutex> lk(gCreateMu);
    if (!gService) gService.reset(new ChainService(es));
    return *gService;
  }

  ChainService::ChainService(edm::EventSetup const& es) {
    const auto& cab = es.get<CablingMapImage>();
    const auto& fed = es.get<FedIdsImage>();
    const auto& gain = es.get<GainImage>();
    const auto& cpe = es.get<CPEImage>();
    const auto& bs = es.get<BeamSpotImage>();
    fedIds_ = fed.fedIds;
    pg_es_images img{cab.bytes.data(), cab.bytes.size(), gain.bytes.data(), gain.bytes.size(),
                     cpe.bytes.data(), cpe.bytes.size(), bs.bytes.data(),   bs.bytes.size(),
                     fed.bytes.data(), fed.bytes.size()};
    pg_config cfg;
    pg_default_config(&cfg);
    // events per batch and batches in flight (PIXB200_MAX_BATCH, PIXB200_SLOTS)
    maxBatch_ = std::max(1u, envOr("PIXB200_MAX_BATCH", 16));
    cfg.max_events = maxBatch_;
    cfg.max_words_per_batch = maxBatch_ * 300000u;
    cfg.slots = std::max(1u, envOr("PIXB200_SLOTS", 3));
    cfg.device = int(envOr("PIXB200_DEVICE", 0));
    int rc = pg_create(&img, &cfg, &ctx_);
    if (rc != PG_OK) throw std::runtime_error("B200 chain: pg_create failed with status " + std::to_string(rc));
    thread_ = std::thread([this] { loop(); });
  }

  ChainService::~ChainService() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    if (thread_.joinable()) thread_.join();
    inflight_.clear();
    std::lock_guard<std::mutex> lk(abiMu_);
    pg_destroy(ctx_);
  }

  void ChainService::submit(std::vector<uint8_t> raw, std::shared_ptr<EventRef> ref, Done done) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      pending_.push_back(Pending{std::move(raw), std::move(ref), std::move(done)});
    }
    cv_.notify_all();
  }

  std::vector<uint8_t> ChainService::product(uint32_t slot, uint32_t k, const char* name, int elemBytes) {
    std::lock_guard<std::mutex> lk(abiMu_);
    size_t count = 0;
    int elem = 0;
    int rc = pg_slot_product(ctx_, slot, k, name, nullptr, 0, &count, &elem);
    if (rc != PG_OK)
      throw std::runtime_error(std::string("B200 chain: product ") + name + ": " + pg_last_error(ctx_));
    if (elem != elemBytes)
      throw std::runtime_error(std::string("B200 chain: product ") + name + " has " + std::to_string(elem) +
                               "-byte elements");
    std::vector<uint8_t> out(count * size_t(elem));
    rc = pg_slot_product(ctx_, slot, k, name, out.data(), out.size(), &count, &elem);
    if (rc != PG_OK)
      throw std::runtime_error(std::string("B200 chain: product ") + name + ": " + pg_last_error(ctx_));
    return out;
  }

  void ChainService::release(uint32_t slot) {
    std::lock_guard<std::mutex> lk(abiMu_);
    pg_release(ctx_, slot);
  }

  void ChainService::loop() {
    for (;;) {
      std::vector<std::pair<Done, std::exception_ptr>> calls;
      bool idle = true;
      // finished batches: their events are complete
      for (size_t i = 0; i < inflight_.size();) {
        int q;
        {
          std::lock_guard<std::mutex> lk(abiMu_);
          q = pg_query(ctx_, inflight_[i].batch->slot());
        }
        if (q == PG_ERR_BUSY) {
          ++i;
          continue;
        }
        idle = false;
        std::exception_ptr ex;
        if (q != PG_OK) {
          std::lock_guard<std::mutex> lk(abiMu_);
          ex = std::make_exception_ptr(std::runtime_error(std::string("B200 chain: batch failed: ") +
                                                          pg_last_error(ctx_)));
        }
        for (uint32_t k = 0; k < inflight_[i].events.size(); ++k) {
          Pending& p = inflight_[i].events[k];
          p.ref->batch = inflight_[i].batch;
          p.ref->index = k;
          calls.emplace_back(std::move(p.done), ex);
        }
        inflight_.erase(inflight_.begin() + long(i));
      }
      // the events queued meanwhile, as batches on the free slots
      std::vector<Pending> take;
      {
        std::unique_lock<std::mutex> lk(mu_);
        if (stop_ && pending_.empty() && inflight_.empty()) return;
        while (!pending_.empty() && take.size() < maxBatch_) {
          take.push_back(std::move(pending_.front()));
          pending_.pop_front();
        }
      }
      if (!take.empty()) {
        std::vector<const uint8_t*> raws;
        std::vector<size_t> sizes;
        for (auto& p : take) {
          raws.push_back(p.raw.data());
          sizes.push_back(p.raw.size());
        }
        uint32_t slot = 0;
        int rc;
        {
          std::lock_guard<std::mutex> lk(abiMu_);
          rc = pg_submit(ctx_, uint32_t(take.size()), raws.data(), sizes.data(), &slot);
        }
        if (rc == PG_OK) {
          idle = false;
          inflight_.push_back(InFlight{std::make_shared<Batch>(this, slot), std::move(take)});
        } else if (rc == PG_ERR_BUSY) {
          // no free slot: put them back in front, in order
          std::lock_guard<std::mutex> lk(mu_);
          for (auto it = take.rbegin(); it != take.rend(); ++it) pending_.push_front(std::move(*it));
        } else {
          std::string msg;
          {
            std::lock_guard<std::mutex> lk(abiMu_);
            msg = pg_last_error(ctx_);
          }
          auto ex = std::make_exception_ptr(std::runtime_error("B200 chain: submit failed: " + msg));
          for (auto& p : take) calls.emplace_back(std::move(p.done), ex);
          idle = false;
        }
      }
      for (auto& c : calls) c.first(c.second);
      if (idle) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait_for(lk, std::chrono::microseconds(inflight_.empty() ? 2000 : 20));
      }
    }
  }

}  // namespace pixelb200
