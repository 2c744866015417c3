// Product types of the B200 pixel chain inside the reference framework
// (the edm::EventProcessor of cms-patatrack/pixeltrack-standalone).
//
// EventSetup products: the file images the four ESProducers read (the
// reference's cablingMap.bin, fedIds.bin, gain.bin, cpefast.bin and
// beamspot.bin layouts, include/pixfmt.h); the chain builds its device
// conditions from them once per job.
//
// Event products of the device modules: the reference's CUDA modules put
// cms::cuda::Product<SiPixelDigisCUDA>, ... here the whole chain of one event
// runs in the batch that SiPixelRawToClusterCUDA's acquire() submitted, and
// each module puts a handle on that event's device-resident results
// (EventRef), with the counts its consumers read on the host.  The transfer
// modules turn them into the reference's host SoA products.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace pixelb200 {

  // ---------------------------------------------------------------- EventSetup
  struct CablingMapImage {
    std::vector<uint8_t> bytes;  // cablingMap.bin
  };
  struct FedIdsImage {
    std::vector<uint8_t> bytes;  // fedIds.bin
    std::vector<uint32_t> fedIds;
  };
  struct GainImage {
    std::vector<uint8_t> bytes;  // gain.bin
  };
  struct CPEImage {
    std::vector<uint8_t> bytes;  // cpefast.bin
  };
  struct BeamSpotImage {
    std::vector<uint8_t> bytes;  // beamspot.bin
  };

  class Batch;

  // One event of a batch on the device: valid once the batch has finished
  // (the acquire() of SiPixelRawToClusterCUDA returns before; its produce()
  // runs after).  Keeps the batch slot alive; the slot is released when the
  // last event of the batch has dropped its handles.
  class EventRef {
  public:
    std::shared_ptr<Batch> batch;
    uint32_t index = 0;  // the event's place in the batch
    // a copy of a product of this event (pg_slot_product names)
    template <typename T>
    std::vector<T> product(const char* name) const;
    uint32_t scalar(const char* name) const;

  private:
    std::vector<uint8_t> bytes(const char* name, int elemBytes) const;
  };

  // ---------------------------------------------------------------- Event (device side)
  struct SiPixelDigisB200 {
    std::shared_ptr<EventRef> event;
    uint32_t nModules = 0, nDigis = 0;
  };
  struct SiPixelClustersB200 {
    std::shared_ptr<EventRef> event;
    uint32_t nClusters = 0;
  };
  struct TrackingRecHit2DB200 {
    std::shared_ptr<EventRef> event;
    uint32_t nHits = 0;
  };
  struct PixelTrackB200 {
    std::shared_ptr<EventRef> event;
    uint32_t nTuples = 0;  // tuples before the first empty one (the reference's track count)
  };
  struct ZVertexB200 {
    std::shared_ptr<EventRef> event;
    uint32_t nVertices = 0;
  };

  template <typename T>
  std::vector<T> EventRef::product(const char* name) const {
    std::vector<uint8_t> b = bytes(name, int(sizeof(T)));
    std::vector<T> out(b.size() / sizeof(T));
    if (!out.empty()) std::memcpy(out.data(), b.data(), out.size() * sizeof(T));
    return out;
  }

}  // namespace pixelb200
