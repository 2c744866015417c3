// SiPixelRawToClusterCUDA on the B200 chain (the reference module:
// plugin-SiPixelClusterizer/SiPixelRawToClusterCUDA.cc, an
// edm::EDProducerExternalWork).  acquire() packs the event's pixel FEDs into
// a raw.bin record and queues it with the chain service, which runs it with
// the other streams' events as one batch: raw-to-digi through vertices in one
// captured launch sequence.  produce() runs once that batch has finished and
// puts the device-resident digis and clusters with their counts.
#include <cstring>
#include <memory>
#include <vector>

#include "DataFormats/FEDRawData.h"
#include "DataFormats/FEDRawDataCollection.h"
#include "Framework/EDProducer.h"
#include "Framework/Event.h"
#include "Framework/EventSetup.h"
#include "Framework/PluginFactory.h"

#include "B200Products.h"
#include "ChainService.h"

class SiPixelRawToClusterCUDA : public edm::EDProducerExternalWork {
public:
  explicit SiPixelRawToClusterCUDA(edm::ProductRegistry& reg)
      : rawGetToken_(reg.consumes<FEDRawDataCollection>()),
        digiPutToken_(reg.produces<pixelb200::SiPixelDigisB200>()),
        clusterPutToken_(reg.produces<pixelb200::SiPixelClustersB200>()) {}

private:
  void acquire(edm::Event const& iEvent, edm::EventSetup const& iSetup,
               edm::WaitingTaskWithArenaHolder holder) override {
    auto& chain = pixelb200::ChainService::get(iSetup);
    auto const& buffers = iEvent.get(rawGetToken_);
    // the FEDs of the cabling map, in its order, as one raw.bin record
    // (uint32 nfeds, then per FED: uint32 id, uint32 size, the bytes)
    std::vector<uint8_t> raw(4);
    uint32_t nfeds = 0;
    for (uint32_t fedId : chain.fedIds()) {
      FEDRawData const& data = buffers.FEDData(int(fedId));
      if (data.size() == 0) continue;
      const uint32_t head[2] = {fedId, uint32_t(data.size())};
      const size_t at = raw.size();
      raw.resize(at + 8 + data.size());
      std::memcpy(raw.data() + at, head, 8);
      std::memcpy(raw.data() + at + 8, data.data(), data.size());
      ++nfeds;
    }
    std::memcpy(raw.data(), &nfeds, 4);
    event_ = std::make_shared<pixelb200::EventRef>();
    chain.submit(std::move(raw), event_, [holder](std::exception_ptr e) mutable { holder.doneWaiting(e); });
  }

  void produce(edm::Event& iEvent, edm::EventSetup const&) override {
    auto ev = std::move(event_);
    pixelb200::SiPixelDigisB200 digis{ev, ev->scalar("nModules"), ev->scalar("nDigis")};
    pixelb200::SiPixelClustersB200 clusters{ev, ev->scalar("nClusters")};
    iEvent.emplace(digiPutToken_, std::move(digis));
    iEvent.emplace(clusterPutToken_, std::move(clusters));
  }

  edm::EDGetTokenT<FEDRawDataCollection> rawGetToken_;
  edm::EDPutTokenT<pixelb200::SiPixelDigisB200> digiPutToken_;
  edm::EDPutTokenT<pixelb200::SiPixelClustersB200> clusterPutToken_;
  std::shared_ptr<pixelb200::EventRef> event_;  // between acquire() and produce() of one event
};

DEFINE_FWK_MODULE(SiPixelRawToClusterCUDA);
