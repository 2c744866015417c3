// SiPixelRecHitCUDA on the B200 chain (the reference module:
// plugin-SiPixelRecHits/SiPixelRecHitCUDA.cc).  The hits of the event were
// made in the batch SiPixelRawToClusterCUDA submitted (with the beam spot of
// the chain's conditions); this module puts the handle on them.
#include "DataFormats/BeamSpotPOD.h"
#include "Framework/EDProducer.h"
#include "Framework/Event.h"
#include "Framework/EventSetup.h"
#include "Framework/PluginFactory.h"

#include "B200Products.h"

class SiPixelRecHitCUDA : public edm::EDProducer {
public:
  explicit SiPixelRecHitCUDA(edm::ProductRegistry& reg)
      : tBeamSpot_(reg.consumes<BeamSpotPOD>()),
        tokenClusters_(reg.consumes<pixelb200::SiPixelClustersB200>()),
        tokenDigis_(reg.consumes<pixelb200::SiPixelDigisB200>()),
        tokenHit_(reg.produces<pixelb200::TrackingRecHit2DB200>()) {}

private:
  void produce(edm::Event& iEvent, edm::EventSetup const&) override {
    auto const& clusters = iEvent.get(tokenClusters_);
    iEvent.emplace(tokenHit_, pixelb200::TrackingRecHit2DB200{clusters.event, clusters.event->scalar("nHits")});
  }

  edm::EDGetTokenT<BeamSpotPOD> tBeamSpot_;
  edm::EDGetTokenT<pixelb200::SiPixelClustersB200> tokenClusters_;
  edm::EDGetTokenT<pixelb200::SiPixelDigisB200> tokenDigis_;
  edm::EDPutTokenT<pixelb200::TrackingRecHit2DB200> tokenHit_;
};

DEFINE_FWK_MODULE(SiPixelRecHitCUDA);
