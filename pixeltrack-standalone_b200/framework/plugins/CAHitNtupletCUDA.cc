// CAHitNtupletCUDA on the B200 chain (the reference module:
// plugin-PixelTriplets/CAHitNtupletCUDA.cc): the n-tuplets and their fits of
// the event, made in its batch, as a device-resident track product.
#include "Framework/EDProducer.h"
#include "Framework/Event.h"
#include "Framework/EventSetup.h"
#include "Framework/PluginFactory.h"

#include "B200Products.h"

class CAHitNtupletCUDA : public edm::EDProducer {
public:
  explicit CAHitNtupletCUDA(edm::ProductRegistry& reg)
      : tokenHit_(reg.consumes<pixelb200::TrackingRecHit2DB200>()),
        tokenTrack_(reg.produces<pixelb200::PixelTrackB200>()) {}

private:
  void produce(edm::Event& iEvent, edm::EventSetup const&) override {
    auto const& hits = iEvent.get(tokenHit_);
    iEvent.emplace(tokenTrack_, pixelb200::PixelTrackB200{hits.event, hits.event->scalar("nTuples")});
  }

  edm::EDGetTokenT<pixelb200::TrackingRecHit2DB200> tokenHit_;
  edm::EDPutTokenT<pixelb200::PixelTrackB200> tokenTrack_;
};

DEFINE_FWK_MODULE(CAHitNtupletCUDA);
