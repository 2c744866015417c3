// PixelVertexProducerCUDA on the B200 chain (the reference module:
// plugin-PixelVertexFinding/PixelVertexProducerCUDA.cc): the event's
// vertices, found in its batch, as a device-resident vertex product.
#include "Framework/EDProducer.h"
#include "Framework/Event.h"
#include "Framework/EventSetup.h"
#include "Framework/PluginFactory.h"

#include "B200Products.h"

class PixelVertexProducerCUDA : public edm::EDProducer {
public:
  explicit PixelVertexProducerCUDA(edm::ProductRegistry& reg)
      : tokenTrack_(reg.consumes<pixelb200::PixelTrackB200>()),
        tokenVertex_(reg.produces<pixelb200::ZVertexB200>()) {}

private:
  void produce(edm::Event& iEvent, edm::EventSetup const&) override {
    auto const& tracks = iEvent.get(tokenTrack_);
    iEvent.emplace(tokenVertex_, pixelb200::ZVertexB200{tracks.event, tracks.event->scalar("nVertices")});
  }

  edm::EDGetTokenT<pixelb200::PixelTrackB200> tokenTrack_;
  edm::EDPutTokenT<pixelb200::ZVertexB200> tokenVertex_;
};

DEFINE_FWK_MODULE(PixelVertexProducerCUDA);
