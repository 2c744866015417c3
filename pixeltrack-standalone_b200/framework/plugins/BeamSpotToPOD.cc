// The beam spot of the EventSetup as an event product (the reference's
// BeamSpotToPOD / BeamSpotToCUDA: the chain's device copy of the beam spot is
// part of its conditions, uploaded with them).
#include "DataFormats/BeamSpotPOD.h"
#include "Framework/EDProducer.h"
#include "Framework/Event.h"
#include "Framework/EventSetup.h"
#include "Framework/PluginFactory.h"

class BeamSpotToPOD : public edm::EDProducer {
public:
  explicit BeamSpotToPOD(edm::ProductRegistry& reg) : bsPutToken_{reg.produces<BeamSpotPOD>()} {}
  void produce(edm::Event& iEvent, const edm::EventSetup& iSetup) override {
    iEvent.emplace(bsPutToken_, iSetup.get<BeamSpotPOD>());
  }

private:
  const edm::EDPutTokenT<BeamSpotPOD> bsPutToken_;
};

DEFINE_FWK_MODULE(BeamSpotToPOD);
