// Transfer of the vertices to the host (the reference module:
// src/cuda/plugin-PixelVertexFinding/PixelVertexSoAFromCUDA.cc): the event's
// ZVertexSoA filled from the chain's vertex products.
#include <algorithm>
#include <memory>
#include <stdexcept>

#include "CUDADataFormats/ZVertexHeterogeneous.h"
#include "Framework/EDProducer.h"
#include "Framework/Event.h"
#include "Framework/EventSetup.h"
#include "Framework/PluginFactory.h"

#include "B200Products.h"

class PixelVertexSoAFromCUDA : public edm::EDProducer {
public:
  explicit PixelVertexSoAFromCUDA(edm::ProductRegistry& reg)
      : tokenVertex_(reg.consumes<pixelb200::ZVertexB200>()),
        tokenTrack_(reg.consumes<pixelb200::PixelTrackB200>()),
        tokenSoA_(reg.produces<ZVertexHeterogeneous>()) {}

private:
  void produce(edm::Event& iEvent, edm::EventSetup const&) override {
    auto const& v = iEvent.get(tokenVertex_);
    auto const& t = iEvent.get(tokenTrack_);
    const pixelb200::EventRef& ev = *v.event;
    const uint32_t nv = v.nVertices;
    if (nv > ZVertexSoA::MAXVTX) throw std::runtime_error("B200 chain: more vertices than ZVertexSoA holds");
    auto soa = std::make_unique<ZVertexSoA>();
    soa->init();
    const auto zv = ev.product<float>("zv");
    const auto wv = ev.product<float>("wv");
    const auto chi2 = ev.product<float>("vchi2");
    const auto ptv2 = ev.product<float>("ptv2");
    const auto ndof = ev.product<int32_t>("ndof");
    const auto sortInd = ev.product<uint16_t>("sortInd");
    const auto idv = ev.product<int16_t>("idv");
    if (zv.size() < nv || ndof.size() < nv || sortInd.size() < nv)
      throw std::runtime_error("B200 chain: vertex products inconsistent with the vertex count");
    std::copy(zv.begin(), zv.begin() + nv, soa->zv);
    std::copy(wv.begin(), wv.begin() + nv, soa->wv);
    std::copy(chi2.begin(), chi2.begin() + nv, soa->chi2);
    std::copy(ptv2.begin(), ptv2.begin() + nv, soa->ptv2);
    std::copy(ndof.begin(), ndof.begin() + nv, soa->ndof);
    std::copy(sortInd.begin(), sortInd.begin() + nv, soa->sortInd);
    const size_t nt = std::min<size_t>({idv.size(), size_t(t.nTuples), size_t(ZVertexSoA::MAXTRACKS)});
    std::copy(idv.begin(), idv.begin() + nt, soa->idv);
    soa->nvFinal = nv;
    iEvent.emplace(tokenSoA_, std::move(soa));
  }

  edm::EDGetTokenT<pixelb200::ZVertexB200> tokenVertex_;
  edm::EDGetTokenT<pixelb200::PixelTrackB200> tokenTrack_;
  edm::EDPutTokenT<ZVertexHeterogeneous> tokenSoA_;
};

DEFINE_FWK_MODULE(PixelVertexSoAFromCUDA);
