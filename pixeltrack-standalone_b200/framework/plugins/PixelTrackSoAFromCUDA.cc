// Transfer of the tracks to the host (the reference module:
// src/cuda/plugin-PixelTrackFitting/PixelTrackSoAFromCUDA.cc): the event's
// TrackSoA (pixelTrack::TrackSoA, PixelTrackHeterogeneous.h) filled from the
// chain's track products -- quality, chi2, state and covariance at the beam
// spot, eta, pt, and the hit and detector index containers.  Tuples beyond the
// stored ones keep the value-initialised zeros of the reference's SoA.
#include <cstring>
#include <memory>
#include <stdexcept>

#include "CUDADataFormats/PixelTrackHeterogeneous.h"
#include "Framework/EDProducer.h"
#include "Framework/Event.h"
#include "Framework/EventSetup.h"
#include "Framework/PluginFactory.h"

#include "B200Products.h"

class PixelTrackSoAFromCUDA : public edm::EDProducer {
public:
  explicit PixelTrackSoAFromCUDA(edm::ProductRegistry& reg)
      : tokenTrack_(reg.consumes<pixelb200::PixelTrackB200>()),
        tokenSoA_(reg.produces<PixelTrackHeterogeneous>()) {}

private:
  void produce(edm::Event& iEvent, edm::EventSetup const&) override {
    using TrackSoA = pixelTrack::TrackSoA;
    auto const& t = iEvent.get(tokenTrack_);
    const pixelb200::EventRef& ev = *t.event;
    const uint32_t n = t.nTuples;
    constexpr uint32_t S = TrackSoA::stride();
    if (n >= S) throw std::runtime_error("B200 chain: more tuples than the TrackSoA stride");
    const auto off = ev.product<uint32_t>("tupleOff");           // n + 1
    const auto hits = ev.product<uint32_t>("tupleHits");
    const auto dets = ev.product<uint16_t>("tupleDet");
    const auto q = ev.product<uint8_t>("quality");
    const auto st = ev.product<float>("state");                  // n x 5
    const auto cv = ev.product<float>("cov");                    // n x 15
    const auto pt = ev.product<float>("pt");
    const auto eta = ev.product<float>("eta");
    const auto chi2 = ev.product<float>("chi2");
    if (off.size() != n + 1 || q.size() < n || st.size() < 5 * size_t(n) || cv.size() < 15 * size_t(n))
      throw std::runtime_error("B200 chain: track products inconsistent with the tuple count");
    auto soa = std::make_unique<TrackSoA>();
    for (uint32_t i = 0; i < n; ++i) {
      soa->m_quality(i) = q[i];
      soa->chi2(i) = chi2[i];
      soa->pt(i) = pt[i];
      soa->eta(i) = eta[i];
      for (int k = 0; k < 5; ++k) soa->stateAtBS.state(i)(k) = st[5 * size_t(i) + k];
      for (int k = 0; k < 15; ++k) soa->stateAtBS.covariance(i)(k) = cv[15 * size_t(i) + k];
    }
    // HitContainer (OneToManyAssoc<uint16_t, S, 5 S>): offsets of the stored
    // tuples, every later bin empty at the total, as the reference's finalize
    const uint32_t total = off[n];
    if (hits.size() < total || dets.size() < total) throw std::runtime_error("B200 chain: tuple hits truncated");
    for (uint32_t b = 0; b <= S; ++b) {
      const uint32_t o = b <= n ? off[b] : total;
      soa->hitIndices.off[b] = o;
      soa->detIndices.off[b] = o;
    }
    for (uint32_t k = 0; k < total; ++k) {
      if (hits[k] > 0xffffu) throw std::runtime_error("B200 chain: hit index beyond the TrackSoA's 16 bits");
      soa->hitIndices.bins[k] = uint16_t(hits[k]);
      soa->detIndices.bins[k] = dets[k];
    }
    soa->m_nTracks = n;
    iEvent.emplace(tokenSoA_, std::move(soa));
  }

  edm::EDGetTokenT<pixelb200::PixelTrackB200> tokenTrack_;
  edm::EDPutTokenT<PixelTrackHeterogeneous> tokenSoA_;
};

DEFINE_FWK_MODULE(PixelTrackSoAFromCUDA);
