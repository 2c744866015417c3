// Transfer of the digis and clusters to the host (the reference module:
// src/cuda/plugin-SiPixelRawToDigi/SiPixelDigisSoAFromCUDA.cc, which copies
// pdigi, rawIdArr, adc and clus into a SiPixelDigisSoA).  The serial
// framework's consumers (CountValidator, HistoValidator) read
// SiPixelDigisSoA and SiPixelClustersSoA; the reference's CUDA program has no
// cluster transfer because its validators read the cluster count from the
// device product, so this module puts both host products.
#include <algorithm>
#include <cstring>
#include <stdexcept>

#include "CUDADataFormats/SiPixelClustersSoA.h"
#include "CUDADataFormats/SiPixelDigisSoA.h"
#include "Framework/EDProducer.h"
#include "Framework/Event.h"
#include "Framework/EventSetup.h"
#include "Framework/PluginFactory.h"

#include "B200Products.h"

namespace {
  template <typename T>
  void fill(T* dst, std::vector<T> const& src, size_t n) {
    if (src.size() < n) throw std::runtime_error("B200 chain: product shorter than its count");
    std::copy(src.begin(), src.begin() + n, dst);
  }
}  // namespace

class SiPixelDigisSoAFromCUDA : public edm::EDProducer {
public:
  explicit SiPixelDigisSoAFromCUDA(edm::ProductRegistry& reg)
      : digiGetToken_(reg.consumes<pixelb200::SiPixelDigisB200>()),
        clusterGetToken_(reg.consumes<pixelb200::SiPixelClustersB200>()),
        digiPutToken_(reg.produces<SiPixelDigisSoA>()),
        clusterPutToken_(reg.produces<SiPixelClustersSoA>()) {}

private:
  void produce(edm::Event& iEvent, edm::EventSetup const&) override {
    auto const& d = iEvent.get(digiGetToken_);
    auto const& c = iEvent.get(clusterGetToken_);
    const pixelb200::EventRef& ev = *d.event;
    const size_t n = d.nDigis;
    SiPixelDigisSoA digis(std::max<size_t>(n, 1));
    fill(digis.xx(), ev.product<uint16_t>("xx"), n);
    fill(digis.yy(), ev.product<uint16_t>("yy"), n);
    fill(digis.adc(), ev.product<uint16_t>("adc"), n);
    fill(digis.moduleInd(), ev.product<uint16_t>("moduleInd"), n);
    fill(digis.clus(), ev.product<int32_t>("clus"), n);
    fill(digis.pdigi(), ev.product<uint32_t>("pdigi"), n);
    fill(digis.rawIdArr(), ev.product<uint32_t>("rawIdArr"), n);
    digis.setNModulesDigis(d.nModules, d.nDigis);
    // per-module arrays (gpuClusteringConstants.h: MaxNumModules = 2000)
    constexpr size_t kModules = 2000;
    SiPixelClustersSoA clusters(kModules);
    fill(clusters.moduleStart(), c.event->product<uint32_t>("moduleStart"), kModules + 1);
    fill(clusters.clusInModule(), c.event->product<uint32_t>("clusInModule"), kModules);
    fill(clusters.moduleId(), c.event->product<uint32_t>("moduleId"), kModules);
    fill(clusters.clusModuleStart(), c.event->product<uint32_t>("clusModuleStart"), kModules + 1);
    clusters.setNClusters(c.nClusters);
    iEvent.emplace(digiPutToken_, std::move(digis));
    iEvent.emplace(clusterPutToken_, std::move(clusters));
  }

  edm::EDGetTokenT<pixelb200::SiPixelDigisB200> digiGetToken_;
  edm::EDGetTokenT<pixelb200::SiPixelClustersB200> clusterGetToken_;
  edm::EDPutTokenT<SiPixelDigisSoA> digiPutToken_;
  edm::EDPutTokenT<SiPixelClustersSoA> clusterPutToken_;
};

DEFINE_FWK_MODULE(SiPixelDigisSoAFromCUDA);
