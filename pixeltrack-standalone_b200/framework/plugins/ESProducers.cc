// The four ESProducers of the pixel chain: the file images of the
// conditions, read once per job from the data directory as the reference's
// ESProducers read them (SiPixelFedCablingMapGPUWrapperESProducer.cc,
// SiPixelGainCalibrationForHLTGPUESProducer.cc, PixelCPEFastESProducer.cc,
// BeamSpotESProducer.cc: the same file names and layouts, include/pixfmt.h).
// The chain uploads them to the device when the first event arrives
// (ChainService); BeamSpotPOD is put as the reference puts it.
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <memory>
#include <stdexcept>

#include "DataFormats/BeamSpotPOD.h"
#include "Framework/ESPluginFactory.h"
#include "Framework/ESProducer.h"
#include "Framework/EventSetup.h"

#include "B200Products.h"

namespace {
  std::vector<uint8_t> readFile(std::filesystem::path const& p) {
    std::ifstream in(p, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + p.string());
    return std::vector<uint8_t>(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
  }
}  // namespace

class SiPixelFedCablingMapGPUWrapperESProducer : public edm::ESProducer {
public:
  explicit SiPixelFedCablingMapGPUWrapperESProducer(std::filesystem::path const& datadir) : data_(datadir) {}
  void produce(edm::EventSetup& eventSetup) override {
    auto fed = std::make_unique<pixelb200::FedIdsImage>();
    fed->bytes = readFile(data_ / "fedIds.bin");
    uint32_t n = 0;
    if (fed->bytes.size() < 4) throw std::runtime_error("fedIds.bin: truncated");
    std::memcpy(&n, fed->bytes.data(), 4);
    if (fed->bytes.size() < 4 + size_t(n) * 4) throw std::runtime_error("fedIds.bin: truncated");
    fed->fedIds.resize(n);
    std::memcpy(fed->fedIds.data(), fed->bytes.data() + 4, size_t(n) * 4);
    auto cab = std::make_unique<pixelb200::CablingMapImage>();
    cab->bytes = readFile(data_ / "cablingMap.bin");
    eventSetup.put(std::move(fed));
    eventSetup.put(std::move(cab));
  }

private:
  std::filesystem::path data_;
};

class SiPixelGainCalibrationForHLTGPUESProducer : public edm::ESProducer {
public:
  explicit SiPixelGainCalibrationForHLTGPUESProducer(std::filesystem::path const& datadir) : data_(datadir) {}
  void produce(edm::EventSetup& eventSetup) override {
    auto gain = std::make_unique<pixelb200::GainImage>();
    gain->bytes = readFile(data_ / "gain.bin");
    eventSetup.put(std::move(gain));
  }

private:
  std::filesystem::path data_;
};

class PixelCPEFastESProducer : public edm::ESProducer {
public:
  explicit PixelCPEFastESProducer(std::filesystem::path const& datadir) : data_(datadir) {}
  void produce(edm::EventSetup& eventSetup) override {
    auto cpe = std::make_unique<pixelb200::CPEImage>();
    cpe->bytes = readFile(data_ / "cpefast.bin");
    eventSetup.put(std::move(cpe));
  }

private:
  std::filesystem::path data_;
};

class BeamSpotESProducer : public edm::ESProducer {
public:
  explicit BeamSpotESProducer(std::filesystem::path const& datadir) : data_(datadir) {}
  void produce(edm::EventSetup& eventSetup) override {
    auto img = std::make_unique<pixelb200::BeamSpotImage>();
    img->bytes = readFile(data_ / "beamspot.bin");
    if (img->bytes.size() < sizeof(BeamSpotPOD)) throw std::runtime_error("beamspot.bin: truncated");
    auto bs = std::make_unique<BeamSpotPOD>();
    std::memcpy(bs.get(), img->bytes.data(), sizeof(BeamSpotPOD));
    eventSetup.put(std::move(bs));
    eventSetup.put(std::move(img));
  }

private:
  std::filesystem::path data_;
};

DEFINE_FWK_EVENTSETUP_MODULE(SiPixelFedCablingMapGPUWrapperESProducer);
DEFINE_FWK_EVENTSETUP_MODULE(SiPixelGainCalibrationForHLTGPUESProducer);
DEFINE_FWK_EVENTSETUP_MODULE(PixelCPEFastESProducer);
DEFINE_FWK_EVENTSETUP_MODULE(BeamSpotESProducer);
