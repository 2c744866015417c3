// Test driver of the reference's edm::EventProcessor (src/serial/bin) with the
// B200 chain's plugins: the module path of the reference's CUDA program
// (src/cuda/bin/main.cc) with its transfer modules, plus
// SiPixelDigisSoAFromCUDA for the host digis and clusters the serial
// CountValidator reads.  Checker infrastructure: built with oracle/ref/Makefile
// (target fw) from the reference's framework sources.
//
//   edm_b200 --data DIR [--numberOfStreams NS] [--maxEvents ME] [--warmupEvents WE] [--validation]
#include <chrono>
#include <cstdlib>
#include <filesystem>
#include <iostream>
#include <string>
#include <vector>

#include <tbb/task_arena.h>

#include "EventProcessor.h"

int main(int argc, char** argv) {
  std::vector<std::string> args(argv, argv + argc);
  int numberOfStreams = 1, maxEvents = -1, warmupEvents = 0;
  bool validation = false;
  std::filesystem::path datadir;
  for (size_t i = 1; i < args.size(); ++i) {
    if (args[i] == "--numberOfStreams" && i + 1 < args.size())
      numberOfStreams = std::stoi(args[++i]);
    else if (args[i] == "--maxEvents" && i + 1 < args.size())
      maxEvents = std::stoi(args[++i]);
    else if (args[i] == "--warmupEvents" && i + 1 < args.size())
      warmupEvents = std::stoi(args[++i]);
    else if (args[i] == "--data" && i + 1 < args.size())
      datadir = args[++i];
    else if (args[i] == "--validation")
      validation = true;
    else {
      std::cout << "Invalid parameter " << args[i] << std::endl;
      return EXIT_FAILURE;
    }
  }
  if (datadir.empty() || !std::filesystem::exists(datadir)) {
    std::cout << "Data directory '" << datadir << "' does not exist" << std::endl;
    return EXIT_FAILURE;
  }
  std::vector<std::string> edmodules = {"BeamSpotToPOD",          "SiPixelRawToClusterCUDA", "SiPixelDigisSoAFromCUDA",
                                        "SiPixelRecHitCUDA",      "CAHitNtupletCUDA",        "PixelTrackSoAFromCUDA",
                                        "PixelVertexProducerCUDA", "PixelVertexSoAFromCUDA"};
  std::vector<std::string> esmodules = {"BeamSpotESProducer", "SiPixelFedCablingMapGPUWrapperESProducer",
                                        "SiPixelGainCalibrationForHLTGPUESProducer", "PixelCPEFastESProducer"};
  if (validation) edmodules.emplace_back("CountValidator");
  try {
    edm::EventProcessor processor(warmupEvents, maxEvents, -1, numberOfStreams, edmodules, esmodules, datadir,
                                  validation);
    std::cout << "Processing " << processor.maxEvents() << " events with " << numberOfStreams
              << " concurrent events." << std::endl;
    tbb::task_arena arena(1);
    arena.execute([&] { processor.warmUp(); });
    auto start = std::chrono::steady_clock::now();
    arena.execute([&] { processor.runToCompletion(); });
    auto stop = std::chrono::steady_clock::now();
    processor.endJob();
    const double t = std::chrono::duration<double>(stop - start).count();
    std::cout << "Processed " << processor.processedEvents() << " events in " << t << " seconds, throughput "
              << processor.processedEvents() / t << " events/s" << std::endl;
  } catch (std::exception& e) {
    std::cout << "\n----------\nCaught exception\n" << e.what() << std::endl;
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}
