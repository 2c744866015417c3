/*
 * pixfmt.h — binary layouts and constants shared by the B200 pixel chain,
 * its C-ABI callers, the synthetic-event generator and the CPU oracle.
 *
 * Every struct here is a byte-for-byte image of a record that the reference
 * ESProducers read from disk with a single `ifstream::read`, so a file written
 * from these structs is readable by the reference unchanged:
 *   cablingMap.bin : SiPixelFedCablingMapGPU (CondFormats/SiPixelFedCablingMapGPU.h:15-24)
 *                    + uint32 n + uint8 modToUnp[n]
 *                    (plugin-SiPixelClusterizer/SiPixelFedCablingMapGPUWrapperESProducer.cc:20-41)
 *   gain.bin       : SiPixelGainForHLTonGPU (CondFormats/SiPixelGainForHLTonGPU.h:16-61)
 *                    + uint32 nbytes + payload of {uint8 gain, uint8 ped} pairs
 *                    (plugin-SiPixelClusterizer/SiPixelGainCalibrationForHLTGPUESProducer.cc:20-30)
 *   cpefast.bin    : CommonParams, uint32 n, DetParams[n], AverageGeometry, LayerGeometry
 *                    (CondFormats/PixelCPEFast.cc:17-28)
 *   beamspot.bin   : BeamSpotPOD (DataFormats/BeamSpotPOD.h:12-20)
 *   fedIds.bin     : uint32 n + uint32 fedId[n]
 *   raw.bin        : per event: uint32 nfeds, then nfeds x (uint32 fedId, uint32 size, bytes)
 *                    (bin/Source.cc:9-21)
 * Paths above are relative to the reference's src/serial tree.
 */
#ifndef PIXFMT_H
#define PIXFMT_H

#include <stdint.h>

#ifdef __cplusplus
#define PF_ALIGN(n) alignas(n)
extern "C" {
#else
#define PF_ALIGN(n) _Alignas(n)
#endif

/* ---- detector / capacity constants (reference values) ---- */
enum {
  PF_MAX_FED = 150,                /* SiPixelFedCablingMapGPU.h:8 */
  PF_MAX_LINK = 48,                /* :9 */
  PF_MAX_ROC = 8,                  /* :10 */
  PF_MAX_SIZE = 150 * 48 * 8,      /* 57600 cabling slots */
  PF_MAX_WORD = 2000,              /* SiPixelRawToClusterGPUKernel.h:52 */
  PF_MAX_FED_WORDS = 150 * 2000,   /* SiPixelRawToClusterGPUKernel.cc:34 */
  PF_MAX_MODULES = 2000,           /* gpuClusteringConstants.h:24 (MaxNumModules) */
  PF_INV_ID = 9999,                /* gpuClusteringConstants.h:28 */
  PF_MAX_PIX_IN_MODULE = 4000,     /* gpuClustering.h:78 */
  PF_MAX_CLUS_PER_MODULE = 1024,   /* gpuClusteringConstants.h:22 */
  PF_MAX_HITS_IN_ITER = 160,       /* gpuClusteringConstants.h:20 */
  PF_MAX_HITS = 48 * 1024,         /* pixelGPUConstants::maxNumberOfHits */
  PF_N_MODULES = 1856,             /* phase1PixelTopology.h:24 */
  PF_N_LAYERS = 10,                /* phase1PixelTopology.h:25 */
  PF_N_LADDERS_BARREL = 148,       /* 1184 / 8 */
  PF_LAYER_INDEX_SIZE = 116,       /* 1856 / maxModuleStride(16) */
  PF_MAX_TUPLES = 24 * 1024,       /* CAConstants.h:22 */
  PF_MAX_DOUBLETS = 512 * 1024,    /* CAConstants.h:30 */
  PF_MAX_DOUBLETS_PARAM = 458752,  /* CAHitNtupletGeneratorOnGPU.cc:48 */
  PF_MAX_CELLS_PER_HIT = 128,      /* CAConstants.h:31 */
  PF_MAX_CELL_NEIGHBORS = 36,      /* CAConstants.h:51 */
  PF_MAX_CELL_TRACKS = 48,         /* CAConstants.h:52 */
  PF_MAX_ACTIVE_DOUBLETS = 65536,  /* CAConstants.h:40 maxNumOfActiveDoublets */
  PF_TRACK_STRIDE = 32 * 1024,     /* PixelTrackHeterogeneous.h:62 */
  PF_MAX_VTX = 1024,               /* ZVertexSoA.h:12 */
  PF_PHI_BINS = 128,               /* TrackingRecHit2DSOAView.h:21 */
  PF_N_PAIRS = 19                  /* gpuPixelDoublets.h:14 */
};

/* ---- ES records (byte images) ---- */

/* CondFormats/SiPixelFedCablingMapGPU.h:15-24: seven 128-byte-aligned arrays + size */
typedef struct PfCablingMap {
  PF_ALIGN(128) uint32_t fed[PF_MAX_SIZE];
  PF_ALIGN(128) uint32_t link[PF_MAX_SIZE];
  PF_ALIGN(128) uint32_t roc[PF_MAX_SIZE];
  PF_ALIGN(128) uint32_t rawId[PF_MAX_SIZE];
  PF_ALIGN(128) uint32_t rocInDet[PF_MAX_SIZE];
  PF_ALIGN(128) uint32_t moduleId[PF_MAX_SIZE];
  PF_ALIGN(128) uint8_t badRocs[PF_MAX_SIZE];
  PF_ALIGN(128) uint32_t size;
} PfCablingMap;

/* CondFormats/SiPixelGainForHLTonGPU.h:16-61 (DecodingStructure {gain, ped}) */
typedef struct PfRangeAndCols {
  uint32_t first;  /* byte offset of the module's block */
  uint32_t second; /* one past its end */
  int32_t nCols;
} PfRangeAndCols;

typedef struct PfGainHeader {
  uint64_t v_pedestals; /* a pointer in the reference; ignored on read */
  PfRangeAndCols rangeAndCols[PF_MAX_MODULES];
  float minPed, maxPed, minGain, maxGain;
  float pedPrecision, gainPrecision;
  uint32_t numberOfRowsAveragedOver; /* 80 */
  uint32_t nBinsToUseForEncoding;
  uint32_t deadFlag;
  uint32_t noisyFlag;
} PfGainHeader;

/* CondFormats/pixelCPEforGPU.h:20-25 */
typedef struct PfCommonParams {
  float thicknessB, thicknessE, pitchX, pitchY;
} PfCommonParams;

/* DataFormats/SOARotation.h SOAFrame<float>: position then 3x3 rotation (rows = local axes) */
typedef struct PfFrame {
  float px, py, pz;
  float R11, R12, R13, R21, R22, R23, R31, R32, R33;
} PfFrame;

/* CondFormats/pixelCPEforGPU.h:27-47 */
typedef struct PfDetParams {
  uint8_t isBarrel;
  uint8_t isPosZ;
  uint16_t layer;
  uint16_t index;
  uint32_t rawId;
  float shiftX, shiftY;
  float chargeWidthX, chargeWidthY;
  float x0, y0, z0;
  float sx[3], sy[3];
  PfFrame frame;
} PfDetParams;

/* Geometry/phase1PixelTopology.h:161-170 */
typedef struct PfAverageGeometry {
  float ladderZ[PF_N_LADDERS_BARREL];
  float ladderX[PF_N_LADDERS_BARREL];
  float ladderY[PF_N_LADDERS_BARREL];
  float ladderR[PF_N_LADDERS_BARREL];
  float ladderMinZ[PF_N_LADDERS_BARREL];
  float ladderMaxZ[PF_N_LADDERS_BARREL];
  float endCapZ[2];
} PfAverageGeometry;

/* CondFormats/pixelCPEforGPU.h:51-54 */
typedef struct PfLayerGeometry {
  uint32_t layerStart[PF_N_LAYERS + 1];
  uint8_t layer[PF_LAYER_INDEX_SIZE];
} PfLayerGeometry;

/* DataFormats/BeamSpotPOD.h:12-20 */
typedef struct PfBeamSpot {
  float x, y, z, sigmaZ, beamWidthX, beamWidthY, dxdz, dydz, emittanceX, emittanceY, betaStar;
} PfBeamSpot;

/* DataFormats/PixelErrors.h:9-14 */
typedef struct PfPixelError {
  uint32_t rawId;
  uint32_t word;
  uint8_t errorType;
  uint8_t fedId;
} PfPixelError;

/* one entry of PixelFormatterErrors (DataFormats/PixelErrors.h:16), the
   S-Link framing errors of the FED loop (ErrorChecker.cc:38-91): all under
   the dummy detector id 0xffffffff, in FED-loop order.  SiPixelRawDataError
   (DataFormats/SiPixelRawDataError.h:16-50) keeps the 64-bit header or
   trailer word, the error type (32, 33, 34, 39) and the full FED id; its
   message follows from the type (pg_error_message). */
typedef struct PfFormatterError {
  uint64_t word64;
  uint32_t errorType;
  uint32_t fedId;
} PfFormatterError;

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
static_assert(sizeof(PfCablingMap) == 1440128, "cabling map image size");
static_assert(sizeof(PfGainHeader) == 24048, "gain header image size");
static_assert(sizeof(PfDetParams) == 112, "DetParams image size");
static_assert(sizeof(PfAverageGeometry) == 3560, "AverageGeometry image size");
static_assert(sizeof(PfLayerGeometry) == 160, "LayerGeometry image size");
static_assert(sizeof(PfBeamSpot) == 44, "BeamSpotPOD image size");
static_assert(sizeof(PfPixelError) == 12, "PixelErrorCompact image size");
static_assert(sizeof(PfFormatterError) == 16, "formatter error record size");
#endif

#endif /* PIXFMT_H */
