/*
 * pixgpu.h — C ABI of the B200-native pixel reconstruction chain.
 *
 * One context owns the device-resident conditions (cabling map, gains, CPE
 * parameters, beam spot) and a set of batch slots.  A batch is 1..max_events
 * events in the reference's raw.bin record layout; the chain runs raw-to-digi,
 * clustering, rechits, CA n-tuplets, broken-line fits and vertexing for all
 * of them in one sequence of launches.  Every call returns a status code;
 * no C++ exception crosses this boundary.
 *
 * Reference interfaces replaced (paths in the reference's src/serial tree):
 *   pg_create            the ESProducers SiPixelFedCablingMapGPUWrapperESProducer,
 *                        SiPixelGainCalibrationForHLTGPUESProducer, PixelCPEFastESProducer,
 *                        BeamSpotESProducer (their produce(): file images in,
 *                        device-resident ES product out)
 *   pg_unpack_raw        SiPixelRawToClusterCUDA::produce host part, FED loop
 *                        (plugin-SiPixelClusterizer/SiPixelRawToClusterCUDA.cc:78-138)
 *   pg_process_batch     the module chain SiPixelRawToClusterCUDA -> SiPixelRecHitCUDA ->
 *                        CAHitNtupletCUDA -> PixelVertexProducerCUDA (their produce() calls,
 *                        SiPixelRawToClusterCUDA.cc:60-158, SiPixelRecHitCUDA.cc:37-50,
 *                        CAHitNtupletCUDA.cc:30-36, PixelVertexProducerCUDA.cc:42-62)
 *   pg_get_product       the product getters of SiPixelDigisSoA, SiPixelClustersSoA,
 *                        TrackingRecHit2DCPU, PixelTrackHeterogeneous, ZVertexHeterogeneous
 *                        (the *SoAFromCUDA transfer modules of the CUDA program)
 *   pg_fit_broken_line   HelixFitOnGPU::launchBrokenLineKernels (BrokenLineFitOnGPU.cc:3-68)
 */
#ifndef PIXGPU_H
#define PIXGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum pg_status {
  PG_OK = 0,
  PG_ERR_ARG = -1,       /* invalid argument or call order */
  PG_ERR_CUDA = -2,      /* a CUDA runtime call failed (see pg_last_error) */
  PG_ERR_FORMAT = -3,    /* malformed ES image or raw record */
  PG_ERR_CAPACITY = -4,  /* batch or event larger than the context was created for */
  PG_ERR_BUSY = -5,      /* no free batch slot (asynchronous API) */
  PG_ERR_NOMEM = -6,     /* device or pinned host allocation failed / admission refused */
  PG_ERR_NOTFOUND = -7   /* unknown product name */
};

typedef struct pg_ctx pg_ctx;

typedef struct pg_es_images {
  const uint8_t* cabling; size_t cabling_size;   /* cablingMap.bin */
  const uint8_t* gain; size_t gain_size;         /* gain.bin */
  const uint8_t* cpe; size_t cpe_size;           /* cpefast.bin */
  const uint8_t* beamspot; size_t beamspot_size; /* beamspot.bin */
  const uint8_t* fedids; size_t fedids_size;     /* fedIds.bin */
} pg_es_images;

typedef struct pg_config {
  int device;                    /* CUDA device ordinal */
  uint32_t max_events;           /* events per batch */
  uint32_t max_words_per_batch;  /* FED payload words over a whole batch */
  uint32_t slots;                /* independent batch slots (streams + workspaces) */
} pg_config;

typedef struct pg_event_counts {
  uint32_t n_words, n_modules, n_digi_errors, n_hits;
  uint32_t n_cells, n_tuples, n_loose, n_vertices;
  uint32_t flags;               /* capacity flags (PG_FLAG_*) */
} pg_event_counts;

void pg_default_config(pg_config* cfg);
int pg_create(const pg_es_images* es, const pg_config* cfg, pg_ctx** out);
void pg_destroy(pg_ctx* ctx);
const char* pg_last_error(const pg_ctx* ctx);
/* device bytes held by one batch slot */
size_t pg_slot_bytes(const pg_ctx* ctx);

/* FED scan of one raw.bin record into the flat word buffer and the per-word-pair
 * FED index, as SiPixelRawToClusterCUDA::produce does on the host. */
int pg_unpack_raw(const pg_ctx* ctx, const uint8_t* raw, size_t raw_size, uint32_t* words, uint8_t* fed_ids,
                  uint32_t cap_words, uint32_t* n_words);

/* Synchronous: unpack, copy to the device, run the chain on slot 0 and wait. */
int pg_process_batch(pg_ctx* ctx, uint32_t n_events, const uint8_t* const* raws, const size_t* raw_sizes);

/* Counts and products of event k of the last completed batch on slot 0.
 * Names: digis xx yy adc moduleInd clus pdigi rawIdArr errors; clusters
 * moduleStart clusInModule moduleId clusModuleStart; hits xl yl xerr yerr xg yg
 * zg rg charge iphi xsize ysize detInd hitsLayerStart phiOff phiBins; CA cellInner
 * cellOuter cellLayerPair cellDoubletId cellUsed cellNbrOff cellNbr cellTrkOff
 * cellTrk outerHitOff outerHitCells; tracks tupleOff tupleHits tupleDet quality
 * state cov pt eta chi2; vertices zv wv vchi2 ptv2 ndof sortInd idv; scalar
 * counters nDigis nModules nClusters nHits nCells nTuples nVertices nNbrLists
 * nTrkLists.  *count receives the number of elements, *elem_bytes their size. */
int pg_event_counts_get(pg_ctx* ctx, uint32_t k, pg_event_counts* out);
int pg_get_product(pg_ctx* ctx, uint32_t k, const char* name, void* dst, size_t cap_bytes, size_t* count,
                   int* elem_bytes);

/* Device-resident path (inputs staged once, then the kernels alone):
 * pg_stage_batch unpacks and copies a batch into slot s; pg_run_staged
 * launches the chain on it on the slot's stream (asynchronous); pg_sync
 * waits for slot s.  pg_slot_stream returns the slot's cudaStream_t. */
int pg_stage_batch(pg_ctx* ctx, uint32_t slot, uint32_t n_events, const uint8_t* const* raws,
                   const size_t* raw_sizes);
int pg_run_staged(pg_ctx* ctx, uint32_t slot);
int pg_sync(pg_ctx* ctx, uint32_t slot);
void* pg_slot_stream(pg_ctx* ctx, uint32_t slot);

/* Broken-line fits of n tuples of N (3 or 4) hits already on the device:
 * hits[(t*N+i)*3+k], ge[(t*N+i)*6+k]; outputs state[t*5+k], cov[t*15+k],
 * pt[t], eta[t], chi2[t]; B in GeV/cm (0.0114256972711507 in the reference). */
int pg_fit_broken_line(pg_ctx* ctx, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                       float* cov, float* pt, float* eta, float* chi2, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PIXGPU_H */
