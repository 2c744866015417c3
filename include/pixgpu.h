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
 *   pg_fit_riemann       HelixFitOnGPU::launchRiemannKernelsOnCPU (RiemannFitOnGPU.cc:3-110)
 *   pg_submit / pg_query / pg_wait / pg_result / pg_release
 *                        the acquire()/produce() split of the CUDA modules (ExternalWork:
 *                        work queued on the event's stream, the framework told when done)
 *                        and the SoA-from-CUDA transfer modules
 *   pg_pool_* / pg_serve the reference has no counterpart: its EventProcessor runs one event
 *                        per stream; these are the batching and admission layer above
 *                        the same chain
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

/* per-event flag bits (pg_event_counts.flags, the results' flags): conditions
   where the reference's behaviour is undefined or its truncation order is not
   reproduced exactly */
enum pg_flag {
  PG_FLAG_MODULE_TOO_BIG = 1u << 0,    /* a module of > 4000 pixels or > 1024 clusters (clustered on its
                                          first 4000 pixels / its first 1024 clusters kept, as the
                                          reference's serial build does) */
  PG_FLAG_EDGE_OVERFLOW = 1u << 1,     /* more CA links than the edge capacity */
  PG_FLAG_NBR_POOL_OVERFLOW = 1u << 2, /* more cells with neighbours than the list pool */
  PG_FLAG_TRK_POOL_OVERFLOW = 1u << 3, /* more cells with tracks than the list pool */
  PG_FLAG_FIT_BIN_OVERFLOW = 1u << 4,  /* > 24576 tuples of one multiplicity */
  PG_FLAG_TUPLE_OVERFLOW = 1u << 5,    /* > 32768 tuples (the tail is dropped, as in the reference) */
  PG_FLAG_CELL_OVERFLOW = 1u << 6,     /* doublet capacity reached (truncated as in the reference) */
  PG_FLAG_HIT_OVERFLOW = 1u << 7,      /* > 49152 clusters (truncated as in the reference) */
  PG_FLAG_ERR_OVERFLOW = 1u << 8,      /* more digi errors than kept */
  PG_FLAG_TOO_MANY_WORDS = 1u << 9,    /* event larger than MAX_FED_WORDS */
  PG_FLAG_H2T_OVERFLOW = 1u << 10,     /* hit-to-tuple capacity exceeded */
  PG_FLAG_TM_OVERFLOW = 1u << 11,      /* tuple multiplicity capacity exceeded */
  PG_FLAG_VTX_OVERFLOW = 1u << 12,     /* split vertex with >= 512 tracks or > 1024 vertices */
  PG_FLAG_DEEP_TUPLE = 1u << 13,       /* a CA path longer than 5 hits (the reference aborts) */
  PG_FLAG_J_OVERFLOW = 1u << 14,       /* more doublet inner-hit slots than kept */
  PG_FLAG_BAD_INPUT = 1u << 15,        /* payload words outside the cabling tables (read as padding) */
  /* bit 16 is the results' "more loose tracks than stored" */
  PG_FLAG_SPLIT_MODULE = 1u << 17,     /* a module's digis in several runs: the later runs are read as
                                          padding (the reference's result is loop-order dependent) */
  PG_FLAG_TOO_MANY_RUNS = 1u << 18,    /* more than 2000 module runs: the first 2000 found are kept (the
                                          reference's countModules counter wraps, gpuClustering.h:33) */
  PG_FLAG_SCAN_STALL = 1u << 19        /* a prefix-scan tile waited past its bound for the tile before it:
                                          the event's offsets are invalid (not expected to occur) */
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
  uint32_t max_events;           /* events per batch (1..1024) */
  uint32_t max_words_per_batch;  /* FED payload words over a whole batch */
  uint32_t slots;                /* independent batch slots (streams + workspaces); 0: as many as fit in
                                    hbm_fraction of the free device memory, at most 16 */
  uint32_t use_graphs;           /* 1: the chain for each batch size is captured once as a CUDA graph */
  uint64_t pool_words;           /* device-resident input pool, in FED words (0: no pool) */
  double hbm_fraction;           /* share of free device memory the slots may take when slots == 0 */
  uint32_t riemann_fit;          /* 1: Riemann fits in place of broken-line fits (the useRiemannFit
                                    parameter of CAHitNtupletGeneratorOnGPU.cc:49, default off) */
  uint32_t vertex_algo;          /* vertex clusterer of PixelVertexProducerCUDA.cc:26-35: 0 useDensity
                                    (the default), 1 useDBSCAN, 2 useIterative */
  /* CAHitNtupletGeneratorOnGPU parameters (CAHitNtupletGeneratorOnGPU.cc:45-66); pg_default_config
     sets the reference's values */
  uint32_t min_hits_per_ntuplet;              /* 3 (default) or 4 */
  uint32_t include_jumping_forward_doublets;  /* 1 */
  uint32_t early_fishbone;                    /* 1 */
  uint32_t late_fishbone;                     /* 0; 1 adds the late fishbone and the fishbone cleaner */
  uint32_t ideal_conditions;                  /* 1 */
  uint32_t do_cluster_cut, do_z0_cut, do_pt_cut; /* 1, 1, 1 */
  /* the FED loop's ErrorChecker (plugin-SiPixelClusterizer/ErrorChecker.cc:38-91) */
  uint32_t formatter_errors;     /* 1: record its S-Link framing errors (types 32, 33, 34, 39) as the
                                    "formatterErrors" product; 0 (default): as the reference, whose
                                    ErrorChecker records none (ErrorChecker.cc:36) */
  uint32_t fed_scan;             /* 0: the FED header/trailer checks and word concatenation on the host
                                    (default); 1: on the device, from the whole FED buffers */
  uint32_t mixed_fit;            /* 1: the chain fits with the mixed-precision variant of its fit
                                    (pg_fit_broken_line_mixed, pg_fit_riemann_mixed) in place of FP64
                                    (the reference's precision, default 0); see pg_event_counts for the
                                    cut decisions whose outcome precision can change */
  /* Per-event container capacities.  0 keeps the reference's value (given
     beside each), whose truncation order the results reproduce.  Larger
     values run the same algorithm on events whose containers would overflow
     (the reference changes them only by recompiling, CAConstants.h:18-40);
     indices are 32-bit throughout, and every per-event array of a slot is
     sized by them (pg_slot_bytes).  Smaller values are refused. */
  uint32_t cap_fed_words;        /* 300000: MAX_FED_WORDS (SiPixelRawToClusterGPUKernel.cc:34) */
  uint32_t cap_hits;             /* 49152: maxNumberOfHits (gpuClusteringConstants.h:10,27); <= 2^21 */
  uint32_t cap_doublets;         /* 458752: maxNumberOfDoublets (CAHitNtupletGeneratorOnGPU.cc:48) */
  uint32_t cap_lists;            /* 65536: maxNumOfActiveDoublets, the cells that may hold a neighbour
                                    or a track list (CAConstants.h:40) */
  uint32_t cap_tuples;           /* 32768: HitContainer bins = TrackSoA stride (PixelTrackHeterogeneous.h:20,62);
                                    < 2^20 */
  uint32_t cap_multiplicity;     /* 24576: maxNumberOfTuples, the TupleMultiplicity content and the fits
                                    per multiplicity (CAConstants.h:22); <= cap_tuples */
  uint32_t cap_hit_to_tuple;     /* 98304: the HitToTuple content (CAConstants.h:64) */
} pg_config;

typedef struct pg_event_counts {
  uint32_t n_words, n_modules, n_digi_errors, n_hits;
  uint32_t n_cells, n_tuples, n_loose, n_vertices;
  uint32_t flags;               /* capacity flags (PG_FLAG_*) */
  /* cut decisions whose two sides lie within four single-precision ulps
     (2^-22 relative) of each other, counted over every decision the chain
     evaluates: the doublet cuts (gpuPixelDoubletsAlgos.h:146-170: z window,
     dr, z0, pt), the CA cuts (GPUCACell.h:175-206: RZ alignment, curvature,
     dca) and the classification cuts (CAHitNtupletGeneratorKernelsImpl.h:
     340-406: chi2, tip, pt, zip).  These are the decisions that can flip when
     the operands come from another precision (an FP32 fit, FMA contraction). */
  uint32_t n_cut_margin_doublets, n_cut_margin_ca, n_cut_margin_quality;
} pg_event_counts;

/* the reference's configuration; start every pg_config from it */
void pg_default_config(pg_config* cfg);
int pg_create(const pg_es_images* es, const pg_config* cfg, pg_ctx** out);
/* the configuration in force (slots resolved when created with slots == 0) */
int pg_get_config(const pg_ctx* ctx, pg_config* out);
void pg_destroy(pg_ctx* ctx);
const char* pg_last_error(const pg_ctx* ctx);
/* device bytes held by one batch slot */
size_t pg_slot_bytes(const pg_ctx* ctx);

/* FED scan of one raw.bin record into the flat word buffer and the per-word-pair
 * FED index, as SiPixelRawToClusterCUDA::produce does on the host. */
int pg_unpack_raw(const pg_ctx* ctx, const uint8_t* raw, size_t raw_size, uint32_t* words, uint8_t* fed_ids,
                  uint32_t cap_words, uint32_t* n_words);

/* Clustering of given digis on slot 0 (synchronous): countModules, findClus
 * and clusterChargeCut (plugin-SiPixelClusterizer/gpuClustering.h:19-273,
 * gpuClusterChargeCut.h:14-114) on n digis in host memory -- module index
 * (9999 for an invalid digi), row, column and calibrated charge, the
 * input of the reference's clustering kernels and of its clustering test
 * (test/gpuClustering_t.h).  Out: the module index after the charge cut
 * (9999 for removed pixels), the cluster index per digi, and per module the
 * cluster count, module id and the module-run starts (module_start[0] = the
 * run count, as countModules leaves it; 2000 / 2001 entries). */
int pg_cluster_digis(pg_ctx* ctx, uint32_t n, const uint16_t* module_ind, const uint16_t* xx, const uint16_t* yy,
                     const uint16_t* adc, uint16_t* module_ind_out, int32_t* clus, uint32_t* clus_in_module,
                     uint32_t* module_id, uint32_t* module_start, uint32_t* n_modules, uint32_t* flags);

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
/* The same products of event k of the finished asynchronous batch on `slot`
 * (after pg_wait, or pg_query returning PG_OK, and before pg_release):
 * PG_ERR_BUSY while the batch runs.  The full-size products the framework
 * modules hand to host consumers (SiPixelDigisSoA, SiPixelClustersSoA,
 * PixelTrackHeterogeneous, ZVertexHeterogeneous) come from here; pg_result
 * is the compact form. */
int pg_slot_product(pg_ctx* ctx, uint32_t slot, uint32_t k, const char* name, void* dst, size_t cap_bytes,
                    size_t* count, int* elem_bytes);

/* Device-resident path (inputs staged once, then the kernels alone):
 * pg_stage_batch unpacks and copies a batch into slot s; pg_run_staged
 * launches the chain on it on the slot's stream (asynchronous); pg_sync
 * waits for slot s.  pg_slot_stream returns the slot's cudaStream_t. */
int pg_stage_batch(pg_ctx* ctx, uint32_t slot, uint32_t n_events, const uint8_t* const* raws,
                   const size_t* raw_sizes);
int pg_run_staged(pg_ctx* ctx, uint32_t slot);
int pg_sync(pg_ctx* ctx, uint32_t slot);
void* pg_slot_stream(pg_ctx* ctx, uint32_t slot);

/* Compact per-event result of an asynchronous batch: the loose tracks (quality >= loose)
 * in tuple order and the vertices, the content of PixelTrackHeterogeneous /
 * ZVertexHeterogeneous that a consumer reads (PixelTrackSoAFromCUDA.cc,
 * PixelVertexSoAFromCUDA.cc).  Written by the device into mapped pinned host memory;
 * the pointers stay valid until pg_release of the slot. */
typedef struct pg_result_view {
  uint32_t n_tracks;       /* loose tracks stored (at most 16384) */
  uint32_t n_loose_all;    /* loose tracks found */
  uint32_t n_vertices, n_hits, n_tuples, n_digis, n_cells;
  uint32_t flags;          /* capacity flags; bit 16: more loose tracks than stored */
  const uint32_t* tuple_index;   /* [n_tracks] index of the tuple in the full track SoA */
  const uint8_t* track_n_hits;   /* [n_tracks] */
  const uint8_t* quality;        /* [n_tracks] */
  const float* state;            /* [n_tracks][5] phi, Tip, 1/pt*q, cot(theta), Zip */
  const float* cov;              /* [n_tracks][15] */
  const float* pt;               /* [n_tracks] */
  const float* eta;
  const float* chi2;
  const uint32_t* hits;          /* [n_tracks][5] hit indices, 0xffffffff past track_n_hits */
  const int16_t* vertex;         /* [n_tracks] vertex index or -1 */
  const float* zv;               /* [n_vertices] */
  const float* wv;
  const float* vchi2;
  const float* ptv2;
  const int32_t* ndof;
  const uint16_t* sort_ind;      /* vertices by decreasing sum pt^2 */
} pg_result_view;

/* Asynchronous batches.  pg_submit unpacks, copies and launches on a free slot
 * and returns its index (PG_ERR_BUSY when every slot is in use); pg_query returns
 * PG_OK when the batch has finished and PG_ERR_BUSY while it runs; pg_wait blocks;
 * pg_result gives the view of event k; pg_release makes the slot free again. */
int pg_submit(pg_ctx* ctx, uint32_t n_events, const uint8_t* const* raws, const size_t* raw_sizes,
              uint32_t* slot);
int pg_query(pg_ctx* ctx, uint32_t slot);
int pg_wait(pg_ctx* ctx, uint32_t slot);
int pg_result(pg_ctx* ctx, uint32_t slot, uint32_t k, pg_result_view* view);
int pg_release(pg_ctx* ctx, uint32_t slot);

/* Totals over the finished batch on a slot: result sizes (the bytes the device
 * wrote into host memory) and the per-event counts the roofline model uses. */
typedef struct pg_batch_summary {
  uint32_t n_events, flags;          /* flags: OR over the events */
  uint64_t n_tracks, n_vertices, result_bytes;
  uint64_t n_digis, n_modules, n_hits, n_cells, n_edges, n_tuples, n_tuple_hits;
  uint64_t n_cut_margin;             /* cut decisions on their float boundary (pg_event_counts) */
  uint64_t n_flagged_events;         /* events with any capacity flag (PG_FLAG_*; not bit 16) */
} pg_batch_summary;
int pg_batch_summary_get(pg_ctx* ctx, uint32_t slot, pg_batch_summary* out);

/* Device-resident input pool (contexts created with pool_words > 0).  pg_pool_put
 * unpacks one event, copies its words into the pool on the upload stream and
 * returns a handle; PG_ERR_NOMEM means the pool has no room now (admission
 * refused), PG_ERR_BUSY that all pinned staging buffers are in flight.
 * pg_submit_pooled gathers the given events into a free slot and launches the
 * chain; their pool space is released once the gather has run, unless flags has
 * PG_POOL_KEEP (the events stay resident and may be submitted again).
 * pg_pool_release drops an event that is not part of a pending batch. */
#define PG_POOL_KEEP 1u
int pg_pool_put(pg_ctx* ctx, const uint8_t* raw, size_t raw_size, uint32_t* handle);
int pg_pool_release(pg_ctx* ctx, uint32_t handle);
int pg_pool_info(pg_ctx* ctx, uint64_t* cap_words, uint64_t* free_words, uint32_t* live_events);
int pg_submit_pooled(pg_ctx* ctx, uint32_t n_events, const uint32_t* handles, uint32_t flags, uint32_t* slot);

/* Captures the chain of every batch size 1..max_batch on every slot (graphs are
 * otherwise captured on first use). */
int pg_prepare(pg_ctx* ctx, uint32_t max_batch);

/* Serving loop with continuous batching over a device-resident pool.  Request i
 * arrives at arrivals[i] seconds (or on a Poisson schedule of rate_hz when
 * arrivals is NULL) and carries raw event request_event[i] (or i % n_raw).
 * Arrivals are unpacked by upload_threads host threads and admitted into the pool
 * while it has room; whenever a slot is free, all admitted events waiting (up to
 * max_batch and the slot's word capacity) are dispatched as one batch.  Latency is
 * measured from arrival to the host seeing the batch complete.  fn, when given, is
 * called on the calling thread for every request with its result view. */
typedef struct pg_serve_config {
  uint32_t n_requests;
  double rate_hz;
  uint64_t seed;
  uint32_t max_batch;        /* 0: max_events */
  uint32_t upload_threads;
} pg_serve_config;

typedef struct pg_serve_stats {
  uint32_t completed, batches, max_batch_seen, admission_waits;
  double wall_s;             /* first arrival to last completion */
  double events_per_s;
  double mean_batch;
  double offered_hz;
  double p50_ms, p90_ms, p99_ms, mean_ms, max_ms;
} pg_serve_stats;

typedef void (*pg_result_fn)(void* user, uint32_t request, uint32_t event, const pg_result_view* view);

void pg_default_serve_config(pg_serve_config* cfg);
int pg_serve(pg_ctx* ctx, uint32_t n_raw, const uint8_t* const* raws, const size_t* raw_sizes,
             const pg_serve_config* cfg, const double* arrivals, const uint32_t* request_event,
             pg_serve_stats* stats, double* latencies, pg_result_fn fn, void* user);

/* Kernel timing.  pg_set_probe(ctx, name) brackets every launch of the named
 * kernel ("*": every kernel, NULL: none) with timing events, in plain launches
 * and inside graphs captured afterwards (existing graphs are dropped; every slot
 * must be free).  pg_probe_read gives the device time of each timed launch of
 * the last finished batch on a slot. */
typedef struct pg_probe_entry {
  const char* kernel;
  float ms;
} pg_probe_entry;
int pg_set_probe(pg_ctx* ctx, const char* kernel);
int pg_probe_read(pg_ctx* ctx, uint32_t slot, uint32_t max, pg_probe_entry* out, uint32_t* n);

/* Launch-shape tuning.  Each tunable kernel loops grid-stride over its
 * event's work; its grid x-extent is the default for the batch size times
 * 2^scale, scale in -3..3 (0: default), kept per batch size (a batch uses the
 * table of its size, else of the largest tuned size below it).  Results do
 * not depend on the scales.  pg_tune_kernel_name(i) names the i-th tunable
 * kernel (NULL past the last).  pg_tune_set/pg_tune_load need every slot free
 * and drop the captured graphs.
 * pg_autotune times each tunable kernel (kernel probe, median of `repeats`
 * batches of the first n records) at scales -2..2 and keeps the fastest when
 * it gains 2%, kernel by kernel; *gain_ms receives the summed saving per batch.
 * pg_tune_save writes the table as lines "<device name>|<n> <kernel> <scale>";
 * pg_tune_load applies the lines of this context's device and returns their
 * number (>= 0), or PG_ERR_NOTFOUND when the file is missing. */
const char* pg_tune_kernel_name(uint32_t i);
int pg_tune_set(pg_ctx* ctx, uint32_t n_events, const char* kernel, int scale);
int pg_tune_get(const pg_ctx* ctx, uint32_t n_events, const char* kernel, int* scale);
int pg_autotune(pg_ctx* ctx, uint32_t n_events, const uint8_t* const* raws, const size_t* sizes, uint32_t repeats,
                double* gain_ms);
int pg_tune_save(const pg_ctx* ctx, const char* path);
int pg_tune_load(pg_ctx* ctx, const char* path);

/* Vertex finding without device allocation.  No counterpart in the reference:
 * it exists for callers that cannot allocate device memory where they need the
 * vertices, e.g. a per-event module inside a framework that owns all device
 * memory through its own caching allocator (cudaFree synchronises the whole
 * device), or a latency-critical path that must not stall on the allocator.
 * It runs the chain's vertex finder on one event's track SoA given by the
 * caller in device memory: tuple_off[n_tuples+1], quality[n_tuples],
 * pt[n_tuples], state[n_tuples*5], cov[n_tuples*15]; it writes idv[n_tuples] and
 * zv, wv, chi2, ptv2, ndof, sort_ind (1024 entries each) and returns the vertex
 * count (and the capacity flags) on the host.  All temporaries live in one
 * static device array of 1.25 MB that every GPU loading the library keeps until
 * exit; nothing is allocated and no context is needed.  n_tuples must be at most
 * 32767 (PG_ERR_CAPACITY otherwise).  The first call on a device looks up the
 * array's device address and sets the kernel's shared-memory attribute, so make
 * it before any stream capture on that device.  Every call shares the array:
 * calls that overlap on the GPU (other streams, other threads) race, so
 * serialise them.  The call waits for its work on `stream` before returning.
 * msg (msg_cap bytes, may be NULL) receives an error text. */
int pg_vertices_noalloc(const uint32_t* tuple_off, const uint8_t* quality, const float* pt, const float* state,
                        const float* cov, uint32_t n_tuples, int16_t* idv, float* zv, float* wv, float* chi2,
                        float* ptv2, int32_t* ndof, uint16_t* sort_ind, uint32_t* n_vertices, uint32_t* flags,
                        void* stream, char* msg, size_t msg_cap);

/* Broken-line fits of n tuples of N (3 or 4) hits already on the device:
 * hits[(t*N+i)*3+k], ge[(t*N+i)*6+k]; outputs state[t*5+k], cov[t*15+k],
 * pt[t], eta[t], chi2[t]; B in GeV/cm (0.0114256972711507 in the reference). */
int pg_fit_broken_line(pg_ctx* ctx, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                       float* cov, float* pt, float* eta, float* chi2, void* stream);

/* The same fits in mixed precision: FP32 arithmetic for the multiple-scattering
 * model, the band matrices and the parameter updates; FP64 for the circle and
 * line Cholesky inversions with their solves, the covariance propagation, and
 * the three-point reference circle with what is measured from it (the arc
 * lengths and the radial residuals), which lose the sagitta of stiff tracks
 * in FP32.  A variant beside HelixFitOnGPU's FP64 fit; its deviation from the
 * FP64 result is measured in tests/test_gpu_fit_mixed.py. */
int pg_fit_broken_line_mixed(pg_ctx* ctx, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                       float* cov, float* pt, float* eta, float* chi2, void* stream);

/* Riemann fits of n tuples of N (3 or 4) hits already on the device, same
 * layout as pg_fit_broken_line.  Replaces HelixFitOnGPU::launchRiemannKernelsOnCPU
 * (RiemannFitOnGPU.cc:3-110; kernelFastFit/kernelCircleFit/kernelLineFit,
 * RiemannFitOnGPU.h:20-162), the fit that CAHitNtupletGeneratorOnGPU selects
 * with useRiemannFit (CAHitNtupletGeneratorOnGPU.cc:49). */
int pg_fit_riemann(pg_ctx* ctx, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                   float* cov, float* pt, float* eta, float* chi2, void* stream);

/* The Riemann fits in mixed precision: FP32 for the multiple-scattering
 * models, the s-z projection and the single-precision eigen-solves of the
 * numerical Jacobian; FP64 for the prefit circle, the path lengths of the
 * radiation-length model, the Riemann matrix and its smallest eigenvector,
 * the Cholesky inversions with their solves and the covariance propagation.  A variant beside the FP64 fit; its deviation from the FP64
 * result is measured in tests/test_gpu_riemann.py. */
int pg_fit_riemann_mixed(pg_ctx* ctx, int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                         float* cov, float* pt, float* eta, float* chi2, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PIXGPU_H */
