/* A C client of the two public libraries, built the way an integrator would:
 * it includes include/pixgpu.h and include/pixsynth.h, links libpixgpu.so and
 * libpixsynth.so, and drives the chain through the C ABI only.  Compiled as
 * C99 and as C++17 by tests/test_capi_client.py.
 *
 *   capi_client cpu        calls that need no device: defaults, argument
 *                          checks, tunable kernel names
 *   capi_client gpu PU     a seeded event of pileup PU through pg_process_batch
 *                          and through pg_submit/pg_result; prints one line
 *                          "words hits cells tuples vertices loose" and checks
 *                          that both paths agree */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pixgpu.h"
#include "pixsynth.h"

#define CHECK(cond)                                                   \
  do {                                                                \
    if (!(cond)) {                                                    \
      fprintf(stderr, "capi_client: check failed: %s (line %d)\n", #cond, __LINE__); \
      return 1;                                                       \
    }                                                                 \
  } while (0)

static int cpu_checks(void) {
  pg_config cfg;
  pg_serve_config scfg;
  pg_ctx* ctx = NULL;
  uint32_t i = 0;
  memset(&cfg, 0xff, sizeof(cfg));
  pg_default_config(&cfg);
  /* the reference's CAHitNtupletGeneratorOnGPU defaults */
  CHECK(cfg.min_hits_per_ntuplet == 3 && cfg.include_jumping_forward_doublets == 1);
  CHECK(cfg.early_fishbone == 1 && cfg.late_fishbone == 0 && cfg.ideal_conditions == 1);
  CHECK(cfg.do_cluster_cut == 1 && cfg.do_z0_cut == 1 && cfg.do_pt_cut == 1);
  CHECK(cfg.riemann_fit == 0 && cfg.vertex_algo == 0 && cfg.formatter_errors == 0 && cfg.fed_scan == 0);
  CHECK(cfg.max_events > 0 && cfg.max_words_per_batch > 0);
  pg_default_serve_config(&scfg);
  CHECK(scfg.n_requests > 0 && scfg.rate_hz > 0);
  /* argument errors come back as status codes, never as a crash */
  CHECK(pg_create(NULL, &cfg, &ctx) == PG_ERR_ARG && ctx == NULL);
  CHECK(pg_last_error(NULL) != NULL);
  CHECK(pg_query(NULL, 0) == PG_ERR_ARG);
  CHECK(pg_release(NULL, 0) == PG_ERR_ARG);
  while (pg_tune_kernel_name(i) != NULL) ++i;
  CHECK(i >= 20);
  printf("cpu ok: %u tunable kernels\n", i);
  return 0;
}

static int gpu_run(double pu) {
  ps_detector_config dcfg;
  ps_event_config ecfg;
  ps_detector* det = NULL;
  ps_event* ev = NULL;
  pg_es_images img;
  pg_config cfg;
  pg_ctx* ctx = NULL;
  pg_event_counts counts;
  pg_result_view view;
  const uint8_t* raw = NULL;
  size_t rawSize = 0;
  uint32_t slot = 0;
  int kind, rc;
  const uint8_t** parts[5];
  size_t* sizes[5];

  ps_default_detector_config(&dcfg);
  dcfg.seed = 20261203u;
  CHECK(ps_detector_create(&dcfg, &det) == 0);
  parts[0] = &img.cabling; sizes[0] = &img.cabling_size;
  parts[1] = &img.gain; sizes[1] = &img.gain_size;
  parts[2] = &img.cpe; sizes[2] = &img.cpe_size;
  parts[3] = &img.beamspot; sizes[3] = &img.beamspot_size;
  parts[4] = &img.fedids; sizes[4] = &img.fedids_size;
  for (kind = 0; kind < 5; ++kind) CHECK(ps_detector_es(det, kind, parts[kind], sizes[kind]) == 0);
  ps_default_event_config(&ecfg);
  CHECK(ps_event_generate(det, 20261203u, pu, &ecfg, &ev) == 0);
  CHECK(ps_event_raw(ev, &raw, &rawSize) == 0);

  pg_default_config(&cfg);
  cfg.max_events = 1;
  cfg.max_words_per_batch = 300000;
  rc = pg_create(&img, &cfg, &ctx);
  if (rc != PG_OK) {
    fprintf(stderr, "pg_create: %d\n", rc);
    return 1;
  }
  rc = pg_process_batch(ctx, 1, &raw, &rawSize);
  if (rc != PG_OK) {
    fprintf(stderr, "pg_process_batch: %d %s\n", rc, pg_last_error(ctx));
    return 1;
  }
  CHECK(pg_event_counts_get(ctx, 0, &counts) == PG_OK);
  CHECK(pg_submit(ctx, 1, &raw, &rawSize, &slot) == PG_OK);
  CHECK(pg_wait(ctx, slot) == PG_OK);
  CHECK(pg_result(ctx, slot, 0, &view) == PG_OK);
  /* the synchronous products and the compact asynchronous result agree */
  CHECK(view.n_hits == counts.n_hits && view.n_tuples == counts.n_tuples);
  CHECK(view.n_vertices == counts.n_vertices && view.n_loose_all == counts.n_loose);
  CHECK(view.n_cells == counts.n_cells);
  printf("%u %u %u %u %u %u\n", counts.n_words, counts.n_hits, counts.n_cells, counts.n_tuples, counts.n_vertices,
         counts.n_loose);
  CHECK(pg_release(ctx, slot) == PG_OK);
  pg_destroy(ctx);
  ps_event_destroy(ev);
  ps_detector_destroy(det);
  return 0;
}

int main(int argc, char** argv) {
  if (argc >= 2 && strcmp(argv[1], "cpu") == 0) return cpu_checks();
  if (argc >= 3 && strcmp(argv[1], "gpu") == 0) return gpu_run(atof(argv[2]));
  fprintf(stderr, "usage: capi_client cpu | gpu PU\n");
  return 2;
}
