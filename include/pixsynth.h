/*
 * pixsynth.h — seeded synthetic Phase-1 pixel detector and events.
 *
 * The generator stands in for the CMS open-data sample that the reference
 * downloads at build time (data/url.txt): it builds a 1856-module detector
 * (4 barrel layers of 96/224/352/512 modules, 6 disks of 112), a 108-FED
 * cabling map, a gain/pedestal payload, CPE parameters and a beam spot, and
 * writes them in the reference's ES file layouts (pixfmt.h).  Events are
 * helices in a 3.8 T field from Gaussian-z pile-up vertices, digitised with
 * Landau charge and packed into S-Link framed FED words through the same
 * cabling map, so the reference reads them through its own Source and
 * SiPixelRawToClusterCUDA code path.
 */
#ifndef PIXSYNTH_H
#define PIXSYNTH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ps_detector ps_detector;
typedef struct ps_event ps_event;

enum ps_es_kind {
  PS_ES_CABLING = 0,  /* cablingMap.bin image */
  PS_ES_GAIN = 1,     /* gain.bin image */
  PS_ES_CPE = 2,      /* cpefast.bin image */
  PS_ES_BEAMSPOT = 3, /* beamspot.bin image */
  PS_ES_FEDIDS = 4    /* fedIds.bin image */
};

typedef struct ps_detector_config {
  uint64_t seed;             /* seeds gains/pedestals */
  double dead_column_frac;   /* fraction of (module, column, 80-row block) flagged dead */
  double bad_roc_frac;       /* fraction of ROCs flagged in cablingMap.badRocs */
} ps_detector_config;

typedef struct ps_event_config {
  double tracks_per_vertex;  /* Poisson mean of charged tracks per pile-up vertex */
  double pt_min;             /* GeV, lower edge of the power law */
  double pt_index;           /* dN/dpT ~ pT^-index */
  double eta_max;
  double noise_frac;         /* noise digis as a fraction of signal digis */
  int inject_errors;         /* >0: add that many FED error words per event */
  int fixed_pu;              /* 1: exactly round(pu) vertices; 0: Poisson(pu) */
  /* soft component per vertex (0 by default: no random numbers drawn, the
     events of the plain configuration are unchanged) */
  double soft_per_vertex;    /* Poisson mean of soft tracks per vertex */
  double soft_pt_min;        /* GeV; soft pT = soft_pt_min + Exp(soft_pt_mean) */
  double soft_pt_mean;       /* GeV */
  double secondary_frac;     /* share of soft tracks produced 2-12 cm from the vertex */
} ps_event_config;

typedef struct ps_truth {
  uint32_t n_vertices;
  uint32_t n_tracks;
  uint32_t n_sim_hits;
  uint32_t n_digis;
  const float* vertex_z;     /* [n_vertices] */
  const float* track_pt;     /* [n_tracks] */
  const float* track_eta;
  const float* track_phi;
  const int32_t* track_q;
  const int32_t* track_vertex;
  const uint8_t* track_nhits;
} ps_truth;

/* Fill *cfg with the defaults used by the benchmark workloads. */
void ps_default_detector_config(ps_detector_config* cfg);
void ps_default_event_config(ps_event_config* cfg);
/* The calibrated event model: fewer prompt tracks above 0.5 GeV plus a soft
 * exponential component, most of it produced displaced, so that a PU50 event
 * has about 57k digis, 18k hits and 1.6k loose tracks (the benchmark
 * workload's stated sizes).  The default configuration above is the denser
 * model of earlier versions (all tracks prompt and above 0.5 GeV). */
void ps_calibrated_event_config(ps_event_config* cfg);

int ps_detector_create(const ps_detector_config* cfg, ps_detector** out);
void ps_detector_destroy(ps_detector* det);
/* File image of one ES record; the memory is owned by the detector. */
int ps_detector_es(const ps_detector* det, int kind, const uint8_t** data, size_t* size);
/* Write cablingMap.bin, gain.bin, cpefast.bin, beamspot.bin, fedIds.bin into dir. */
int ps_detector_write(const ps_detector* det, const char* dir);

/* One event at pile-up `pu` from seed `seed`. */
int ps_event_generate(const ps_detector* det, uint64_t seed, double pu, const ps_event_config* cfg,
                      ps_event** out);
void ps_event_destroy(ps_event* ev);
/* The event as one raw.bin record (uint32 nfeds, then per FED: fedId, size, bytes). */
int ps_event_raw(const ps_event* ev, const uint8_t** data, size_t* size);
int ps_event_truth(const ps_event* ev, ps_truth* out);

/*
 * Broken-line/Riemann fit workload: n tuples of `nhits` (3..5) hits on
 * helices from the beam line, hits smeared by multiple scattering and by the
 * hit errors.  Output layout per tuple t, hit i:
 *   hits[(t*nhits + i)*3 + {0,1,2}]   global x, y, z (double, cm)
 *   hits_ge[(t*nhits + i)*6 + k]      covariance {xx, xy, yy, xz, yz, zz} (float, cm^2)
 *   truth[t*5 + {0..4}]               phi, tip, pt, cot(theta), zip
 */
int ps_fit_tuples(uint64_t seed, uint32_t n, uint32_t nhits, double* hits, float* hits_ge, double* truth);

#ifdef __cplusplus
}
#endif

#endif /* PIXSYNTH_H */
