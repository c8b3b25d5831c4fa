/*
 * Seeded synthetic VELO event generator (host library libvelo_gen.so).
 *
 * No counterpart in the reference: it stands in for the Monte Carlo samples the
 * reference validates on.  Output is Allen's non-MEP raw-bank layout for VP
 * super-pixel banks (main/src/Transpose.cpp:333-425), ready to be passed to
 * velo_chain_run() or to any of the per-algorithm entry points in velo_b200.h.
 */
#ifndef VELO_GENERATOR_H
#define VELO_GENERATOR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double mean_pileup;          /* Poisson mean of primary vertices per event (7.6) */
  double pileup_min;           /* if pileup_max > pileup_min, each event draws nu ~ U[min, max] */
  double pileup_max;
  double tracks_per_pv;        /* Poisson mean of tracks per vertex (25) */
  double eta_min, eta_max;     /* pseudorapidity range (2, 5) */
  double beam_sigma_xy;        /* mm (0.04) */
  double beam_sigma_z;         /* mm (45) */
  double hit_efficiency;       /* per crossed sensor (0.98) */
  double scatter_sigma;        /* mm, Gaussian smear of each hit in x and y (0.01) */
  double noise_rate;           /* noise pixels per pixel (1e-5) */
  double share_fraction;       /* charge-sharing band at each pixel edge (0.15) */
  double drop_corner_fraction; /* 2x2 clusters that lose their far corner (0.3) */
  int bank_version;            /* 2 (one bank per sensor), 3, or 4 (one per sensor pair) */
  int sp_order;                /* SP order inside a bank: 0 column order, 1 shuffled as read out (1) */
  int raw_format;              /* 0 super-pixel banks (type 63), 1 retina-cluster banks (type 73) (0) */
} VeloGenConfig;

typedef struct {
  uint64_t n_events;
  uint64_t raw_bytes;      /* bytes of the event blobs */
  uint64_t sizes_words;    /* u32 words of the bank-size array */
  uint64_t types_words;    /* u32 words of the bank-type array */
  uint64_t n_truth_pixels;
  uint64_t n_particles;
} VeloGenSizes;

typedef struct {
  uint32_t lhcb_id;  /* VELO LHCb id of the pixel's channel */
  uint32_t particle; /* index into the event's particles */
} VeloGenTruthPixel;

typedef struct {
  uint32_t pv;
  float eta;
  float phi;
  uint32_t n_hits;    /* sensors with a recorded hit */
  uint32_t n_modules; /* distinct modules with a recorded hit */
} VeloGenParticle;

void velo_gen_default_config(VeloGenConfig* cfg);

/* Generates events [first_event, first_event + n_events) of the stream `seed`.
 * Returns NULL on a malformed geometry blob or an unsupported bank version. */
void* velo_gen_create(
  const VeloGenConfig* cfg,
  const char* geometry,
  size_t geometry_size,
  uint64_t seed,
  unsigned first_event,
  unsigned n_events,
  unsigned n_threads);

void velo_gen_sizes(const void* handle, VeloGenSizes* sizes);

/* Copies into caller buffers sized from velo_gen_sizes(); any pointer may be NULL.
 * raw_offsets, truth_offsets and particle_offsets take n_events + 1 entries. */
void velo_gen_copy(
  const void* handle,
  char* raw,
  unsigned* raw_offsets,
  unsigned* raw_sizes,
  unsigned* raw_types,
  VeloGenTruthPixel* truth_pixels,
  unsigned* truth_offsets,
  VeloGenParticle* particles,
  unsigned* particle_offsets);

void velo_gen_destroy(void* handle);

#ifdef __cplusplus
}
#endif

#endif
