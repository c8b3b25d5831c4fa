/*
 * Test infrastructure: the CPU-side checkers of the VELO super-pixel chain.
 *
 * Two CPU implementations export this same interface:
 *   - oracle/velo_oracle.c   : a plain-C restatement of the reference algorithm
 *                              (symbols prefixed velo_oracle_), and
 *   - oracle/ref_driver.cpp  : the reference's own VELO kernels compiled as CPU
 *                              C++ from their source tree (symbols prefixed velo_ref_),
 *                              built into oracle/_ref/ only where that tree exists.
 *
 * Neither is part of the product: only the tests, the smoke check and the CPU
 * baseline leg of the benchmark load them.  Every buffer they return is named
 * after the Allen argument it mirrors (e.g. "dev_sorted_velo_cluster_container")
 * and has exactly the layout and size the reference sequence gives it.
 */
#ifndef VELO_CPU_API_H
#define VELO_CPU_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  /* Allen raw-bank layout (non-MEP): payload, byte offsets per event,
   * bank sizes (u32 offsets + u16 sizes) and bank types (u32 offsets + u8 types). */
  const char* raw;
  const unsigned* raw_offsets;
  const unsigned* raw_sizes;
  const unsigned* raw_types;
  unsigned event_start; /* first event of the slice inside the arrays above */
  unsigned n_events;    /* events in the slice */
  int bank_version;     /* 2, 3 or 4; < 0 = no VP banks */
  /* velo_geometry.bin blob (format of Dumpers/BinaryDumpers/src/DumpVPGeometry.cpp) */
  const char* geometry;
  size_t geometry_size;
  /* algorithm properties (reference defaults: 0.045, 0.08, 1, 20) */
  float phi_tolerance;
  float max_scatter;
  unsigned max_skipped_modules;
  float max_chi2;
  /* beamline position in x and y (Constants::dev_beamline; beamline.bin holds 0, 0) */
  float beamline_x;
  float beamline_y;
  /* 0: super-pixel banks (VP, type 63) through velo_masked_clustering; 1: retina-cluster
   * banks (VPRetinaCluster, type 73) through decode_retinaclusters (velo_reconstruction.py:18-71) */
  int retina_decoding;
  /* 1: the four raw arrays are in the MEP layout (main/include/MEPTools.h:55-205); only the
   * reference build (velo_ref_) reads it, the restatement (velo_oracle_) refuses it */
  int mep_layout;
} VeloCpuInput;

#ifdef __cplusplus
}
#endif

#endif
