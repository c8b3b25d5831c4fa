/*
 * C ABI of the B200 (sm_100a) VELO super-pixel reconstruction (libvelo_b200.so).
 *
 * Drop-in boundary.  The reference runs this path as the Allen algorithms of
 * configuration/python/AllenConf/velo_reconstruction.py:72-292, each a
 * `struct X_t : DeviceAlgorithm, Parameters` with set_arguments_size()/operator()
 * (stream/gear/include/Algorithm.cuh:319-461), host prefix sums in between
 * (host/prefix_sum/src/HostPrefixSum.cpp:76-108).  This library replaces that whole
 * chain with one call that an Allen algorithm wrapper (or any C caller) makes:
 *
 *   inputs  (device pointers, Allen non-MEP layout, as data_provider_t produces them,
 *            host/data_provider/include/DataProvider.h:11-19):
 *       dev_velo_raw_input, dev_velo_raw_input_offsets, dev_velo_raw_input_sizes,
 *       dev_velo_raw_input_types, host_raw_bank_version, the event slice;
 *   outputs (device pointers into the chain's workspace, same layouts and names as the
 *            reference's DEVICE_OUTPUTs, velo_reconstruction.py:269-292 and :153-164):
 *       dev_offsets_estimated_input_size, dev_module_cluster_num,
 *       dev_sorted_velo_cluster_container, dev_velo_track_hits,
 *       dev_offsets_all_velo_tracks, dev_offsets_velo_track_hit_number,
 *       dev_accepted_velo_tracks, ... and the host scalars
 *       host_total_number_of_velo_clusters, host_number_of_reconstructed_velo_tracks,
 *       host_accumulated_number_of_hits_in_velo_tracks.
 *
 * Conventions: plain pointers and sizes only; every function returns a VeloStatus
 * (0 = success) instead of throwing (the reference throws from cudaCheck,
 * backend/include/CUDABackend.h:23-41); the caller owns the CUDA stream; the device workspace
 * is either the chain's own (velo_chain_reserve) or the caller's (velo_chain_sizes +
 * velo_chain_bind, outputs included).
 */
#ifndef VELO_B200_H
#define VELO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct VeloChain VeloChain;
typedef void* VeloStream; /* a cudaStream_t */

typedef enum {
  VELO_OK = 0,
  VELO_ERR_ARGUMENT = 1,       /* null pointer, bad geometry blob, unsupported bank version */
  VELO_ERR_CUDA = 2,           /* a CUDA runtime call failed; see velo_last_error_string() */
  VELO_ERR_CAPACITY = 3,       /* the slice does not fit the reserved workspace */
  VELO_ERR_DEVICE_FLAGS = 4,   /* the last run raised device status flags (velo_chain_totals) */
  VELO_ERR_NO_DEVICE = 5       /* no sm_100 device or the kernels are not loadable */
} VeloStatus;

/* Algorithm properties (reference defaults: SearchByTriplet.cuh:129-131,
 * ThreeHitTracksFilter.cuh:44). */
typedef struct {
  float phi_tolerance;          /* 0.045 */
  float max_scatter;            /* 0.08 */
  unsigned max_skipped_modules; /* 1 */
  float max_chi2;               /* 20 */
} VeloChainProperties;

/* An event slice in Allen's non-MEP raw-bank layout, on the device. */
typedef struct {
  const char* raw;          /* dev_velo_raw_input (16-byte aligned base enables bulk staging) */
  const unsigned* offsets;  /* dev_velo_raw_input_offsets [n_events + 1] */
  const unsigned* sizes;    /* dev_velo_raw_input_sizes */
  const unsigned* types;    /* dev_velo_raw_input_types */
  unsigned event_start;     /* first event of the slice (RuntimeOptions::event_interval) */
  unsigned n_events;
  int bank_version;         /* host_raw_bank_version: 2, 3 or 4 */
  int mep_layout;           /* RuntimeOptions::mep_layout: 1 = MEP layout (main/include/MEPTools.h:55-205):
                               offsets = [n_banks, n_events, source ids, per event the fragment offset
                               of every bank]; sizes and types indexed by bank, then event */
} VeloDeviceSlice;

/* The same slice on the host (page-locked memory gives asynchronous copies). */
typedef struct {
  const char* raw;
  size_t raw_bytes;
  const unsigned* offsets;
  const unsigned* sizes;
  size_t sizes_bytes;
  const unsigned* types;
  size_t types_bytes;
  unsigned n_events;
  int bank_version;
} VeloHostSlice;

/* Device pointers of the last run's outputs (valid until the next run or destroy). */
typedef struct {
  unsigned* dev_number_of_candidates;              /* [N] */
  unsigned* dev_estimated_input_size;              /* [26 N] */
  unsigned* dev_module_candidate_num;              /* [N] */
  unsigned* dev_offsets_estimated_input_size;      /* [26 N + 1] */
  unsigned* dev_module_cluster_num;                /* [26 N] */
  char* dev_sorted_velo_cluster_container;         /* [18 T] */
  void* dev_tracks;                                /* Velo::TrackHits (54 B) per entry */
  void* dev_three_hit_tracks;                      /* Velo::TrackletHits (6 B) per entry */
  uint8_t* dev_hit_used;                           /* [T] */
  unsigned* dev_atomics_velo;                      /* [3 N] */
  unsigned* dev_number_of_velo_tracks;             /* [N] */
  unsigned* dev_offsets_velo_tracks;               /* [N + 1] */
  void* dev_three_hit_tracks_output;               /* Velo::TrackletHits per entry */
  unsigned* dev_number_of_three_hit_tracks_output; /* [N] */
  unsigned* dev_offsets_number_of_three_hit_tracks_filtered; /* [N + 1] */
  unsigned* dev_offsets_all_velo_tracks;           /* [N + 1] */
  unsigned* dev_velo_track_hit_number;             /* [tracks] */
  unsigned* dev_offsets_velo_track_hit_number;     /* [tracks + 1] */
  char* dev_velo_track_hits;                       /* [18 TH] */
  uint8_t* dev_accepted_velo_tracks;               /* [tracks + three-hit tracks] */
  unsigned* dev_seed_stats;                        /* [3 N]: seed candidates met unused, candidates searched,
                                                      mode (0 plain, 1 learned, 2 gate out of bounds: plain) */
  uint8_t* dev_is_backward;                        /* [tracks] velo_kalman_filter (when enabled) */
  char* dev_velo_kalman_beamline_states;           /* [56 tracks] Velo::Consolidated::States */
  char* dev_velo_kalman_endvelo_states;            /* [56 tracks] */
  unsigned* dev_each_sensor_pair_size;             /* retina front end: [S N], S = 208 (v2/v3) or 104 (v4) */
  unsigned* dev_offsets_each_sensor_pair_size;     /* [S N + 1] */
  unsigned* dev_retina_bank_index;                 /* [S] */
  uint8_t* dev_seed_gate;                          /* [T] learned mode: 1 = the hit is searched as a seed's h1 */
  unsigned* dev_gate_stats;                        /* [2 N] learned mode: seed candidates, candidates kept */
} VeloChainOutputs;

/* Host scalars of the last run, available after velo_chain_synchronize(). */
typedef struct {
  unsigned n_events;
  unsigned host_total_number_of_velo_clusters;           /* T: estimated clusters */
  unsigned host_number_of_cluster_candidates;
  unsigned host_number_of_velo_tracks_at_least_four_hits;
  unsigned host_number_of_three_hit_tracks_filtered;
  unsigned host_number_of_reconstructed_velo_tracks;
  unsigned host_accumulated_number_of_hits_in_velo_tracks; /* TH */
  unsigned track_container_size;
  unsigned device_flags;                                 /* velo::ErrorBits raised by the kernels */
} VeloChainTotals;

/* The reference's debug-build contracts on a run's outputs, checked on the device: the
 * cluster checks of SearchByTripletContracts.cu:6-81 (per module pair the sorted container is
 * strictly increasing in (phi, id, x, y); -100 < x, y < 100 mm), its track checks (:83-120: at
 * most 26 hits, no hit twice) and lhcb_id_container_checks (VeloConsolidateTracks.cu:194-269:
 * consolidated LHCb ids non-zero with the VELO type in bits 28-31; offsets that never decrease
 * and end at the run's totals).  Counts of violations go to dev_counts[VELO_CONTRACTS] (device
 * u32, zeroed by this call); outputs in the FP32 coordinate layout (velo_chain_outputs) with
 * the totals velo_chain_synchronize() returned for them, which bound every read (from a run
 * that raised no device flag, every buffer holds at least what its total names).  Enqueued on
 * `stream` without host synchronisation and without allocation; all zero for a correct run, in
 * plain and learned mode alike. */
typedef enum {
  VELO_CONTRACT_CLUSTER_OUTSIDE = 0, /* clusters outside (-100, 100) mm in x or y */
  VELO_CONTRACT_UNSORTED = 1,        /* neighbouring clusters of a module pair out of (phi, id, x, y) order */
  VELO_CONTRACT_TRACK_SIZE = 2,      /* tracks above 26 hits (or beyond their container) */
  VELO_CONTRACT_REPEATED_HIT = 3,    /* tracks with a hit twice */
  VELO_CONTRACT_ZERO_ID = 4,         /* zero consolidated LHCb ids */
  VELO_CONTRACT_ID_TYPE = 5,         /* consolidated LHCb ids without the VELO type */
  VELO_CONTRACT_OFFSETS = 6,         /* decreasing track or hit offsets, or ends other than the totals */
  VELO_CONTRACTS = 7
} VeloContract;
VeloStatus velo_check_contracts(
  const VeloChainOutputs* outputs, const VeloChainTotals* totals, VeloStream stream, unsigned* dev_counts);

/* Library */
const char* velo_last_error_string(void);
VeloStatus velo_device_check(void); /* an sm_100 device is current and the kernels load */
void velo_default_properties(VeloChainProperties* props);

/* Replaces the per-algorithm Allen objects and Constants::dev_velo_geometry /
 * dev_velo_sp_patterns / dev_velo_sp_fx / dev_velo_sp_fy
 * (integration/non_event_data/src/VPGeometry.cpp:21-63): parses the velo_geometry.bin
 * blob and builds the super-pixel tables on the current device. */
VeloStatus velo_chain_create(
  const void* geometry, size_t geometry_size, const VeloChainProperties* props, VeloChain** chain);

/* Sizes the workspace for slices of up to max_events events and max_super_pixels
 * super pixels in total (the count follows from the bank sizes alone) and, for the
 * host-buffer path, max_raw_bytes of raw input.  Replaces the scheduler's per-algorithm
 * set_arguments_size() + arena reservation (stream/gear/include/Scheduler.cuh:353-387). */
VeloStatus velo_chain_reserve(
  VeloChain* chain, unsigned max_events, unsigned long long max_super_pixels, unsigned long long max_raw_bytes);

/* Caller-owned memory (Allen's model: the scheduler's per-stream arena owns every buffer,
 * stream/store/include/MemoryManager.cuh:100-135, sized by each algorithm's set_arguments_size,
 * stream/gear/include/Scheduler.cuh:31-137).  velo_chain_sizes() gives, for slices of up to
 * max_events events and max_super_pixels super pixels, the element count of every output the
 * caller supplies and the bytes of scratch workspace; velo_chain_bind() then makes the chain use
 * that memory instead of its own: no allocation happens in it or in the runs that follow (the
 * chain's fixed buffers, a few KB plus one 16 KiB ring per resident search CTA, come from
 * velo_chain_create / velo_chain_configure).  Binding the same memory and bounds again is free;
 * new pointers drop the cached graphs.  Outputs hold the reference's layouts and names;
 * max_reconstructed_tracks bounds host_number_of_reconstructed_velo_tracks. */
typedef struct {
  unsigned long long offsets_estimated_input_size;       /* u32 elements: 26 N + 1 */
  unsigned long long module_cluster_num;                 /* u32: 26 N */
  unsigned long long sorted_velo_cluster_container_bytes; /* 18 (FP16: 12) x T, T = 2 x super pixels + 64 */
  unsigned long long offsets_all_velo_tracks;            /* u32: N + 1 */
  unsigned long long velo_track_hit_number;              /* u32: tracks */
  unsigned long long offsets_velo_track_hit_number;      /* u32: tracks + 1 */
  unsigned long long velo_track_hits_bytes;              /* 18 (FP16: 12) x T */
  unsigned long long accepted_velo_tracks;               /* bytes: 2 x tracks */
  unsigned long long max_reconstructed_tracks;           /* tracks = max(0.34 T, 10 N) + 64 */
  unsigned long long workspace_bytes;                    /* scratch, 256-byte aligned base */
} VeloChainSizes;

typedef struct {
  unsigned* dev_offsets_estimated_input_size;
  unsigned* dev_module_cluster_num;
  char* dev_sorted_velo_cluster_container;
  unsigned* dev_offsets_all_velo_tracks;
  unsigned* dev_velo_track_hit_number;
  unsigned* dev_offsets_velo_track_hit_number;
  char* dev_velo_track_hits;
  uint8_t* dev_accepted_velo_tracks;
} VeloChainOutputBuffers; /* device pointers, 16-byte aligned (the last one any alignment) */

/* Coordinate layout of the two cluster containers a caller supplies (dev_sorted_velo_cluster_container,
 * dev_velo_track_hits): FP32, as the reference's CPU build lays out Velo::Clusters_t (half_t = float,
 * 18 bytes per element), or FP16, as its CUDA build does (half_t = half, backend/include/CUDABackend.h:14;
 * 12 bytes: u32 id[T], half xyz[3T], i16 phi[T]).  The chain computes in FP32 either way (its
 * results are the CPU build's) and, for FP16, rounds the coordinates to nearest when it writes
 * the caller's containers. */
typedef enum { VELO_COORDINATES_FP32 = 0, VELO_COORDINATES_FP16 = 1 } VeloCoordinateLayout;

VeloStatus velo_chain_sizes( /* chain may be NULL: the sizes depend on the bounds and layout alone */
  const VeloChain* chain, unsigned max_events, unsigned long long max_super_pixels, int layout, VeloChainSizes* sizes);
VeloStatus velo_chain_bind(
  VeloChain* chain,
  void* dev_workspace,
  unsigned long long workspace_bytes,
  unsigned max_events,
  unsigned long long max_super_pixels,
  int layout,
  const VeloChainOutputBuffers* outputs);

/* Enqueues the whole chain on `stream` for a device-resident slice: velo_calculate_number_of_candidates,
 * velo_estimate_input_size, velo_masked_clustering, velo_sort_by_phi, velo_search_by_triplet,
 * velo_three_hit_tracks_filter, velo_copy_track_hit_number, velo_consolidate_tracks and the
 * five prefix sums, with no host synchronisation.  When use_graph != 0 the launches are captured
 * once per (slice pointers, sizes) into a CUDA graph and replayed. */
VeloStatus velo_chain_run(VeloChain* chain, const VeloDeviceSlice* slice, VeloStream stream, int use_graph);

/* End-to-end entry for host buffers: copies the slice to the device, runs the chain and
 * copies the consolidated tracks back (dev_offsets_all_velo_tracks,
 * dev_offsets_velo_track_hit_number and dev_velo_track_hits into the host buffers given,
 * each with its capacity in bytes), then synchronises.  Reports the bytes moved. */
VeloStatus velo_chain_run_host(
  VeloChain* chain,
  const VeloHostSlice* slice,
  VeloStream stream,
  unsigned* host_offsets_all_velo_tracks,
  size_t offsets_all_capacity,
  unsigned* host_offsets_velo_track_hit_number,
  size_t offsets_hit_number_capacity,
  char* host_velo_track_hits,
  size_t track_hits_capacity,
  VeloChainTotals* totals,
  unsigned long long* h2d_bytes,
  unsigned long long* d2h_bytes);

/* Waits for the last run on its stream and returns its host scalars.  Returns
 * VELO_ERR_DEVICE_FLAGS when the kernels raised a flag (capacity, overflow). */
VeloStatus velo_chain_synchronize(VeloChain* chain, VeloChainTotals* totals);

VeloStatus velo_chain_outputs(const VeloChain* chain, VeloChainOutputs* outputs);

/* Launch configuration (no counterpart in the reference, whose block sizes are algorithm
 * PROPERTYs, e.g. SearchByTriplet.cuh:132): block size and lanes per seed candidate of the
 * search kernel (a compiled pair: (128,1) (128,2) (256,1) (256,2) (256,4) (512,2) (512,4), and
 * lanes 0 = flattened seeding, one thread per h1 candidate: (128,0) (256,0) (512,0), and with
 * search_ring_global (64,0) (96,0) (128,0) (256,0)), the shared-memory staging capacities (0:
 * staged in L2-resident global scratch, or not staged for the raw-event blobs), the work queue
 * and the clustering block size.  Chosen by allen_b200/autotune.py; the chain starts from
 * allen_b200/data/launch_config.json through the Python binding, from fixed defaults through the
 * C ABI. */
typedef struct {
  unsigned search_threads;
  unsigned search_lanes_per_seed;
  unsigned search_hit_capacity;    /* hits of an event staged in shared memory (15 B each) */
  unsigned cluster_stage_capacity; /* clusters of an event staged in shared memory (22 B each) */
  unsigned cluster_blob_bytes;     /* raw event bytes staged by the clustering kernel */
  unsigned estimate_blob_bytes;    /* raw event bytes staged by the estimate kernel */
  unsigned persistent;             /* 1: estimate, clustering and search kernels run as many CTAs
                                      as fit the device, claiming events (largest raw size first)
                                      from a work queue; 0: one CTA per event */
  unsigned events_per_claim;       /* events a persistent CTA claims at once (1..64) */
  unsigned search_ring_global;     /* 1: the search's ring of tracks to follow (16 KiB per CTA) lives in
                                      global scratch instead of shared memory, leaving room for more
                                      resident CTAs; flat seeding with 64, 96, 128 or 256 threads,
                                      persistent launches only */
  unsigned cluster_threads;        /* block size of the clustering kernel: 256, or 128 (twice the
                                      resident CTAs per SM where shared memory allows) */
  unsigned retina_order_capacity;  /* retina front end: clusters of an event ranked through key buckets
                                      in shared memory (2 B each, at most 8192, default 8192); larger
                                      events are ranked by comparing every pair of keys */
  unsigned kalman_warp_hits;       /* Kalman filter: hits of a warp's 32 tracks staged in shared memory
                                      (at most 368, default 368); longer spans are read in place */
  unsigned seed_window;            /* learned mode only: h0 candidates searched per seed candidate after the
                                      first module pair, 1..4 (0: the reference's 4, SearchByTriplet.cu:228) */
} VeloLaunchConfig;
VeloStatus velo_chain_configure(VeloChain* chain, const VeloLaunchConfig* config);
VeloStatus velo_chain_get_config(const VeloChain* chain, VeloLaunchConfig* config);

/* Per-kernel CUDA-event timing (no counterpart in the reference; its CI profiles with ncu,
 * scripts/ci/jobs/run_throughput.sh:61-67).  When enabled, every run records an event
 * between consecutive kernels, inside the captured graphs too; velo_chain_kernel_times()
 * sums, per kernel, the last execution of every cached graph (and of the last direct run)
 * and reports how many executions were summed. */
VeloStatus velo_chain_set_timing(VeloChain* chain, int enable);
unsigned velo_chain_kernel_count(void);
const char* velo_chain_kernel_name(unsigned kernel);
VeloStatus velo_chain_kernel_times(VeloChain* chain, float* ms_sum, unsigned* n_runs);

void velo_chain_destroy(VeloChain* chain);

/* Allocation-free decoding (no counterpart in the reference).  For callers that cannot
 * call cudaMalloc: code running inside a pre-reserved device-memory arena, such as an
 * Allen algorithm whose buffers all belong to the scheduler's per-stream arena.  Runs the
 * decoding half of the chain (velo_calculate_number_of_candidates, velo_estimate_input_size,
 * its prefix sum, velo_masked_clustering and velo_sort_by_phi) with the same kernels as
 * velo_chain_run() and writes dev_offsets_estimated_input_size [26 N + 1],
 * dev_module_cluster_num [26 N] and dev_sorted_velo_cluster_container (at least
 * 18 x 2 x super_pixels bytes) into caller buffers.  Its scratch is a file-scope static
 * device array of velo_noalloc_scratch_bytes() (8 MiB at most) that every GPU loading the
 * library holds until exit; slices above velo_noalloc_max_events() events or
 * 2 x super_pixels > velo_noalloc_max_clusters() are rejected with VELO_ERR_CAPACITY.
 * The first call on a device makes synchronous set-up calls (scratch address, kernel
 * attributes) and uploads the geometry on `stream`: make it before any stream capture.  All
 * calls share the scratch, which keeps the last call's contents; calls that overlap on the
 * GPU race.  The geometry is shared the same way: a call with a different blob uploads it
 * again on its own stream (not allowed inside a capture), rewriting it under any
 * overlapping call.
 * dev_status (optional, device u32) receives the kernels' error flags. */
VeloStatus velo_decode_noalloc(
  const void* geometry,
  size_t geometry_size,
  const VeloDeviceSlice* slice,
  unsigned long long super_pixels,
  VeloStream stream,
  unsigned* dev_offsets_estimated_input_size,
  unsigned* dev_module_cluster_num,
  char* dev_sorted_velo_cluster_container,
  unsigned long long container_bytes,
  unsigned* dev_status);
unsigned velo_noalloc_max_events(void);
unsigned velo_noalloc_max_clusters(void);
unsigned long long velo_noalloc_scratch_bytes(void);
const char* velo_noalloc_last_error_string(void);

/* Decoding front end.  0 (default): super-pixel banks (VP, type 63) through
 * velo_calculate_number_of_candidates, velo_estimate_input_size, velo_masked_clustering and
 * velo_sort_by_phi.  1: retina-cluster banks (VPRetinaCluster, type 73) through
 * calculate_number_of_retinaclusters_each_sensor_pair, its prefix sum and decode_retinaclusters
 * (configuration/python/AllenConf/velo_reconstruction.py:18-71, Allen's default); the search
 * then reads dev_offsets_module_pair_cluster as dev_offsets_estimated_input_size.  In retina
 * mode the kernel timings of stages 0 and 2 are retina_count_kernel and retina_decode_kernel,
 * and dev_number_of_candidates, dev_estimated_input_size and dev_module_candidate_num are not
 * produced. */
VeloStatus velo_chain_set_front_end(VeloChain* chain, int retina_clusters);

/* velo_kalman_filter (device/velo/simplified_kalman_filter/src/VeloKalmanFilter.cu:153-399,
 * wired at configuration/python/AllenConf/velo_reconstruction.py:295-322): the simplified
 * Kalman fit of every consolidated track to the beamline and to the end of the VELO.
 * velo_chain_set_kalman() appends it to the chain (outputs in VeloChainOutputs; beamline =
 * Constants::dev_beamline, 0, 0 in beamline.bin).  velo_run_kalman_filter() runs it alone on
 * caller buffers, allocating nothing: inputs are the consolidation outputs, outputs
 * dev_is_backward [tracks] and the two Velo::Consolidated::States containers (56 bytes per
 * track, 8-byte aligned).  States are bit-identical to the reference CPU build; the fields
 * the reference leaves unwritten (qop, chi2, ndof) are written as 0.  track_capacity bounds
 * the reconstructed tracks (more raise err_output_capacity in dev_status, optional). */
VeloStatus velo_chain_set_kalman(VeloChain* chain, int enable, float beamline_x, float beamline_y);
VeloStatus velo_run_kalman_filter(
  unsigned n_events,
  const unsigned* dev_offsets_all_velo_tracks,
  const unsigned* dev_offsets_velo_track_hit_number,
  const char* dev_velo_track_hits,
  unsigned track_capacity,
  float beamline_x,
  float beamline_y,
  uint8_t* dev_is_backward,
  char* dev_velo_kalman_beamline_states,
  char* dev_velo_kalman_endvelo_states,
  unsigned* dev_status,
  VeloStream stream);

/* The consolidated track views (create_velo_views,
 * device/velo/consolidate_tracks/src/VeloConsolidateTracks.cu:11-46): plain structs with the
 * layouts of Allen::Views::Velo::Consolidated::{Hits, Track, Tracks, MultiEventTracks}
 * (device/event_model/velo/include/VeloConsolidated.cuh:58-298; 24, 24, 16 and 24 bytes), so
 * that the reference's consumers (velo_kalman_filter's dev_velo_tracks_view,
 * configuration/python/AllenConf/velo_reconstruction.py:295-307) read them as their own types.
 * velo_create_velo_views() writes them from the consolidated outputs into caller buffers:
 * dev_velo_hits_view [N], dev_velo_track_view [track_capacity >= reconstructed tracks],
 * dev_velo_tracks_view [N], dev_velo_multi_event_tracks_view [1] and dev_imec_velo_tracks [1]
 * (a pointer to the multi-event view).  Allocates nothing; more tracks than track_capacity set
 * err_output_capacity in dev_status (optional) and write nothing. */
typedef struct {
  const void* base_pointer;      /* dev_velo_track_hits */
  unsigned offset;               /* the event's first track hit */
  unsigned size;                 /* the event's track hits */
  unsigned total_number_of_hits; /* track hits of the slice */
} VeloHitsView;
typedef struct {
  const VeloHitsView* hits;        /* the event's Hits view */
  unsigned track_index;            /* within the event */
  unsigned track_container_offset; /* the event's first track */
  unsigned offset;                 /* first hit of the track, relative to the event */
  unsigned number_of_hits;
} VeloTrackView;
typedef struct {
  const VeloTrackView* track; /* the event's first Track view */
  unsigned size;
  unsigned offset;
} VeloTracksView;
typedef struct {
  int type_id; /* Allen::TypeIDs::VeloTracks = 1 */
  const VeloTracksView* container;
  unsigned number_of_events;
} VeloMultiEventTracksView;
VeloStatus velo_create_velo_views(
  unsigned n_events,
  const char* dev_velo_track_hits,
  const unsigned* dev_offsets_all_velo_tracks,
  const unsigned* dev_offsets_velo_track_hit_number,
  VeloHitsView* dev_velo_hits_view,
  VeloTrackView* dev_velo_track_view,
  unsigned track_capacity,
  VeloTracksView* dev_velo_tracks_view,
  VeloMultiEventTracksView* dev_velo_multi_event_tracks_view,
  const void** dev_imec_velo_tracks,
  unsigned* dev_status,
  VeloStream stream);

/* On-device VELO validation (host/validators/src/HostVeloValidator.cpp:9-30 with
 * checker/tracking/src/PrepareTracks.cpp and TrackChecker.h:180-320 run on the host in the
 * reference): efficiency, ghost and clone counts of the consolidated tracks against Monte Carlo
 * truth, computed on the GPU.  Truth per event: LHCb ids of the truth pixels sorted ascending
 * (dev_truth_ids [truth_offsets[N]]) with the owning particle's index within the event
 * (dev_truth_owner), and per particle a reconstructible flag (dev_particle_reconstructible,
 * particle_offsets [N + 1]).  dev_matched_scratch holds n_particles u32 (zeroed here);
 * dev_counts receives 5 u64: tracks, ghosts, reconstructible, reconstructed, clones.  Rules: a
 * track matches the particle owning >= 70 % of its hits (ties to the lower index), unmatched
 * tracks are ghosts, further matches of a particle are clones.  Allocates nothing. */
VeloStatus velo_validate_tracks(
  unsigned n_events,
  const unsigned* dev_offsets_all_velo_tracks,
  const unsigned* dev_offsets_velo_track_hit_number,
  const char* dev_velo_track_hits,
  const unsigned* dev_truth_offsets,
  const unsigned* dev_truth_ids,
  const unsigned* dev_truth_owner,
  const unsigned* dev_particle_offsets,
  const uint8_t* dev_particle_reconstructible,
  unsigned n_particles,
  unsigned* dev_matched_scratch,
  unsigned long long* dev_counts,
  VeloStream stream);

/* Learned seed gate (no counterpart in the reference).  Before the triplet search, a 12-32-32-1
 * network scores every hit of module pairs 1..24 as a seed candidate (the middle hit h1 of the
 * seeding, SearchByTriplet.cu:298-446) from geometric features of its neighbours in the module
 * pairs on either side; the seeding then searches (h0 candidates, h2 windows) only the unused
 * candidates whose logit is above threshold_logit.  An event whose fraction of kept candidates
 * falls outside [kept_lo, kept_hi] is searched by the plain search instead.  Weights are used as
 * bf16 on the tensor cores (fp32 accumulation); inputs are standardised with mean / inv_std.
 * Parameter order of a flat gradient or parameter vector (VELO_SEED_PARAMS floats): w1, b1, w2,
 * b2, w3, b3. */
#define VELO_SEED_FEATURES 12
#define VELO_SEED_HIDDEN 32
#define VELO_SEED_PARAMS (32 * 12 + 32 + 32 * 32 + 32 + 32 + 1)
typedef struct {
  float w1[VELO_SEED_HIDDEN][VELO_SEED_FEATURES];
  float b1[VELO_SEED_HIDDEN];
  float w2[VELO_SEED_HIDDEN][VELO_SEED_HIDDEN];
  float b2[VELO_SEED_HIDDEN];
  float w3[VELO_SEED_HIDDEN];
  float b3;
  float mean[VELO_SEED_FEATURES];
  float inv_std[VELO_SEED_FEATURES];
  float threshold_logit;
  float kept_lo, kept_hi;
} VeloSeedModel;

/* One training record (64 bytes): a seed candidate's raw features, label 1 if the plain
 * seeding made a seed with it as middle hit, event index, h0 = 0xFFFFFFFF, and the candidate's
 * index in the sorted container.  Features: r, z, sqrt of the smallest and second smallest
 * beam-axis distance of the lines to its 4 nearest-in-phi h0 candidates, z of closest approach
 * and slope of the best line, sqrt of the smallest h2 scatter of the best and second line,
 * neighbours within twice the phi tolerance in the two module pairs, smallest |dphi| to the h0
 * candidates (rad / pi), phi (rad / pi). */
typedef struct {
  float f[VELO_SEED_FEATURES];
  float label;
  unsigned event, h0, h1;
} VeloSeedRecord;

/* model != NULL: the chain searches in learned mode (flat seeding, search_threads block size,
 * the gate kernel before the search); NULL: the plain search. */
VeloStatus velo_chain_set_seed_model(VeloChain* chain, const VeloSeedModel* model);
/* dev_records != NULL: the following runs (plain search) append one seed candidate in
 * record_every (the ones the search met unused) to dev_records (capacity entries) and count them
 * in *dev_count (device u32; entries beyond the capacity are counted, not written). */
VeloStatus velo_chain_record_seeds(
  VeloChain* chain, VeloSeedRecord* dev_records, unsigned capacity, unsigned record_every, unsigned* dev_count);

/* Training on the GPU: binary cross-entropy (positives weighted by pos_weight), mean over the
 * batch, Adam (beta1 0.9, beta2 0.999, eps 1e-8).  Forward and backward passes are warp-level
 * tensor-core kernels over 16-record tiles. */
typedef struct VeloSeedTrainer VeloSeedTrainer;
VeloStatus velo_seed_trainer_create(
  const VeloSeedModel* init, float learning_rate, float pos_weight, VeloSeedTrainer** trainer);
/* One Adam step on records [first, first + batch).  loss (optional, host) receives the
 * batch's mean loss and makes the call synchronous. */
VeloStatus velo_seed_trainer_step(
  VeloSeedTrainer* trainer,
  const VeloSeedRecord* dev_records,
  unsigned long long first,
  unsigned batch,
  VeloStream stream,
  float* loss);
/* Gradients (VELO_SEED_PARAMS floats, host) and mean loss of a batch, without a step. */
VeloStatus velo_seed_trainer_gradients(
  VeloSeedTrainer* trainer,
  const VeloSeedRecord* dev_records,
  unsigned long long first,
  unsigned batch,
  VeloStream stream,
  float* grads,
  float* loss);
/* Logits of records [0, n) into dev_logits (device floats) with the current weights. */
VeloStatus velo_seed_trainer_score(
  VeloSeedTrainer* trainer, const VeloSeedRecord* dev_records, unsigned long long n, float* dev_logits, VeloStream stream);
/* The current fp32 weights, with the standardisation, threshold and bounds of the model. */
VeloStatus velo_seed_trainer_model(VeloSeedTrainer* trainer, VeloSeedModel* model);
void velo_seed_trainer_destroy(VeloSeedTrainer* trainer);

/* Utilities (synchronous copies on the current device), for callers without a CUDA runtime binding. */
VeloStatus velo_copy_to_host(void* host, const void* device, size_t bytes);
VeloStatus velo_copy_to_device(void* device, const void* host, size_t bytes);
/* Asynchronous device-to-host copy on `stream` (page-locked host memory overlaps with compute). */
VeloStatus velo_copy_to_host_async(void* host, const void* device, size_t bytes, VeloStream stream);

#ifdef __cplusplus
}
#endif

#endif
