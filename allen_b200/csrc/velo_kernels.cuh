// Kernel parameter blocks and launch declarations of the VELO chain (sm_100a).
#pragma once

#include "velo_common.cuh"
#include "velo_mlp.cuh"

namespace velo {

  // ---- persistent launches: a CTA claims events from a global counter ----
  // next == null: one CTA per event (blockIdx.x).  Otherwise the grid holds as many CTAs as
  // fit on the device at once and each claims `chunk` events at a time, in `order` (largest
  // events first) when given.  Results do not depend on which CTA processes an event.
  struct WorkQueue {
    unsigned* next;
    const unsigned* order;
    unsigned chunk;
  };

  // Calls body(event, call) for the events of this CTA; call counts the CTA's events.  One
  // call site for the body, so it is inlined once.
  template<typename Body>
  __device__ __forceinline__ void for_each_event(const WorkQueue& q, unsigned n, Body&& body)
  {
    __shared__ unsigned claimed;
    const bool queued = q.next != nullptr;
    unsigned first = blockIdx.x, last = blockIdx.x + 1, call = 0;
    for (bool once = true;; once = false) {
      if (queued) {
        if (threadIdx.x == 0) claimed = atomicAdd(q.next, q.chunk);
        __syncthreads();
        first = claimed;
        __syncthreads(); // read before thread 0 claims again
        if (first >= n) break;
        last = min(first + q.chunk, n);
      }
      else if (!once) {
        break;
      }
      for (unsigned k = first; k < last; ++k) {
        body(queued && q.order ? q.order[k] : k, call++);
        __syncthreads(); // the next event reuses the shared memory
      }
    }
  }

  // ---- decoding: velo_calculate_number_of_candidates + velo_estimate_input_size ----
  struct EstimateParams {
    RawInput in;
    unsigned* estimated_input_size;       // [26 N] dev_estimated_input_size
    unsigned* number_of_candidates;       // [N]    dev_number_of_candidates
    unsigned* module_candidate_num;       // [N]    dev_module_candidate_num
    unsigned* event_estimate;             // [N]    sum of the event's 26 estimates
    unsigned long long* bank_index_key;   // [208]  (event << 32 | bank), max-reduced
    unsigned designated_stride;           // events e with e % stride == 0 set the bank index
    unsigned* status;
    unsigned smem_blob_bytes;
    // sorted bank copies for this kernel's neighbour search and the clustering kernel's (null:
    // full scans): each event takes total_sp words of sp_scratch from the counter sp_alloc
    // (zeroed before the launch) and records where in sp_base[e] (no_sorted_copy: no room)
    uint32_t* sp_scratch;
    unsigned sp_capacity;
    unsigned* sp_alloc;
    unsigned* sp_base;
    WorkQueue queue;
  };

  constexpr unsigned no_sorted_copy = 0xFFFFFFFFu;

  // ---- masked clustering + phi + sort by phi, one event per CTA ----
  struct ClusterSortParams {
    RawInput in;
    const Geometry* geo;
    Constants k;
    const unsigned* estimated_input_size;       // [26 N]
    const unsigned* event_base;                 // [N + 1] exclusive scan of event_estimate
    const unsigned long long* bank_index_key;   // [208]
    unsigned* offsets_estimated_input_size;     // [26 N + 1] dev_offsets_estimated_input_size
    unsigned* module_cluster_num;               // [26 N]     dev_module_cluster_num
    char* sorted_container;                     // [18 T]     dev_sorted_velo_cluster_container
    char* staging;                              // [24 T]     fallback staging for large events
    const unsigned* candidates_offsets;         // [N + 1] dev_candidates_offsets (2 x SP words per event)
    uint32_t* sp_scratch;                       // [S] sorted bank copies of events whose copies do not
                                                //     fit the shared-memory blob (null: full scans)
    unsigned sp_capacity;                       // S, allocated words of sp_scratch
    const unsigned* sp_base;                    // [N] where the estimate kernel sorted each event's banks
                                                //     in sp_scratch (null: this kernel sorts them)
    unsigned* status;
    unsigned smem_blob_bytes;
    unsigned smem_cluster_capacity;             // clusters staged in shared memory per event
    unsigned cluster_capacity;                  // allocated T of the containers
    WorkQueue queue;
  };

  // ---- search by triplet + three-hit filter, one event per CTA ----
  struct SearchParams {
    Geometry const* geo;
    Constants k;
    unsigned n_events;
    const unsigned* offsets_estimated_input_size; // [26 N + 1]
    const unsigned* module_cluster_num;           // [26 N]
    const char* sorted_container;                 // [18 T]
    unsigned track_capacity;                      // allocated entries of the track containers
    TrackHits* tracks;                            // dev_tracks
    TrackletHits* three_hit_tracks;               // dev_three_hit_tracks
    bool* hit_used;                               // [T] dev_hit_used
    unsigned* atomics_velo;                       // [3 N] dev_atomics_velo
    unsigned* number_of_velo_tracks;              // [N] dev_number_of_velo_tracks
    TrackletHits* three_hit_tracks_output;        // dev_three_hit_tracks_output
    unsigned* number_of_three_hit_tracks_output;  // [N]
    unsigned* event_track_hits;                   // [N] hits of the event's consolidated tracks
    unsigned* status;
    unsigned smem_hit_capacity;                   // hits staged in shared memory per event
    unsigned cluster_capacity;                    // allocated T of the containers
    char* hit_scratch;                            // [16 T] staging of events above the capacity
    uint64_t* ring_scratch;                       // [2048 grid] rings of tracks to follow (RING = 1)
    // learned seed gate (search_by_triplet_gated_kernel): a byte per hit, 0 = the hit is not
    // searched as a seed's middle hit; null = the plain search
    const uint8_t* seed_gate;                     // [T]
    const unsigned* gate_stats;                   // [2 N] seed candidates, candidates the gate keeps
    float kept_lo, kept_hi;                       // an event whose kept fraction is outside: plain search
    unsigned* seed_stats;                         // [3 N] candidates met, candidates searched, mode
    uint8_t* h1_outcome;                          // [T] training labels (gated kernel): 1 no seed, 2 seed
    unsigned seed_window;                         // learned mode: h0 candidates per seed candidate after
                                                  // the first module pair (0: the reference's 4)
    WorkQueue queue;
  };

  // seed_stats mode: the search that produced the event's tracks
  constexpr unsigned seed_mode_plain = 0, seed_mode_learned = 1, seed_mode_fallback = 2;

  // ---- copy_track_hit_number + consolidate_tracks, one event per CTA ----
  struct ConsolidateParams {
    unsigned n_events;
    const unsigned* offsets_estimated_input_size;
    const char* sorted_container;
    const TrackHits* tracks;
    const TrackletHits* three_hit_tracks_output;
    const unsigned* offsets_velo_tracks;                  // [N + 1]
    const unsigned* offsets_three_hit;                    // [N + 1]
    const unsigned* event_track_hit_base;                 // [N + 1]
    unsigned* offsets_all_velo_tracks;                    // [N + 1]
    unsigned* velo_track_hit_number;                      // [tracks]
    unsigned* offsets_velo_track_hit_number;              // [tracks + 1]
    char* velo_track_hits;                                // [18 TH]
    bool* accepted_velo_tracks;
    unsigned track_capacity;            // consolidated tracks
    unsigned track_container_capacity;  // entries of dev_tracks / three-hit containers
    unsigned track_hit_capacity;
    unsigned cluster_capacity;
    unsigned* status;
  };

  struct ScanJob {
    const unsigned* in;
    unsigned* out; // n + 1 entries: exclusive scan, total in the last
    unsigned n;
  };
  struct ScanParams {
    ScanJob jobs[4];
  };

  // Dynamic shared memory of cluster_sort_kernel for a staging capacity of `cap` clusters:
  // [cap x 18 B clusters][cap x u16 slot in bucket][cap x u16 members][u16 bucket counters][blob]
  constexpr unsigned sort_buckets = 128;
  constexpr unsigned sort_counters = n_module_pairs * sort_buckets;
  __host__ __device__ constexpr unsigned cluster_sort_counter_offset(unsigned cap)
  {
    return ((cap * (element_size + 4)) + 15u) & ~15u;
  }
  __host__ __device__ constexpr unsigned cluster_sort_blob_offset(unsigned cap)
  {
    return cluster_sort_counter_offset(cap) + ((sort_counters * 2 + 15u) & ~15u);
  }

  __global__ void estimate_kernel(EstimateParams p);
  template<unsigned THREADS> // 128 or 256
  __global__ void cluster_sort_kernel(ClusterSortParams p);
  template<unsigned THREADS, unsigned LPH, unsigned RING>
  __global__ void search_by_triplet_kernel(SearchParams p);
  // flat seeding behind the learned seed gate (and seed-candidate outcome recording);
  // RING = 1: the ring of tracks to follow in global scratch (persistent launches)
  template<unsigned THREADS, unsigned RING>
  __global__ void search_by_triplet_gated_kernel(SearchParams p);
#define VELO_GATED_CONFIGS(X) X(128, 0) X(256, 0) X(512, 0) X(128, 1) X(256, 1) X(96, 1) X(64, 1)
  // (block size, lanes per seed candidate) pairs compiled for the autotuner
// lanes 0 = flattened seeding (one thread per h1 candidate)
#define VELO_SEARCH_CONFIGS(X)                                                                                  \
  X(128, 1, 0) X(128, 2, 0) X(256, 1, 0) X(256, 2, 0) X(256, 4, 0) X(512, 2, 0) X(512, 4, 0) X(128, 0, 0) X(256, 0, 0) \
    X(512, 0, 0) X(128, 0, 1) X(256, 0, 1) X(96, 0, 1) X(64, 0, 1)
  __global__ void consolidate_kernel(ConsolidateParams p);
  // ---- retina-cluster decoding (VPRetinaCluster banks) ----
  struct RetinaParams {
    RawInput in;
    const Geometry* geo;
    Constants k;
    unsigned* each_sensor_pair_size;         // [S N] dev_each_sensor_pair_size (S = 208 v2/v3, 104 v4)
    unsigned* bank_index;                    // [S]   dev_retina_bank_index (zeroed before the count)
    unsigned* event_total;                   // [N]   clusters per event
    const unsigned* event_base;              // [N + 1] exclusive scan of event_total
    unsigned* offsets_each_sensor_pair_size; // [S N + 1]
    unsigned* offsets_module_pair_cluster;   // [26 N + 1] the search's dev_offsets_estimated_input_size
    unsigned* module_cluster_num;            // [26 N]
    char* container;                         // [18 T] dev_velo_cluster_container (sorted)
    long long* key_scratch;                  // [T] cluster keys of the events not keyed in shared memory
    unsigned* status;
    unsigned smem_key_capacity;              // clusters of an event keyed in shared memory
    unsigned smem_order_capacity;            // clusters of an event ranked through key buckets
    unsigned cluster_capacity;               // allocated T
  };
  __global__ void retina_count_kernel(RetinaParams p);
  __global__ void retina_decode_kernel(RetinaParams p);

  // ---- velo_kalman_filter: one thread per consolidated track ----
  struct KalmanParams {
    unsigned n_events;
    const unsigned* offsets_all_velo_tracks;       // [N + 1]
    const unsigned* offsets_velo_track_hit_number; // [tracks + 1]
    const char* velo_track_hits;                   // consolidated hits (ids, then x y z)
    float beamline_x, beamline_y;                  // Constants::dev_beamline
    unsigned track_capacity;                       // entries of the outputs
    uint8_t* is_backward;                          // [tracks] dev_is_backward
    unsigned warp_hits;                            // hits of a warp's tracks staged (<= kalman_warp_hits)
    unsigned abort_flags;                          // status bits that mean the inputs were not written
    float* beamline_states;                        // [14 tracks] dev_velo_kalman_beamline_states
    float* endvelo_states;                         // [14 tracks] dev_velo_kalman_endvelo_states
    unsigned* status;
  };
  __global__ void kalman_filter_kernel(KalmanParams p);

  // The sorted cluster container and the consolidated track hits re-encoded with half-precision
  // coordinates (12 bytes per element: u32 id[T], half xyz[3T], i16 phi[T]), the layout of
  // Velo::Clusters_t when half_t is half (backend/include/CUDABackend.h, VeloEventModel.cuh:92-189).
  struct HalfExportParams {
    unsigned n_events;
    const unsigned* offsets_estimated_input_size;
    const char* sorted_container;
    const unsigned* offsets_all_velo_tracks;
    const unsigned* offsets_velo_track_hit_number;
    const char* velo_track_hits;
    unsigned cluster_capacity, track_capacity, track_hit_capacity;
    char* sorted_half;
    char* track_hits_half;
    unsigned* status;
  };
  __global__ void export_half_kernel(HalfExportParams p);

  // order[0..n) = the slice's events by raw size, largest first (one CTA)
  __global__ void event_order_kernel(RawInput in, unsigned* order);
  __global__ void exclusive_scan_kernel(ScanParams p);

  // Phi buckets of a module pair's sorted hits, shared by the search and the seed gate:
  // bucket[b] = first index with phi >= b * 512 - 32768 (128 buckets + the end).
  constexpr unsigned n_buckets = 128;
  __device__ __forceinline__ unsigned bucket_of(int16_t v) { return static_cast<unsigned>(v + 32768) >> 9; }

  // binary_search_leftmost (BinarySearch.cuh:15-30) through the bucket table of the
  // module pair: the first index with phi >= value.
  __device__ __forceinline__ int leftmost(const uint16_t* table, const int16_t* phis, unsigned n, int16_t value)
  {
    unsigned i = table[bucket_of(value)];
    while (i < n && phis[i] < value)
      ++i;
    return static_cast<int>(i);
  }

  // The bucket table of one module pair, hits [s0, s0 + cnt) (one CTA; phi_of(i) = phi of
  // the event's hit i).
  template<typename PhiOf>
  __device__ __forceinline__ void build_bucket_table_of(uint16_t* t, PhiOf phi_of, unsigned s0, unsigned cnt)
  {
    for (unsigned i = threadIdx.x; i <= cnt; i += blockDim.x) {
      const unsigned lo = i == 0 ? 0u : bucket_of(phi_of(s0 + i - 1)) + 1;
      const unsigned hi = i == cnt ? n_buckets : bucket_of(phi_of(s0 + i));
      for (unsigned b = lo; b <= hi; ++b)
        t[b] = static_cast<uint16_t>(i);
    }
  }

  // The bucket tables of an event's 26 module pairs (phis event-relative).
  __device__ __forceinline__ void build_bucket_tables(
    uint16_t (*table)[n_buckets + 1], const int16_t* phis, const unsigned* start, const unsigned* num, unsigned hit_offset)
  {
    for (unsigned mp = 0; mp < n_module_pairs; ++mp)
      build_bucket_table_of(table[mp], [phis](unsigned i) { return phis[i]; }, start[mp] - hit_offset, num[mp]);
  }

  // ---- learned seed gate (velo_gate.cu): one byte per hit, 1 = searched as a seed's middle hit ----
  struct GateParams {
    Geometry const* geo;
    Constants k;
    unsigned n_events;
    const unsigned* offsets_estimated_input_size;
    const unsigned* module_cluster_num;
    const char* sorted_container;
    unsigned cluster_capacity;
    const MlpModelDevice* model; // inference
    uint8_t* gate;               // [T] inference output
    unsigned* gate_stats;        // [2 N] seed candidates (hits of module pairs 1..24), kept
    const uint8_t* h1_outcome;   // [T] recording input: 1 no seed, 2 seed (from the search)
    SeedRecord* records;         // recording output
    unsigned* record_count;
    unsigned record_capacity;
    unsigned record_every;       // one candidate in record_every (hash of event and hit)
    unsigned* status;
  };
  template<bool RECORD>
  __global__ void seed_gate_kernel(GateParams p);
  constexpr unsigned gate_threads = 128; // one 128-row tensor-core tile of candidates per round

  // Raises a kernel's dynamic shared-memory limit to at least `bytes`, never lowers it: the
  // limit is per kernel and per device, shared by every chain and entry point in the process.
  inline cudaError_t raise_dynamic_smem_limit(const void* kernel, int bytes)
  {
    cudaFuncAttributes a;
    const cudaError_t e = cudaFuncGetAttributes(&a, kernel);
    if (e != cudaSuccess) return e;
    if (a.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  }

  constexpr unsigned decode_threads = 256;
  constexpr unsigned kalman_threads = 256;
  constexpr unsigned kalman_ctas_per_sm = 6; // 40 registers a thread; the grid is one wave of the device
  constexpr unsigned kalman_warp_hits = 368; // hits of a warp's 32 tracks staged in shared memory (4.4 KB)
  constexpr unsigned scan_threads = 1024;
  constexpr unsigned consolidate_threads = 256;
  constexpr unsigned search_hit_bytes = 16; // one record (x, y, z, phi, flags) per staged hit

} // namespace velo

// Host helpers shared by the chain and the allocation-free entry point (velo_chain.cu).
namespace velo_host {
  // cache_sp_patterns (ClusteringCommon.cpp:6-104): SP pattern byte and centroid fractions
  void build_sp_tables(uint8_t* patterns, float* fx, float* fy);
  // velo_geometry.bin (integration/non_event_data/src/VPGeometry.cpp:21-63); false if malformed
  bool parse_geometry(const char* blob, size_t size, velo::Geometry& g);
} // namespace velo_host
