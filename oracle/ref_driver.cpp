/*
 * Test infrastructure (oracle side): drives the reference's own VELO kernels,
 * compiled as CPU C++ (TARGET_DEVICE_CPU, blockDim = 1, sequential atomics),
 * through the same steps the reference sequence takes, without its scheduler.
 *
 * Sequence followed: configuration/python/AllenConf/velo_reconstruction.py:72-164
 * (decode_velo, retina_decoding=False) and :167-292 (make_velo_tracks).
 * Each step below restates the body of the algorithm's operator(): its memsets,
 * buffer sizes and grid, then calls the reference kernel once per block index,
 * exactly as stream/gear/include/Invoke.cuh:40-52 does for the CPU target.
 *
 * This file contains no reference code; it includes the reference headers and
 * links the reference objects built from their own source files by
 * oracle/Makefile.  Output goes to oracle/_ref/.
 */
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "VeloCalculateNumberOfCandidates.cuh"
#include "EstimateInputSize.cuh"
#include "MaskedVeloClustering.cuh"
#include "SortByPhi.cuh"
#include "SearchByTriplet.cuh"
#include "ThreeHitTracksFilter.cuh"
#include "VeloCopyTrackHitNumber.cuh"
#include "VeloConsolidateTracks.cuh"
#include "VeloKalmanFilter.cuh"
#include "CalculateNumberOfRetinaClustersPerSensor.cuh"
#include "DecodeRetinaClusters.cuh"
#include "HostPrefixSum.h"
#include "ClusteringCommon.h"

#include "../velo_cpu_api.h"

// Kernel templates instantiated inside the reference translation units.
template<int decoding_version, bool mep_layout>
__global__ void velo_calculate_number_of_candidates_kernel(
  velo_calculate_number_of_candidates::Parameters parameters,
  const unsigned number_of_events,
  const unsigned event_start);
template<int decoding_version, bool mep_layout>
__global__ void velo_estimate_input_size_kernel(velo_estimate_input_size::Parameters parameters, unsigned const event_start);
template<int decoding_version, bool mep_layout>
__global__ void velo_masked_clustering_kernel(
  velo_masked_clustering::Parameters parameters,
  const unsigned event_start,
  const VeloGeometry* dev_velo_geometry,
  const uint8_t* dev_velo_sp_patterns,
  const float* dev_velo_sp_fx,
  const float* dev_velo_sp_fy);

template<int decoding_version, bool mep_layout>
__global__ void calculate_number_of_retinaclusters_each_sensor_pair_kernel(
  calculate_number_of_retinaclusters_each_sensor_pair::Parameters parameters,
  const unsigned event_start);
template<int decoding_version>
__global__ void populate_module_pair_offsets_and_sizes(
  decode_retinaclusters::Parameters parameters,
  const unsigned module_pair_cluster_num_size);
template<int decoding_version, bool mep_layout>
__global__ void velo_calculate_sorting_key(
  decode_retinaclusters::Parameters parameters,
  const unsigned event_start,
  const VeloGeometry* dev_velo_geometry,
  unsigned* dev_module_pair_zero_cluster_num);
template<bool mep_layout>
__global__ void velo_calculate_permutations(
  decode_retinaclusters::Parameters parameters,
  unsigned* dev_module_pair_zero_cluster_num);
template<int decoding_version, bool mep_layout>
__global__ void decode_retinaclusters_sorted(
  decode_retinaclusters::Parameters parameters,
  const unsigned event_start,
  const VeloGeometry* dev_velo_geometry);

// VeloConsolidateTracks.cu:11-46 (defined at file scope there)
__global__ void create_velo_views(velo_consolidate_tracks::Parameters parameters);

namespace {
  using Allen::device::span;

  // Uninitialised storage for n objects of a view type the reference constructs in place.
  template<typename T>
  struct ViewStorage {
    std::vector<std::max_align_t> raw;
    explicit ViewStorage(size_t n) : raw((n * sizeof(T) + sizeof(std::max_align_t) - 1) / sizeof(std::max_align_t) + 1) {}
    T* data() { return reinterpret_cast<T*>(raw.data()); }
  };

  struct Buffer {
    void* p = nullptr;
    size_t n = 0;
  };

  struct Result {
    std::map<std::string, Buffer> buffers;
    ~Result()
    {
      for (auto& kv : buffers)
        std::free(kv.second.p);
    }
    // 64-byte aligned, zero-initialised (host_prefix_sum_impl uses aligned SSE loads).
    template<typename T>
    T* make(const std::string& name, size_t count)
    {
      const size_t bytes = std::max<size_t>(64, ((count * sizeof(T) + 63) / 64) * 64);
      void* p = std::aligned_alloc(64, bytes);
      std::memset(p, 0, bytes);
      auto& b = buffers[name];
      std::free(b.p);
      b.p = p;
      b.n = count * sizeof(T);
      return static_cast<T*>(p);
    }
  };

  template<typename T>
  span<T> sp(T* p, size_t n)
  {
    return span<T> {p, n};
  }

  // host_prefix_sum_t::operator() (host/prefix_sum/src/HostPrefixSum.cpp:76-108, CPU branch)
  unsigned prefix_sum(Result& r, const std::string& out_name, const unsigned* in, size_t n)
  {
    unsigned* out = r.make<unsigned>(out_name, n + 1);
    out[0] = 0;
    std::memcpy(out + 1, in, n * sizeof(unsigned));
    unsigned total = 0;
    host_prefix_sum::host_prefix_sum_impl(out, n + 1, &total);
    return total;
  }

  template<typename Kernel>
  void launch(unsigned grid, Kernel&& k)
  {
    gridDim = {grid, 1, 1};
    for (unsigned i = 0; i < grid; ++i) {
      blockIdx = {i, 0, 0};
      k();
    }
  }

  template<int V, bool MEP>
  Result* run_chain(const VeloCpuInput& in)
  {
    auto* r = new Result;
    const unsigned n = in.n_events;
    const unsigned start = in.event_start;
    // Payload spans: only their data pointers are read by the kernels.
    const size_t big = size_t(1) << 40;

    std::vector<mask_t> event_list(n);
    for (unsigned i = 0; i < n; ++i)
      event_list[i].m_data = i;
    unsigned host_n = n;
    unsigned dev_n = n;
    int bank_version = in.bank_version;

    // Constants: SP tables (host/velo/clustering/src/ClusteringCommon.cpp) and geometry.
    std::vector<uint8_t> sp_patterns(256, 0), sp_sizes(256, 0);
    std::vector<float> sp_fx(512, 0), sp_fy(512, 0);
    cache_sp_patterns(sp_patterns, sp_sizes, sp_fx, sp_fy);
    const VeloGeometry geometry {std::vector<char>(in.geometry, in.geometry + in.geometry_size)};

    unsigned total_clusters = 0;
    const unsigned* offsets_est = nullptr;
    unsigned* cluster_num = nullptr;
    char* sorted = nullptr;
    std::vector<Velo::Clusters> clusters_views(n);
    // VPRetinaCluster banks (velo_reconstruction.py:18-71): each_sensor_pair_size, its prefix
    // sum and decode_retinaclusters (DecodeRetinaClusters.cu:433-504) give the same three
    // inputs of the search: offsets per module pair, cluster counts, sorted container.
    if (in.retina_decoding) {
      const unsigned per_event = (V == 2 || V == 3) ? Velo::Constants::n_modules * 4 : Velo::Constants::n_modules * 2;
      unsigned* pair_size = r->make<unsigned>("dev_each_sensor_pair_size", size_t(n) * per_event);
      unsigned* retina_bank_index = r->make<unsigned>("dev_retina_bank_index", per_event);
      {
        calculate_number_of_retinaclusters_each_sensor_pair::Parameters p {};
        p.host_number_of_events = sp<const unsigned>(&host_n, 1);
        p.host_raw_bank_version = sp<const int>(&bank_version, 1);
        p.dev_event_list = sp<const mask_t>(event_list.data(), n);
        p.dev_velo_retina_raw_input = sp<const char>(in.raw, big);
        p.dev_velo_retina_raw_input_offsets = sp<const unsigned>(in.raw_offsets, big);
        p.dev_velo_retina_raw_input_sizes = sp<const unsigned>(in.raw_sizes, big);
        p.dev_velo_retina_raw_input_types = sp<const unsigned>(in.raw_types, big);
        p.dev_retina_bank_index = sp<unsigned>(retina_bank_index, per_event);
        p.dev_each_sensor_pair_size = sp<unsigned>(pair_size, size_t(n) * per_event);
        if (bank_version >= 0) launch(n, [&] { calculate_number_of_retinaclusters_each_sensor_pair_kernel<V, MEP>(p, start); });
      }
      total_clusters = prefix_sum(*r, "dev_offsets_each_sensor_pair_size", pair_size, size_t(n) * per_event);
      const unsigned* pair_offsets = static_cast<unsigned*>(r->buffers["dev_offsets_each_sensor_pair_size"].p);
      cluster_num = r->make<unsigned>("dev_module_cluster_num", size_t(n) * 26);
      unsigned* offsets_mp = r->make<unsigned>("dev_offsets_estimated_input_size", size_t(n) * 26 + 1);
      sorted = r->make<char>("dev_sorted_velo_cluster_container", size_t(total_clusters) * Velo::Clusters::element_size);
      unsigned* permutations = r->make<unsigned>("dev_hit_permutations", total_clusters);
      int64_t* keys = r->make<int64_t>("dev_hit_sorting_key", total_clusters);
      std::vector<unsigned> zero_num(size_t(n) * 26, 0);
      decode_retinaclusters::Parameters p {};
      p.host_total_number_of_velo_clusters = sp<const unsigned>(&total_clusters, 1);
      p.host_raw_bank_version = sp<const int>(&bank_version, 1);
      p.host_number_of_events = sp<const unsigned>(&host_n, 1);
      p.dev_velo_retina_raw_input = sp<const char>(in.raw, big);
      p.dev_velo_retina_raw_input_offsets = sp<const unsigned>(in.raw_offsets, big);
      p.dev_velo_retina_raw_input_sizes = sp<const unsigned>(in.raw_sizes, big);
      p.dev_velo_retina_raw_input_types = sp<const unsigned>(in.raw_types, big);
      p.dev_offsets_each_sensor_pair_size = sp<const unsigned>(pair_offsets, size_t(n) * per_event + 1);
      p.dev_retina_bank_index = sp<const unsigned>(retina_bank_index, per_event);
      p.dev_event_list = sp<const mask_t>(event_list.data(), n);
      p.dev_number_of_events = sp<const unsigned>(&dev_n, 1);
      p.dev_module_pair_cluster_num = sp<unsigned>(cluster_num, size_t(n) * 26);
      p.dev_offsets_module_pair_cluster = sp<unsigned>(offsets_mp, size_t(n) * 26 + 1);
      p.dev_velo_cluster_container = sp<char>(sorted, size_t(total_clusters) * Velo::Clusters::element_size);
      p.dev_hit_permutations = sp<unsigned>(permutations, total_clusters);
      p.dev_hit_sorting_key = sp<int64_t>(keys, total_clusters);
      p.dev_velo_clusters = sp<Velo::Clusters>(clusters_views.data(), n);
      if (bank_version >= 0) {
        const unsigned size = n * 26;
        const unsigned block = Velo::Tracking::block_dim_x_populate_module_pair_offsets_and_sizes;
        launch((size + block - 1) / block, [&] { populate_module_pair_offsets_and_sizes<V>(p, size); });
        launch(n, [&] { velo_calculate_sorting_key<V, MEP>(p, start, &geometry, zero_num.data()); });
        launch(n, [&] { velo_calculate_permutations<MEP>(p, zero_num.data()); });
        launch(n, [&] { decode_retinaclusters_sorted<V, MEP>(p, start, &geometry); });
      }
      offsets_est = offsets_mp;
    }
    else {
      // 1. velo_calculate_number_of_candidates (VeloCalculateNumberOfCandidates.cu:50-86)
      unsigned* n_candidates = r->make<unsigned>("dev_number_of_candidates", n);
      unsigned* bank_index = r->make<unsigned>("dev_velo_bank_index", Velo::Constants::n_modules * 4);
      {
        velo_calculate_number_of_candidates::Parameters p {};
        p.host_number_of_events = sp<const unsigned>(&host_n, 1);
        p.host_raw_bank_version = sp<const int>(&bank_version, 1);
        p.dev_event_list = sp<const mask_t>(event_list.data(), n);
        p.dev_velo_raw_input = sp<const char>(in.raw, big);
        p.dev_velo_raw_input_offsets = sp<const unsigned>(in.raw_offsets, big);
        p.dev_velo_raw_input_sizes = sp<const unsigned>(in.raw_sizes, big);
        p.dev_velo_raw_input_types = sp<const unsigned>(in.raw_types, big);
        p.dev_number_of_candidates = sp<unsigned>(n_candidates, n);
        p.dev_velo_bank_index = sp<unsigned>(bank_index, Velo::Constants::n_modules * 4);
        if (bank_version >= 0) {
          launch((n + 255) / 256, [&] { velo_calculate_number_of_candidates_kernel<V, MEP>(p, n, start); });
        }
      }

      // 2. prefix_sum_offsets_velo_candidates
      const unsigned total_candidates = prefix_sum(*r, "dev_candidates_offsets", n_candidates, n);
      const unsigned* candidates_offsets = static_cast<unsigned*>(r->buffers["dev_candidates_offsets"].p);

      // 3. velo_estimate_input_size (EstimateInputSize.cu:241-281)
      unsigned* estimated = r->make<unsigned>("dev_estimated_input_size", size_t(n) * 26);
      unsigned* candidate_num = r->make<unsigned>("dev_module_candidate_num", n);
      unsigned* candidates = r->make<unsigned>("dev_cluster_candidates", total_candidates);
      {
        velo_estimate_input_size::Parameters p {};
        p.host_number_of_events = sp<const unsigned>(&host_n, 1);
        p.host_number_of_cluster_candidates = sp<const unsigned>(&total_candidates, 1);
        p.host_raw_bank_version = sp<const int>(&bank_version, 1);
        p.dev_event_list = sp<const mask_t>(event_list.data(), n);
        p.dev_candidates_offsets = sp<const unsigned>(candidates_offsets, n + 1);
        p.dev_velo_raw_input = sp<const char>(in.raw, big);
        p.dev_velo_raw_input_offsets = sp<const unsigned>(in.raw_offsets, big);
        p.dev_velo_raw_input_sizes = sp<const unsigned>(in.raw_sizes, big);
        p.dev_velo_raw_input_types = sp<const unsigned>(in.raw_types, big);
        p.dev_estimated_input_size = sp<unsigned>(estimated, size_t(n) * 26);
        p.dev_module_candidate_num = sp<unsigned>(candidate_num, n);
        p.dev_cluster_candidates = sp<unsigned>(candidates, total_candidates);
        if (bank_version >= 0) {
          launch(n, [&] { velo_estimate_input_size_kernel<V, MEP>(p, start); });
        }
      }

      // 4. prefix_sum_offsets_estimated_input_size
      total_clusters = prefix_sum(*r, "dev_offsets_estimated_input_size", estimated, size_t(n) * 26);
      offsets_est = static_cast<unsigned*>(r->buffers["dev_offsets_estimated_input_size"].p);

      // 5. velo_masked_clustering (MaskedVeloClustering.cu:578-619)
      cluster_num = r->make<unsigned>("dev_module_cluster_num", size_t(n) * 26);
      char* container = r->make<char>("dev_velo_cluster_container", size_t(total_clusters) * Velo::Clusters::element_size);
      {
        velo_masked_clustering::Parameters p {};
        p.host_total_number_of_velo_clusters = sp<const unsigned>(&total_clusters, 1);
        p.host_number_of_events = sp<const unsigned>(&host_n, 1);
        p.host_raw_bank_version = sp<const int>(&bank_version, 1);
        p.dev_velo_raw_input = sp<const char>(in.raw, big);
        p.dev_velo_raw_input_offsets = sp<const unsigned>(in.raw_offsets, big);
        p.dev_velo_raw_input_sizes = sp<const unsigned>(in.raw_sizes, big);
        p.dev_velo_raw_input_types = sp<const unsigned>(in.raw_types, big);
        p.dev_offsets_estimated_input_size = sp<const unsigned>(offsets_est, size_t(n) * 26 + 1);
        p.dev_module_pair_candidate_num = sp<const unsigned>(candidate_num, n);
        p.dev_cluster_candidates = sp<const unsigned>(candidates, total_candidates);
        p.dev_event_list = sp<const mask_t>(event_list.data(), n);
        p.dev_candidates_offsets = sp<const unsigned>(candidates_offsets, n + 1);
        p.dev_number_of_events = sp<const unsigned>(&dev_n, 1);
        p.dev_velo_bank_index = sp<const unsigned>(bank_index, Velo::Constants::n_modules * 4);
        p.dev_module_pair_cluster_num = sp<unsigned>(cluster_num, size_t(n) * 26);
        p.dev_velo_cluster_container = sp<char>(container, size_t(total_clusters) * Velo::Clusters::element_size);
        p.dev_velo_clusters = sp<Velo::Clusters>(clusters_views.data(), n);
        if (bank_version >= 0) {
          launch(n, [&] {
            velo_masked_clustering_kernel<V, MEP>(
              p, start, &geometry, sp_patterns.data(), sp_fx.data(), sp_fy.data());
          });
        }
      }

      // 6. velo_sort_by_phi (SortByPhi.cu:15-44)
      sorted = r->make<char>("dev_sorted_velo_cluster_container", size_t(total_clusters) * Velo::Clusters::element_size);
      unsigned* permutation = r->make<unsigned>("dev_hit_permutation", total_clusters);
      {
        velo_sort_by_phi::Parameters p {};
        p.host_number_of_events = sp<const unsigned>(&host_n, 1);
        p.host_total_number_of_velo_clusters = sp<const unsigned>(&total_clusters, 1);
        p.dev_event_list = sp<const mask_t>(event_list.data(), n);
        p.dev_offsets_estimated_input_size = sp<const unsigned>(offsets_est, size_t(n) * 26 + 1);
        p.dev_module_cluster_num = sp<const unsigned>(cluster_num, size_t(n) * 26);
        p.dev_velo_cluster_container = sp<const char>(container, size_t(total_clusters) * Velo::Clusters::element_size);
        p.dev_number_of_events = sp<const unsigned>(&dev_n, 1);
        p.dev_sorted_velo_cluster_container = sp<char>(sorted, size_t(total_clusters) * Velo::Clusters::element_size);
        p.dev_hit_permutation = sp<unsigned>(permutation, total_clusters);
        p.dev_velo_clusters = sp<const Velo::Clusters>(clusters_views.data(), n);
        launch(n, [&] { velo_sort_by_phi::velo_sort_by_phi(p); });
      }
    }

    // 7. velo_search_by_triplet (SearchByTriplet.cu:18-63)
    const unsigned track_container_size =
      total_clusters * Velo::Constants::max_number_of_tracks_per_cluster < n * Velo::Constants::minimum_container_size ?
        n * Velo::Constants::minimum_container_size :
        total_clusters * Velo::Constants::max_number_of_tracks_per_cluster;
    auto* tracks = r->make<Velo::TrackHits>("dev_tracks", track_container_size);
    auto* three_hit = r->make<Velo::TrackletHits>("dev_three_hit_tracks", track_container_size);
    auto* tracklets = r->make<Velo::TrackletHits>("dev_tracklets", size_t(n) * Velo::Constants::max_tracks_to_follow);
    auto* ttf = r->make<unsigned>("dev_tracks_to_follow", size_t(n) * Velo::Constants::max_tracks_to_follow);
    auto* hit_used = r->make<bool>("dev_hit_used", total_clusters);
    auto* atomics = r->make<unsigned>("dev_atomics_velo", size_t(n) * Velo::num_atomics);
    auto* n_tracks = r->make<unsigned>("dev_number_of_velo_tracks", n);
    auto* rel_indices = r->make<unsigned short>("dev_rel_indices", total_clusters);
    {
      velo_search_by_triplet::Parameters p {};
      p.host_number_of_events = sp<const unsigned>(&host_n, 1);
      p.host_total_number_of_velo_clusters = sp<const unsigned>(&total_clusters, 1);
      p.dev_event_list = sp<const mask_t>(event_list.data(), n);
      p.dev_number_of_events = sp<const unsigned>(&dev_n, 1);
      p.dev_sorted_velo_cluster_container =
        sp<const char>(sorted, size_t(total_clusters) * Velo::Clusters::element_size);
      p.dev_offsets_estimated_input_size = sp<const unsigned>(offsets_est, size_t(n) * 26 + 1);
      p.dev_module_cluster_num = sp<const unsigned>(cluster_num, size_t(n) * 26);
      p.dev_tracks = sp<Velo::TrackHits>(tracks, track_container_size);
      p.dev_tracklets = sp<Velo::TrackletHits>(tracklets, size_t(n) * Velo::Constants::max_tracks_to_follow);
      p.dev_tracks_to_follow = sp<unsigned>(ttf, size_t(n) * Velo::Constants::max_tracks_to_follow);
      p.dev_three_hit_tracks = sp<Velo::TrackletHits>(three_hit, track_container_size);
      p.dev_hit_used = sp<bool>(hit_used, total_clusters);
      p.dev_atomics_velo = sp<unsigned>(atomics, size_t(n) * Velo::num_atomics);
      p.dev_rel_indices = sp<unsigned short>(rel_indices, total_clusters);
      p.dev_number_of_velo_tracks = sp<unsigned>(n_tracks, n);
      p.dev_velo_clusters = sp<const Velo::Clusters>(clusters_views.data(), n);
      p.phi_tolerance = in.phi_tolerance;
      p.max_scatter = in.max_scatter;
      p.max_skipped_modules = in.max_skipped_modules;
      p.block_dim_x = 64u;
      launch(n, [&] { velo_search_by_triplet::velo_search_by_triplet(p, &geometry); });
    }

    // 8. prefix_sum_offsets_velo_tracks
    const unsigned n_four_hit = prefix_sum(*r, "dev_offsets_velo_tracks", n_tracks, n);
    const unsigned* offsets_tracks = static_cast<unsigned*>(r->buffers["dev_offsets_velo_tracks"].p);

    // 9. velo_three_hit_tracks_filter (ThreeHitTracksFilter.cu:9-42)
    auto* three_out = r->make<Velo::TrackletHits>("dev_three_hit_tracks_output", track_container_size);
    auto* n_three_out = r->make<unsigned>("dev_number_of_three_hit_tracks_output", n);
    {
      velo_three_hit_tracks_filter::Parameters p {};
      p.host_number_of_events = sp<const unsigned>(&host_n, 1);
      p.host_total_number_of_velo_clusters = sp<const unsigned>(&total_clusters, 1);
      p.dev_event_list = sp<const mask_t>(event_list.data(), n);
      p.dev_sorted_velo_cluster_container =
        sp<const char>(sorted, size_t(total_clusters) * Velo::Clusters::element_size);
      p.dev_offsets_estimated_input_size = sp<const unsigned>(offsets_est, size_t(n) * 26 + 1);
      p.dev_three_hit_tracks_input = sp<const Velo::TrackletHits>(three_hit, track_container_size);
      p.dev_atomics_velo = sp<const unsigned>(atomics, size_t(n) * Velo::num_atomics);
      p.dev_hit_used = sp<const bool>(hit_used, total_clusters);
      p.dev_number_of_events = sp<const unsigned>(&dev_n, 1);
      p.dev_three_hit_tracks_output = sp<Velo::TrackletHits>(three_out, track_container_size);
      p.dev_number_of_three_hit_tracks_output = sp<unsigned>(n_three_out, n);
      p.max_chi2 = in.max_chi2;
      p.max_weak_tracks = 500u;
      launch(n, [&] { velo_three_hit_tracks_filter::velo_three_hit_tracks_filter(p); });
    }

    // 10. prefix_sum_offsets_number_of_three_hit_tracks_filtered
    const unsigned n_three_filtered =
      prefix_sum(*r, "dev_offsets_number_of_three_hit_tracks_filtered", n_three_out, n);
    const unsigned* offsets_three = static_cast<unsigned*>(r->buffers["dev_offsets_number_of_three_hit_tracks_filtered"].p);

    // 11. velo_copy_track_hit_number (VeloCopyTrackHitNumber.cu:8-44)
    auto* hit_number = r->make<unsigned>("dev_velo_track_hit_number", n_four_hit + n_three_filtered);
    auto* offsets_all = r->make<unsigned>("dev_offsets_all_velo_tracks", n + 1);
    unsigned host_reconstructed = 0;
    {
      velo_copy_track_hit_number::Parameters p {};
      p.host_number_of_events = sp<const unsigned>(&host_n, 1);
      p.host_number_of_velo_tracks_at_least_four_hits = sp<const unsigned>(&n_four_hit, 1);
      p.host_number_of_three_hit_tracks_filtered = sp<const unsigned>(&n_three_filtered, 1);
      p.host_number_of_reconstructed_velo_tracks = sp<unsigned>(&host_reconstructed, 1);
      p.dev_offsets_estimated_input_size = sp<const unsigned>(offsets_est, size_t(n) * 26 + 1);
      p.dev_tracks = sp<const Velo::TrackHits>(tracks, track_container_size);
      p.dev_offsets_velo_tracks = sp<const unsigned>(offsets_tracks, n + 1);
      p.dev_offsets_number_of_three_hit_tracks_filtered = sp<const unsigned>(offsets_three, n + 1);
      p.dev_velo_track_hit_number = sp<unsigned>(hit_number, n_four_hit + n_three_filtered);
      p.dev_offsets_all_velo_tracks = sp<unsigned>(offsets_all, n + 1);
      launch(n, [&] { velo_copy_track_hit_number::velo_copy_track_hit_number(p); });
      host_reconstructed = offsets_all[n];
    }
    *r->make<unsigned>("host_number_of_reconstructed_velo_tracks", 1) = host_reconstructed;

    // 12. prefix_sum_offsets_velo_track_hit_number
    const unsigned total_track_hits =
      prefix_sum(*r, "dev_offsets_velo_track_hit_number", hit_number, n_four_hit + n_three_filtered);
    const unsigned* offsets_hit_number = static_cast<unsigned*>(r->buffers["dev_offsets_velo_track_hit_number"].p);

    // 13. velo_consolidate_tracks (VeloConsolidateTracks.cu:48-109): the kernel only;
    //     create_velo_views builds C++ view objects over the same buffers and is not run.
    const unsigned total_tracks = host_reconstructed + n_three_filtered;
    auto* accepted = r->make<bool>("dev_accepted_velo_tracks", total_tracks);
    std::fill(accepted, accepted + total_tracks, true);
    char* track_hits = r->make<char>("dev_velo_track_hits", size_t(total_track_hits) * Velo::Clusters::element_size);
    {
      std::vector<unsigned> histo(100, 0), counter(1, 0);
      velo_consolidate_tracks::Parameters p {};
      p.host_accumulated_number_of_hits_in_velo_tracks = sp<const unsigned>(&total_track_hits, 1);
      p.host_number_of_reconstructed_velo_tracks = sp<const unsigned>(&host_reconstructed, 1);
      p.host_number_of_three_hit_tracks_filtered = sp<const unsigned>(&n_three_filtered, 1);
      p.host_number_of_events = sp<const unsigned>(&host_n, 1);
      p.dev_event_list = sp<const mask_t>(event_list.data(), n);
      p.dev_offsets_all_velo_tracks = sp<const unsigned>(offsets_all, n + 1);
      p.dev_tracks = sp<const Velo::TrackHits>(tracks, track_container_size);
      p.dev_offsets_velo_track_hit_number = sp<const unsigned>(offsets_hit_number, total_tracks + 1);
      p.dev_sorted_velo_cluster_container =
        sp<const char>(sorted, size_t(total_clusters) * Velo::Clusters::element_size);
      p.dev_offsets_estimated_input_size = sp<const unsigned>(offsets_est, size_t(n) * 26 + 1);
      p.dev_three_hit_tracks_output = sp<const Velo::TrackletHits>(three_out, track_container_size);
      p.dev_offsets_number_of_three_hit_tracks_filtered = sp<const unsigned>(offsets_three, n + 1);
      p.dev_number_of_events = sp<const unsigned>(&dev_n, 1);
      p.dev_accepted_velo_tracks = sp<bool>(accepted, total_tracks);
      p.dev_velo_track_hits = sp<char>(track_hits, size_t(total_track_hits) * Velo::Clusters::element_size);
      launch(n, [&] {
        velo_consolidate_tracks::velo_consolidate_tracks(
          p, gsl::span<unsigned> {histo.data(), histo.size()}, gsl::span<unsigned> {counter.data(), 1});
      });

      // create_velo_views (VeloConsolidateTracks.cu:99): the views velo_kalman_filter reads
      ViewStorage<Allen::Views::Velo::Consolidated::Hits> hits_view(n);
      ViewStorage<Allen::Views::Velo::Consolidated::Track> track_view(host_reconstructed);
      ViewStorage<Allen::Views::Velo::Consolidated::Tracks> tracks_view(n);
      ViewStorage<Allen::Views::Velo::Consolidated::MultiEventTracks> multi_view(1);
      ViewStorage<Allen::IMultiEventContainer*> imec(1);
      p.dev_velo_hits_view = sp(hits_view.data(), n);
      p.dev_velo_track_view = sp(track_view.data(), host_reconstructed);
      p.dev_velo_tracks_view = sp(tracks_view.data(), n);
      p.dev_velo_multi_event_tracks_view = sp(multi_view.data(), 1);
      p.dev_imec_velo_tracks = sp(imec.data(), 1);
      launch(n, [&] { create_velo_views(p); });

      // 14. velo_kalman_filter (VeloKalmanFilter.cu:8-18 sizes, :153-268 operator(), :362-399 kernel)
      const unsigned reco = host_reconstructed;
      auto* is_backward = r->make<bool>("dev_is_backward", reco);
      char* beamline_states = r->make<char>("dev_velo_kalman_beamline_states", size_t(reco) * Velo::Consolidated::States::size);
      char* endvelo_states = r->make<char>("dev_velo_kalman_endvelo_states", size_t(reco) * Velo::Consolidated::States::size);
      ViewStorage<Allen::Views::Physics::KalmanStates> beam_view(n), end_view(n);
      float beamline[2] = {in.beamline_x, in.beamline_y};
      std::vector<unsigned> h_eta(40), h_phi(16), h_nhits(50), f_eta(40), f_phi(16), f_nhits(50), b_eta(40), b_phi(16),
        b_nhits(50);
      auto us = [](std::vector<unsigned>& v) { return gsl::span<unsigned> {v.data(), v.size()}; };
      velo_kalman_filter::Parameters k {};
      k.host_number_of_reconstructed_velo_tracks = sp<const unsigned>(&reco, 1);
      k.host_number_of_events = sp<const unsigned>(&host_n, 1);
      k.dev_event_list = sp<const mask_t>(event_list.data(), n);
      k.dev_number_of_events = sp<const unsigned>(&dev_n, 1);
      k.dev_offsets_all_velo_tracks = sp<const unsigned>(offsets_all, n + 1);
      k.dev_velo_tracks_view = sp<const Allen::Views::Velo::Consolidated::Tracks>(tracks_view.data(), n);
      k.dev_is_backward = sp<bool>(is_backward, reco);
      k.dev_velo_kalman_beamline_states = sp<char>(beamline_states, size_t(reco) * Velo::Consolidated::States::size);
      k.dev_velo_kalman_endvelo_states = sp<char>(endvelo_states, size_t(reco) * Velo::Consolidated::States::size);
      k.dev_velo_kalman_beamline_states_view = sp(beam_view.data(), n);
      k.dev_velo_kalman_endvelo_states_view = sp(end_view.data(), n);
      k.histogram_velo_track_eta_min = -10.f;
      k.histogram_velo_track_eta_max = 10.f;
      k.histogram_velo_track_eta_nbins = 40u;
      k.histogram_velo_track_phi_min = -4.f;
      k.histogram_velo_track_phi_max = 4.f;
      k.histogram_velo_track_phi_nbins = 16u;
      k.histogram_velo_track_nhits_min = 0.f;
      k.histogram_velo_track_nhits_max = 50.f;
      k.histogram_velo_track_nhits_nbins = 50u;
      launch(n, [&] {
        velo_kalman_filter::velo_kalman_filter(
          k, beamline, us(h_eta), us(h_phi), us(h_nhits), us(f_eta), us(f_phi), us(f_nhits), us(b_eta), us(b_phi),
          us(b_nhits));
      });
    }
    return r;
  }
} // namespace

extern "C" {

void* velo_ref_run(const VeloCpuInput* in)
{
  const bool mep = in->mep_layout != 0;
  switch (in->bank_version) {
  case 3: return mep ? run_chain<3, true>(*in) : run_chain<3, false>(*in);
  case 4: return mep ? run_chain<4, true>(*in) : run_chain<4, false>(*in);
  default: return mep ? run_chain<2, true>(*in) : run_chain<2, false>(*in);
  }
}

const void* velo_ref_get(void* handle, const char* name, size_t* nbytes)
{
  auto* r = static_cast<Result*>(handle);
  auto it = r->buffers.find(name);
  if (it == r->buffers.end()) {
    if (nbytes) *nbytes = 0;
    return nullptr;
  }
  if (nbytes) *nbytes = it->second.n;
  return it->second.p;
}

void velo_ref_free(void* handle) { delete static_cast<Result*>(handle); }

/*
 * CPU baseline timing: the chain over `n_slices` consecutive slices of
 * `slice_size` events starting at in->event_start, distributed round-robin over
 * `n_threads` host threads (one slice per thread at a time, as Allen's -t
 * streams do), cycling over the events available. Returns wall seconds for all slices.
 */
double velo_ref_time(const VeloCpuInput* in, unsigned slice_size, unsigned n_slices, unsigned n_threads)
{
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> workers;
  for (unsigned t = 0; t < n_threads; ++t) {
    workers.emplace_back([=] {
      // slices cycle over the events available, so a sample may be longer than the input
      const unsigned available = in->n_events / slice_size ? in->n_events / slice_size : 1;
      for (unsigned s = t; s < n_slices; s += n_threads) {
        VeloCpuInput slice = *in;
        slice.event_start = in->event_start + (s % available) * slice_size;
        slice.n_events = slice_size;
        velo_ref_free(velo_ref_run(&slice));
      }
    });
  }
  for (auto& w : workers)
    w.join();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
}
