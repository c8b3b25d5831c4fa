/*
 * velo_b200_chain_t: the Allen algorithm that runs the whole VELO super-pixel reconstruction
 * through libvelo_b200.so (include/velo_b200.h).  It is what a maintainer adds to the reference
 * tree (device/velo/b200/) to drop the B200 chain into an Allen sequence in place of
 * decode_velo + make_velo_tracks (configuration/python/AllenConf/velo_reconstruction.py:72-292):
 * the same inputs (data_provider_t's VP banks, host/data_provider/include/DataProvider.h:11-19),
 * the same outputs under the same argument names and layouts, views included, so that
 * velo_kalman_filter (velo_reconstruction.py:295-322) and every other consumer binds to them.
 *
 * Memory is Allen's: every buffer, the chain's scratch workspace included, is an argument that
 * the scheduler's arena holds (stream/store/include/MemoryManager.cuh), sized in
 * set_arguments_size() from the slice's bounds (two estimated clusters per super pixel, the
 * bank sizes give the super pixels) and reduced to the exact sizes in operator() once the host
 * scalars are known, as the reference's host prefix sums make them known.  The library
 * allocates only when a stream first uses the algorithm (its geometry, a few KB, and one ring of
 * tracks to follow per resident search CTA), never per slice.
 *
 * Errors follow Allen's convention (main/include/Common.h:19-33): a slice that does not fit
 * (too many events or clusters for the bounds, a device capacity flag) throws MemoryException,
 * which makes the caller split the slice; anything else throws StrException.
 */
#pragma once

#include <map>
#include <mutex>

#include "AlgorithmTypes.cuh"
#include "VeloConsolidated.cuh"
#include "velo_b200.h"

namespace velo_b200_chain {
  struct Parameters {
    HOST_INPUT(host_number_of_events_t, unsigned) host_number_of_events;
    HOST_INPUT(host_raw_bank_version_t, int) host_raw_bank_version;
    DEVICE_INPUT(dev_velo_raw_input_t, char) dev_velo_raw_input;
    DEVICE_INPUT(dev_velo_raw_input_offsets_t, unsigned) dev_velo_raw_input_offsets;
    DEVICE_INPUT(dev_velo_raw_input_sizes_t, unsigned) dev_velo_raw_input_sizes;
    DEVICE_INPUT(dev_velo_raw_input_types_t, unsigned) dev_velo_raw_input_types;
    // decode_velo's outputs (velo_reconstruction.py:153-164)
    HOST_OUTPUT(host_total_number_of_velo_clusters_t, unsigned) host_total_number_of_velo_clusters;
    DEVICE_OUTPUT(dev_offsets_estimated_input_size_t, unsigned) dev_offsets_estimated_input_size;
    DEVICE_OUTPUT(dev_module_cluster_num_t, unsigned) dev_module_cluster_num;
    DEVICE_OUTPUT(dev_sorted_velo_cluster_container_t, char) dev_sorted_velo_cluster_container;
    // make_velo_tracks' outputs (velo_reconstruction.py:269-292)
    HOST_OUTPUT(host_number_of_reconstructed_velo_tracks_t, unsigned) host_number_of_reconstructed_velo_tracks;
    HOST_OUTPUT(host_number_of_three_hit_tracks_filtered_t, unsigned) host_number_of_three_hit_tracks_filtered;
    HOST_OUTPUT(host_accumulated_number_of_hits_in_velo_tracks_t, unsigned)
    host_accumulated_number_of_hits_in_velo_tracks;
    DEVICE_OUTPUT(dev_offsets_all_velo_tracks_t, unsigned) dev_offsets_all_velo_tracks;
    DEVICE_OUTPUT(dev_velo_track_hit_number_t, unsigned) dev_velo_track_hit_number;
    DEVICE_OUTPUT(dev_offsets_velo_track_hit_number_t, unsigned) dev_offsets_velo_track_hit_number;
    DEVICE_OUTPUT(dev_velo_track_hits_t, char) dev_velo_track_hits;
    DEVICE_OUTPUT(dev_accepted_velo_tracks_t, bool) dev_accepted_velo_tracks;
    DEVICE_OUTPUT_WITH_DEPENDENCIES(
      dev_velo_hits_view_t,
      DEPENDENCIES(dev_velo_track_hits_t, dev_offsets_all_velo_tracks_t, dev_offsets_velo_track_hit_number_t),
      Allen::Views::Velo::Consolidated::Hits)
    dev_velo_hits_view;
    DEVICE_OUTPUT_WITH_DEPENDENCIES(
      dev_velo_track_view_t,
      DEPENDENCIES(dev_velo_hits_view_t),
      Allen::Views::Velo::Consolidated::Track)
    dev_velo_track_view;
    DEVICE_OUTPUT_WITH_DEPENDENCIES(
      dev_velo_tracks_view_t,
      DEPENDENCIES(dev_velo_track_view_t),
      Allen::Views::Velo::Consolidated::Tracks)
    dev_velo_tracks_view;
    DEVICE_OUTPUT_WITH_DEPENDENCIES(
      dev_velo_multi_event_tracks_view_t,
      DEPENDENCIES(dev_velo_tracks_view_t),
      Allen::Views::Velo::Consolidated::MultiEventTracks)
    dev_velo_multi_event_tracks_view;
    DEVICE_OUTPUT_WITH_DEPENDENCIES(
      dev_imec_velo_tracks_t,
      DEPENDENCIES(dev_velo_multi_event_tracks_view_t),
      Allen::IMultiEventContainer*)
    dev_imec_velo_tracks;
    // the chain's scratch (velo_chain_sizes().workspace_bytes) and its device status word
    DEVICE_OUTPUT(dev_velo_b200_workspace_t, char) dev_velo_b200_workspace;
    DEVICE_OUTPUT(dev_velo_b200_status_t, unsigned) dev_velo_b200_status;
    // the algorithm properties of velo_search_by_triplet and velo_three_hit_tracks_filter
    // (SearchByTriplet.cuh:129-131, ThreeHitTracksFilter.cuh:44)
    PROPERTY(phi_tolerance_t, "phi_tolerance", "tolerance of phi", float) phi_tolerance;
    PROPERTY(max_scatter_t, "max_scatter", "maximum scatter for seeding and forwarding", float) max_scatter;
    PROPERTY(max_skipped_modules_t, "max_skipped_modules", "skipped modules", unsigned) max_skipped_modules;
    PROPERTY(max_chi2_t, "max_chi2", "chi2 cut of the three-hit tracks", float) max_chi2;
  };

  struct velo_b200_chain_t : public DeviceAlgorithm, Parameters {
    void set_arguments_size(ArgumentReferences<Parameters> arguments, const RuntimeOptions&, const Constants&) const;

    void operator()(
      const ArgumentReferences<Parameters>& arguments,
      const RuntimeOptions& runtime_options,
      const Constants& constants,
      const Allen::Context& context) const;

    ~velo_b200_chain_t();

  private:
    // one chain per CUDA stream (operator() is const and re-entrant across streams)
    VeloChain* chain_for(cudaStream_t stream, const Constants& constants) const;
    mutable std::mutex m_mutex;
    mutable std::map<cudaStream_t, VeloChain*> m_chains;

    Property<phi_tolerance_t> m_tolerance {this, 0.045f};
    Property<max_scatter_t> m_max_scatter {this, 0.08f};
    Property<max_skipped_modules_t> m_max_skipped_modules {this, 1u};
    Property<max_chi2_t> m_max_chi2 {this, 20.f};
  };
} // namespace velo_b200_chain
