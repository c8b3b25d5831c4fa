/*
 * velo_b200_chain_t (VeloB200Chain.cuh): Allen's algorithm interface
 * (stream/gear/include/Algorithm.cuh:319-461) over the C ABI of libvelo_b200.so.
 */
#include <cstring>
#include <string>
#include <vector>

#include "VeloB200Chain.cuh"
#include "ClusteringDefinitions.cuh"

INSTANTIATE_ALGORITHM(velo_b200_chain::velo_b200_chain_t)

namespace {
  static_assert(sizeof(VeloHitsView) == sizeof(Allen::Views::Velo::Consolidated::Hits));
  static_assert(sizeof(VeloTrackView) == sizeof(Allen::Views::Velo::Consolidated::Track));
  static_assert(sizeof(VeloTracksView) == sizeof(Allen::Views::Velo::Consolidated::Tracks));
  static_assert(sizeof(VeloMultiEventTracksView) == sizeof(Allen::Views::Velo::Consolidated::MultiEventTracks));
  // the coordinate layout of this build's Velo::Clusters_t: float (CPU build) or half (CUDA build)
  constexpr int coordinate_layout = sizeof(half_t) == 2 ? VELO_COORDINATES_FP16 : VELO_COORDINATES_FP32;
  static_assert(Velo::Clusters::element_size == (sizeof(half_t) == 2 ? 12 : 18));

  // status bits of the library's kernels that mean "the slice is larger than its bounds"
  constexpr unsigned capacity_flags = (1u << 0) | (1u << 1) | (1u << 2) | (1u << 5) | (1u << 6) | (1u << 7);

  [[noreturn]] void raise(VeloStatus status, const char* what)
  {
    const std::string message = std::string("velo_b200_chain: ") + what + ": " + velo_last_error_string();
    if (status == VELO_ERR_CAPACITY) throw MemoryException(message);
    throw StrException(message);
  }

  // The super pixels of a slice are bounded by its raw words (one 32-bit word per super pixel).
  unsigned long long super_pixel_bound(size_t raw_bytes) { return raw_bytes / 4 + 1; }

  // velo_geometry.bin back from the device geometry that Allen's VPGeometry consumer uploaded
  // (integration/non_event_data/src/VPGeometry.cpp:58-67): the layout VeloGeometry(std::vector<char>)
  // reads (ClusteringDefinitions.cuh:164-197), so that the library parses the same numbers.
  std::vector<char> geometry_blob(const VeloGeometry* dev_geometry)
  {
    std::vector<char> raw(sizeof(VeloGeometry));
    Allen::memcpy(raw.data(), dev_geometry, sizeof(VeloGeometry), Allen::memcpyDeviceToHost);
    const auto& g = *reinterpret_cast<const VeloGeometry*>(raw.data());
    std::vector<char> blob;
    auto put_count = [&](size_t n) { blob.insert(blob.end(), reinterpret_cast<const char*>(&n), reinterpret_cast<const char*>(&n) + sizeof(n)); };
    auto put_floats = [&](const float* f, size_t n) {
      blob.insert(blob.end(), reinterpret_cast<const char*>(f), reinterpret_cast<const char*>(f + n));
    };
    put_count(Velo::Constants::n_modules);
    put_floats(g.module_zs, Velo::Constants::n_modules);
    put_count(Velo::Constants::number_of_sensor_columns);
    put_floats(g.local_x, Velo::Constants::number_of_sensor_columns);
    put_count(Velo::Constants::number_of_sensor_columns);
    put_floats(g.x_pitch, Velo::Constants::number_of_sensor_columns);
    put_count(Velo::Constants::n_sensors);
    put_count(12);
    put_floats(g.ltg, 12 * Velo::Constants::n_sensors);
    return blob;
  }
} // namespace

VeloChain* velo_b200_chain::velo_b200_chain_t::chain_for(cudaStream_t stream, const Constants& constants) const
{
  std::lock_guard<std::mutex> lock(m_mutex);
  auto it = m_chains.find(stream);
  if (it != m_chains.end()) return it->second;
  if (constants.dev_velo_geometry == nullptr) throw StrException("velo_b200_chain: no VELO geometry in Constants");
  const std::vector<char> blob = geometry_blob(constants.dev_velo_geometry);
  const VeloChainProperties props {property<phi_tolerance_t>(), property<max_scatter_t>(),
                                   property<max_skipped_modules_t>(), property<max_chi2_t>()};
  VeloChain* chain = nullptr;
  const VeloStatus st = velo_chain_create(blob.data(), blob.size(), &props, &chain);
  if (st != VELO_OK) raise(st, "velo_chain_create");
  m_chains.emplace(stream, chain);
  return chain;
}

velo_b200_chain::velo_b200_chain_t::~velo_b200_chain_t()
{
  for (auto& kv : m_chains)
    velo_chain_destroy(kv.second);
}

void velo_b200_chain::velo_b200_chain_t::set_arguments_size(
  ArgumentReferences<Parameters> arguments,
  const RuntimeOptions&,
  const Constants&) const
{
  const unsigned n = first<host_number_of_events_t>(arguments);
  VeloChainSizes s {};
  const VeloStatus st =
    velo_chain_sizes(nullptr, n > 0 ? n : 1, super_pixel_bound(size<dev_velo_raw_input_t>(arguments)), coordinate_layout, &s);
  if (st != VELO_OK) raise(st, "velo_chain_sizes");
  set_size<host_total_number_of_velo_clusters_t>(arguments, 1);
  set_size<dev_offsets_estimated_input_size_t>(arguments, s.offsets_estimated_input_size);
  set_size<dev_module_cluster_num_t>(arguments, s.module_cluster_num);
  set_size<dev_sorted_velo_cluster_container_t>(arguments, s.sorted_velo_cluster_container_bytes);
  set_size<host_number_of_reconstructed_velo_tracks_t>(arguments, 1);
  set_size<host_number_of_three_hit_tracks_filtered_t>(arguments, 1);
  set_size<host_accumulated_number_of_hits_in_velo_tracks_t>(arguments, 1);
  set_size<dev_offsets_all_velo_tracks_t>(arguments, s.offsets_all_velo_tracks);
  set_size<dev_velo_track_hit_number_t>(arguments, s.velo_track_hit_number);
  set_size<dev_offsets_velo_track_hit_number_t>(arguments, s.offsets_velo_track_hit_number);
  set_size<dev_velo_track_hits_t>(arguments, s.velo_track_hits_bytes);
  set_size<dev_accepted_velo_tracks_t>(arguments, s.accepted_velo_tracks);
  set_size<dev_velo_hits_view_t>(arguments, n);
  set_size<dev_velo_track_view_t>(arguments, s.max_reconstructed_tracks);
  set_size<dev_velo_tracks_view_t>(arguments, n);
  set_size<dev_velo_multi_event_tracks_view_t>(arguments, 1);
  set_size<dev_imec_velo_tracks_t>(arguments, 1);
  set_size<dev_velo_b200_workspace_t>(arguments, s.workspace_bytes);
  set_size<dev_velo_b200_status_t>(arguments, 1);
}

void velo_b200_chain::velo_b200_chain_t::operator()(
  const ArgumentReferences<Parameters>& arguments,
  const RuntimeOptions& runtime_options,
  const Constants& constants,
  const Allen::Context& context) const
{
  const unsigned n = first<host_number_of_events_t>(arguments);
  if (n == 0) return;
  const cudaStream_t stream = context.stream();
  VeloChain* chain = chain_for(stream, constants);

  // the arena's buffers become the chain's workspace and outputs (no allocation, no copies)
  const VeloChainOutputBuffers outputs {data<dev_offsets_estimated_input_size_t>(arguments),
                                        data<dev_module_cluster_num_t>(arguments),
                                        data<dev_sorted_velo_cluster_container_t>(arguments),
                                        data<dev_offsets_all_velo_tracks_t>(arguments),
                                        data<dev_velo_track_hit_number_t>(arguments),
                                        data<dev_offsets_velo_track_hit_number_t>(arguments),
                                        data<dev_velo_track_hits_t>(arguments),
                                        reinterpret_cast<uint8_t*>(data<dev_accepted_velo_tracks_t>(arguments))};
  VeloStatus st = velo_chain_bind(
    chain,
    data<dev_velo_b200_workspace_t>(arguments),
    size<dev_velo_b200_workspace_t>(arguments),
    n,
    super_pixel_bound(size<dev_velo_raw_input_t>(arguments)),
    coordinate_layout,
    &outputs);
  if (st != VELO_OK) raise(st, "velo_chain_bind");

  const VeloDeviceSlice slice {data<dev_velo_raw_input_t>(arguments),
                               data<dev_velo_raw_input_offsets_t>(arguments),
                               data<dev_velo_raw_input_sizes_t>(arguments),
                               data<dev_velo_raw_input_types_t>(arguments),
                               std::get<0>(runtime_options.event_interval),
                               n,
                               first<host_raw_bank_version_t>(arguments),
                               runtime_options.mep_layout ? 1 : 0};
  st = velo_chain_run(chain, &slice, stream, 0);
  if (st != VELO_OK) raise(st, "velo_chain_run");

  // the host scalars (the reference's host prefix sums drain the stream the same way)
  VeloChainTotals t {};
  st = velo_chain_synchronize(chain, &t);
  if (st == VELO_ERR_DEVICE_FLAGS && (t.device_flags & capacity_flags)) raise(VELO_ERR_CAPACITY, "velo_chain_run");
  if (st != VELO_OK) raise(st, "velo_chain_run");
  data<host_total_number_of_velo_clusters_t>(arguments)[0] = t.host_total_number_of_velo_clusters;
  data<host_number_of_reconstructed_velo_tracks_t>(arguments)[0] = t.host_number_of_reconstructed_velo_tracks;
  data<host_number_of_three_hit_tracks_filtered_t>(arguments)[0] = t.host_number_of_three_hit_tracks_filtered;
  data<host_accumulated_number_of_hits_in_velo_tracks_t>(arguments)[0] = t.host_accumulated_number_of_hits_in_velo_tracks;

  // the views of velo_consolidate_tracks (VeloConsolidateTracks.cu:11-46, 99)
  Allen::memset_async(data<dev_velo_b200_status_t>(arguments), 0, sizeof(unsigned), context);
  st = velo_create_velo_views(
    n,
    data<dev_velo_track_hits_t>(arguments),
    data<dev_offsets_all_velo_tracks_t>(arguments),
    data<dev_offsets_velo_track_hit_number_t>(arguments),
    reinterpret_cast<VeloHitsView*>(data<dev_velo_hits_view_t>(arguments)),
    reinterpret_cast<VeloTrackView*>(data<dev_velo_track_view_t>(arguments)),
    static_cast<unsigned>(size<dev_velo_track_view_t>(arguments)),
    reinterpret_cast<VeloTracksView*>(data<dev_velo_tracks_view_t>(arguments)),
    reinterpret_cast<VeloMultiEventTracksView*>(data<dev_velo_multi_event_tracks_view_t>(arguments)),
    const_cast<const void**>(reinterpret_cast<void**>(data<dev_imec_velo_tracks_t>(arguments))),
    data<dev_velo_b200_status_t>(arguments),
    stream);
  if (st != VELO_OK) raise(st, "velo_create_velo_views");

  // exact sizes, as the reference's set_arguments_size gives them from the host scalars
  const unsigned reco = t.host_number_of_reconstructed_velo_tracks;
  reduce_size<dev_sorted_velo_cluster_container_t>(
    arguments, size_t(t.host_total_number_of_velo_clusters) * Velo::Clusters::element_size);
  reduce_size<dev_velo_track_hit_number_t>(arguments, reco);
  reduce_size<dev_offsets_velo_track_hit_number_t>(arguments, reco + 1);
  reduce_size<dev_velo_track_hits_t>(
    arguments, size_t(t.host_accumulated_number_of_hits_in_velo_tracks) * Velo::Clusters::element_size);
  reduce_size<dev_accepted_velo_tracks_t>(arguments, reco + t.host_number_of_three_hit_tracks_filtered);
  reduce_size<dev_velo_track_view_t>(arguments, reco);
}
