// The consolidated VELO track views (create_velo_views,
// device/velo/consolidate_tracks/src/VeloConsolidateTracks.cu:11-46): per event a Hits view and
// a Tracks view, per track a Track view, one MultiEventTracks view and the type-erased pointer to
// it (dev_imec_velo_tracks).  These are what every consumer of the VELO tracks binds to, e.g.
// velo_kalman_filter's dev_velo_tracks_view (configuration/python/AllenConf/velo_reconstruction.py:
// 295-307).  The structs of include/velo_b200.h have the reference types' layouts; each field is
// computed as the reference's constructors compute it (VeloConsolidated.cuh:68-80, 217-230,
// 278-281, MultiEventContainer.cuh:48-50).
#include <string>

#include <cuda_fp16.h>

#include "velo_b200.h"
#include "velo_kernels.cuh"

namespace velo_host {
  void set_last_error(const std::string& what);
}

namespace {
  static_assert(sizeof(VeloHitsView) == 24 && sizeof(VeloTrackView) == 24 && sizeof(VeloTracksView) == 16 &&
                  sizeof(VeloMultiEventTracksView) == 24,
                "view layouts of the reference (LP64)");
  constexpr int type_id_velo_tracks = 1; // Allen::TypeIDs::VeloTracks (backend/include/TypeID.h)

  __global__ void create_views_kernel(
    unsigned n_events,
    const char* track_hits,
    const unsigned* offsets_all,
    const unsigned* offsets_hit_number,
    VeloHitsView* hits_view,
    VeloTrackView* track_view,
    unsigned track_capacity,
    VeloTracksView* tracks_view,
    VeloMultiEventTracksView* multi_event_view,
    const void** imec,
    unsigned* status)
  {
    const unsigned e = blockIdx.x;
    const unsigned first = offsets_all[e], n_tracks = offsets_all[e + 1] - first;
    if (offsets_all[n_events] > track_capacity) {
      if (threadIdx.x == 0 && e == 0 && status != nullptr) velo::set_error(status, velo::err_output_capacity);
      return;
    }
    const unsigned* hn = offsets_hit_number + first; // the event's track-hit offsets
    for (unsigned t = threadIdx.x; t < n_tracks; t += blockDim.x) {
      VeloTrackView v;
      v.hits = hits_view + e;
      v.track_index = t;
      v.track_container_offset = first;
      v.offset = hn[t] - hn[0];
      v.number_of_hits = hn[t + 1] - hn[t];
      track_view[first + t] = v;
    }
    if (threadIdx.x == 0) {
      VeloHitsView h;
      h.base_pointer = track_hits;
      h.offset = offsets_hit_number[first];
      h.size = offsets_hit_number[offsets_all[e + 1]] - h.offset;
      h.total_number_of_hits = offsets_hit_number[offsets_all[n_events]];
      hits_view[e] = h;
      VeloTracksView ts;
      ts.track = track_view + first;
      ts.size = n_tracks;
      ts.offset = first;
      tracks_view[e] = ts;
      if (e == 0) {
        VeloMultiEventTracksView m;
        m.type_id = type_id_velo_tracks;
        m.container = tracks_view;
        m.number_of_events = n_events;
        *multi_event_view = m;
        *imec = multi_event_view;
      }
    }
  }
} // namespace

namespace velo {
  namespace {
    __device__ __forceinline__ void export_elements(const char* in, char* out, unsigned total, unsigned begin, unsigned stride)
    {
      const ClusterView v {const_cast<char*>(in), total};
      uint32_t* id = reinterpret_cast<uint32_t*>(out);
      __half* xyz = reinterpret_cast<__half*>(out + 4 * size_t(total));
      int16_t* phi = reinterpret_cast<int16_t*>(out + 10 * size_t(total));
      for (unsigned i = begin; i < total; i += stride) {
        id[i] = v.id(i);
        xyz[3 * size_t(i)] = __float2half_rn(v.x(i));
        xyz[3 * size_t(i) + 1] = __float2half_rn(v.y(i));
        xyz[3 * size_t(i) + 2] = __float2half_rn(v.z(i));
        phi[i] = v.phi(i);
      }
    }
  } // namespace

  // Grid-stride over the T clusters and the TH track hits of the slice (read on the device);
  // nothing is written when an earlier stage found the slice above its bounds.
  __global__ void export_half_kernel(HalfExportParams p)
  {
    const unsigned T = p.offsets_estimated_input_size[p.n_events * n_module_pairs];
    if (T > p.cluster_capacity) return; // flagged by the clustering kernel
    const unsigned begin = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    export_elements(p.sorted_container, p.sorted_half, T, begin, stride);
    const unsigned reco = p.offsets_all_velo_tracks[p.n_events];
    if (reco > p.track_capacity) return; // flagged by the consolidation
    const unsigned TH = p.offsets_velo_track_hit_number[reco];
    if (TH > p.track_hit_capacity) return;
    export_elements(p.velo_track_hits, p.track_hits_half, TH, begin, stride);
  }
} // namespace velo

extern "C" VeloStatus velo_create_velo_views(
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
  VeloStream stream)
{
  if (n_events == 0 || !dev_velo_track_hits || !dev_offsets_all_velo_tracks || !dev_offsets_velo_track_hit_number ||
      !dev_velo_hits_view || !dev_velo_track_view || !dev_velo_tracks_view || !dev_velo_multi_event_tracks_view ||
      !dev_imec_velo_tracks) {
    velo_host::set_last_error("velo_create_velo_views: null argument or no events");
    return VELO_ERR_ARGUMENT;
  }
  create_views_kernel<<<n_events, 256, 0, static_cast<cudaStream_t>(stream)>>>(
    n_events, dev_velo_track_hits, dev_offsets_all_velo_tracks, dev_offsets_velo_track_hit_number, dev_velo_hits_view,
    dev_velo_track_view, track_capacity, dev_velo_tracks_view, dev_velo_multi_event_tracks_view, dev_imec_velo_tracks,
    dev_status);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    velo_host::set_last_error(std::string("velo_create_velo_views: ") + cudaGetErrorString(e));
    return VELO_ERR_CUDA;
  }
  return VELO_OK;
}
