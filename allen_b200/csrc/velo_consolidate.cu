// velo_copy_track_hit_number + velo_consolidate_tracks on sm_100a, one event per CTA.
//
// Reference: device/velo/consolidate_tracks/src/VeloCopyTrackHitNumber.cu:49-78 and
// VeloConsolidateTracks.cu:120-192.  Per event: the >= 4 hit tracks (in track order),
// then the filtered three-hit tracks; every track's hits are gathered from the sorted
// container into the consolidated SoA (u32 id[TH] | f32 xyz[3 TH] | phi unused), at the
// offsets given by the scan of the per-track hit numbers.  The per-event track-hit
// totals come from the search kernel, so the global offsets need one device scan over
// events and a block scan inside the event, instead of the reference's host prefix sum
// over every track.
#include "velo_kernels.cuh"

namespace velo {

  __global__ void __launch_bounds__(consolidate_threads) consolidate_kernel(ConsolidateParams p)
  {
    __shared__ unsigned warp_sums[33];
    __shared__ uint16_t chunk_hits[consolidate_threads * max_track_size]; // hit indices of a chunk's tracks
    const unsigned e = blockIdx.x;
    const unsigned n = p.n_events;
    const unsigned to = track_offset(p.offsets_estimated_input_size, e);
    const unsigned n4 = p.offsets_velo_tracks[e + 1] - p.offsets_velo_tracks[e];
    const unsigned n3 = p.offsets_three_hit[e + 1] - p.offsets_three_hit[e];
    const unsigned total = n4 + n3;
    const unsigned g0 = p.offsets_velo_tracks[e] + p.offsets_three_hit[e];
    const unsigned hit_base = p.event_track_hit_base[e];
    const unsigned TH = p.event_track_hit_base[n];
    const unsigned T = p.offsets_estimated_input_size[n * n_module_pairs];
    const unsigned hit_offset = p.offsets_estimated_input_size[e * n_module_pairs];
    const unsigned all_tracks = p.offsets_velo_tracks[n] + p.offsets_three_hit[n];
    if (T > p.cluster_capacity) return; // flagged by the clustering kernel
    if (TH > p.track_hit_capacity) {
      if (threadIdx.x == 0) set_error(p.status, err_output_capacity);
      return;
    }

    if (threadIdx.x == 0) {
      p.offsets_all_velo_tracks[e + 1] = p.offsets_velo_tracks[e + 1] + p.offsets_three_hit[e + 1];
      if (e == 0) p.offsets_all_velo_tracks[0] = 0;
      if (e == n - 1) {
        if (all_tracks < p.track_capacity) p.offsets_velo_track_hit_number[all_tracks] = TH;
        if (all_tracks + 1 > p.track_capacity || TH > p.track_hit_capacity) set_error(p.status, err_output_capacity);
      }
    }
    // dev_accepted_velo_tracks is sized by the reference as reconstructed tracks (which
    // include the three-hit ones) plus the three-hit tracks again; all entries are 1.
    if (e == n - 1) {
      const unsigned accepted_size = all_tracks + p.offsets_three_hit[n];
      for (unsigned i = all_tracks + threadIdx.x; i < accepted_size && i < p.track_capacity; i += blockDim.x)
        p.accepted_velo_tracks[i] = true;
    }

    // Tracks in chunks of one per thread: a scan of the hit numbers places each track, its
    // thread writes the track's entries and its hit indices (event-relative, in output order)
    // to shared memory, then all threads gather the chunk's hits - one hit per thread, so the
    // gathers run in parallel and the writes to the consolidated SoA are contiguous.
    const ClusterView in {const_cast<char*>(p.sorted_container), T};
    const ClusterView out {p.velo_track_hits, TH};
    unsigned carry = 0;
    for (unsigned c0 = 0; c0 < total; c0 += blockDim.x) {
      const unsigned i = c0 + threadIdx.x;
      unsigned hn = 0;
      const uint16_t* hits = nullptr;
      if (i < n4 && to + i < p.track_container_capacity) {
        hn = p.tracks[to + i].hits_num;
        hits = p.tracks[to + i].hits;
      }
      else if (i >= n4 && i < total && to + i - n4 < p.track_container_capacity) {
        hn = 3;
        hits = p.three_hit_tracks_output[to + i - n4].hits;
      }
      else if (i < total) {
        set_error(p.status, err_track_capacity);
      }
      unsigned block_total;
      const unsigned excl = block_exclusive_scan(hn, warp_sums, &block_total);
      if (i < total) {
        const unsigned g = g0 + i;
        const unsigned pos = hit_base + carry + excl;
        if (g < p.track_capacity && pos + hn <= p.track_hit_capacity) {
          p.velo_track_hit_number[g] = hn;
          p.offsets_velo_track_hit_number[g] = pos;
          p.accepted_velo_tracks[g] = true;
        }
        else {
          set_error(p.status, err_output_capacity);
        }
        for (unsigned j = 0; j < hn; ++j)
          chunk_hits[excl + j] = hits[j];
      }
      __syncthreads();
      const unsigned pos0 = hit_base + carry;
      for (unsigned k = threadIdx.x; k < block_total; k += blockDim.x) {
        const unsigned hi = hit_offset + chunk_hits[k];
        if (pos0 + k >= p.track_hit_capacity || hi >= T) continue; // flagged: a track that did not fit
        out.x(pos0 + k) = in.x(hi);
        out.y(pos0 + k) = in.y(hi);
        out.z(pos0 + k) = in.z(hi);
        out.id(pos0 + k) = in.id(hi);
      }
      __syncthreads(); // chunk_hits is reused by the next chunk
      carry += block_total;
    }
  }

} // namespace velo
