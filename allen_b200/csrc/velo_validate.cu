// On-device VELO track validation: efficiency, ghost and clone counts of the consolidated
// tracks against Monte Carlo truth, without copying tracks to the host.
//
// Restates the rules the reference's VELO validator applies on the host
// (host/validators/src/HostVeloValidator.cpp:9-30 -> checker/tracking/src/PrepareTracks.cpp
// -> TrackChecker.h:180-320, TrackCheckerCategories.h:28-30): a track is matched to the
// particle owning at least 70 % of its hits (m_minweight; ties go to the lower particle
// index), an unmatched track is a ghost, further tracks matched to a particle are clones,
// and the efficiency denominator is the particles flagged reconstructible.  A hit belongs to
// the particle owning the pixel of its LHCb id (the retina fraction bits 26-27 cleared).
//
// One CTA per event: one thread per track binary-searches each hit id in the event's sorted
// truth ids and votes; matched particles are counted in a caller scratch array; the CTA then
// adds the event's five counts to the slice totals.
#include <algorithm>
#include <string>

#include "velo_b200.h"
#include "velo_kernels.cuh"

namespace velo {

  struct ValidateParams {
    unsigned n_events;
    const unsigned* offsets_all_velo_tracks;       // [N + 1]
    const unsigned* offsets_velo_track_hit_number; // [tracks + 1]
    const char* velo_track_hits;                   // consolidated hits: ids first
    const unsigned* truth_offsets;                 // [N + 1]
    const unsigned* truth_ids;                     // per event sorted LHCb ids of truth pixels
    const unsigned* truth_owner;                   // particle index (within the event) per truth id
    const unsigned* particle_offsets;              // [N + 1]
    const uint8_t* particle_reconstructible;       // per particle
    unsigned* matched;                             // per particle: tracks matched (zeroed)
    unsigned long long* counts;                    // [5] tracks, ghosts, reconstructible, reconstructed, clones
  };

  constexpr unsigned validate_threads = 256;
  constexpr unsigned max_track_hits = 26;

  __global__ void __launch_bounds__(validate_threads) validate_kernel(ValidateParams p)
  {
    __shared__ unsigned warp_sums[33];
    const unsigned e = blockIdx.x;
    const unsigned total_tracks = p.offsets_all_velo_tracks[p.n_events];
    const unsigned total_hits = p.offsets_velo_track_hit_number[total_tracks];
    const unsigned* ids = reinterpret_cast<const unsigned*>(p.velo_track_hits);
    const unsigned t_begin = p.truth_offsets[e], t_end = p.truth_offsets[e + 1];
    const unsigned p_begin = p.particle_offsets[e], n_particles = p.particle_offsets[e + 1] - p_begin;
    const unsigned tr_begin = p.offsets_all_velo_tracks[e], tr_end = p.offsets_all_velo_tracks[e + 1];

    unsigned n_tracks = 0, n_ghosts = 0;
    for (unsigned t = tr_begin + threadIdx.x; t < tr_end; t += blockDim.x) {
      const unsigned h0 = p.offsets_velo_track_hit_number[t];
      const unsigned nh = min(p.offsets_velo_track_hit_number[t + 1] - h0, max_track_hits);
      unsigned owner[max_track_hits];
      unsigned n_owned = 0;
      for (unsigned h = 0; h < nh && h0 + h < total_hits; ++h) {
        const unsigned id = ids[h0 + h] & 0xF3FFFFFFu;
        unsigned lo = t_begin, hi = t_end; // first truth id >= id
        while (lo < hi) {
          const unsigned mid = (lo + hi) / 2;
          if (p.truth_ids[mid] < id) lo = mid + 1;
          else hi = mid;
        }
        if (lo < t_end && p.truth_ids[lo] == id) owner[n_owned++] = p.truth_owner[lo];
      }
      // most frequent owner, the lower index on ties
      unsigned best = 0xFFFFFFFFu, best_count = 0;
      for (unsigned i = 0; i < n_owned; ++i) {
        unsigned c = 0;
        for (unsigned j = 0; j < n_owned; ++j)
          c += owner[j] == owner[i];
        if (c > best_count || (c == best_count && owner[i] < best)) {
          best_count = c;
          best = owner[i];
        }
      }
      ++n_tracks;
      if (n_owned > 0 && best_count * 10 >= 7 * nh && best < n_particles) atomicAdd(p.matched + p_begin + best, 1u);
      else ++n_ghosts;
    }
    __syncthreads(); // matched counts of the event complete (same CTA)
    unsigned n_recoble = 0, n_reco = 0, n_clones = 0;
    for (unsigned i = threadIdx.x; i < n_particles; i += blockDim.x) {
      const unsigned m = p.matched[p_begin + i];
      if (p.particle_reconstructible[p_begin + i]) {
        ++n_recoble;
        if (m > 0) {
          ++n_reco;
          n_clones += m - 1;
        }
      }
    }
    const unsigned v[5] = {n_tracks, n_ghosts, n_recoble, n_reco, n_clones};
#pragma unroll
    for (unsigned k = 0; k < 5; ++k) {
      unsigned total;
      block_exclusive_scan(v[k], warp_sums, &total);
      if (threadIdx.x == 0 && total) atomicAdd(p.counts + k, static_cast<unsigned long long>(total));
    }
  }

} // namespace velo

namespace velo_host {
  void set_last_error(const std::string& what); // velo_chain.cu
}

extern "C" VeloStatus velo_validate_tracks(
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
  VeloStream stream)
{
  if (!dev_offsets_all_velo_tracks || !dev_offsets_velo_track_hit_number || !dev_velo_track_hits || !dev_truth_offsets ||
      !dev_truth_ids || !dev_truth_owner || !dev_particle_offsets || !dev_particle_reconstructible ||
      !dev_matched_scratch || !dev_counts) {
    velo_host::set_last_error("velo_validate_tracks: null argument");
    return VELO_ERR_ARGUMENT;
  }
  if (n_events == 0) return VELO_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(dev_matched_scratch, 0, sizeof(unsigned) * std::max(n_particles, 1u), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(dev_counts, 0, 5 * sizeof(unsigned long long), s);
  if (e == cudaSuccess) {
    velo::ValidateParams p {n_events,        dev_offsets_all_velo_tracks, dev_offsets_velo_track_hit_number,
                            dev_velo_track_hits, dev_truth_offsets,      dev_truth_ids,
                            dev_truth_owner, dev_particle_offsets,       dev_particle_reconstructible,
                            dev_matched_scratch, dev_counts};
    velo::validate_kernel<<<n_events, velo::validate_threads, 0, s>>>(p);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    velo_host::set_last_error(std::string("velo_validate_tracks: ") + cudaGetErrorString(e));
    return VELO_ERR_CUDA;
  }
  return VELO_OK;
}
