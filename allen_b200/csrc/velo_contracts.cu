// The reference's debug-build contracts on the VELO chain's outputs, checked on the device.
//
// The reference runs them after its algorithms in debug builds:
//  * cluster_container_checks (device/velo/search_by_triplet/src/SearchByTripletContracts.cu:6-81):
//    per module pair the sorted container is strictly increasing in (phi, id, x, y), and every
//    cluster has -100 < x < 100 and -100 < y < 100 (mm);
//  * track_container_checks (SearchByTripletContracts.cu:83-120): every track of dev_tracks has at
//    most 26 hits and no hit twice;
//  * lhcb_id_container_checks (device/velo/consolidate_tracks/src/VeloConsolidateTracks.cu:194-269):
//    every LHCb id of a consolidated track is non-zero and carries the VELO detector type in its
//    top four bits; the track and hit offsets never decrease and end at the run's totals.
// They are invariants rather than golden values, so they hold in learned mode too, whose tracks
// have no bit-exact oracle.  One CTA per event (grid-stride) for the containers, all threads
// over the consolidated ids; every read is bounded by the run's host totals, so outputs that
// break the contracts are counted, never followed out of their buffers.
#include <algorithm>
#include <string>

#include "velo_b200.h"
#include "velo_kernels.cuh"

namespace velo_host {
  void set_last_error(const std::string& what); // velo_chain.cu
}

namespace velo {

  struct ContractParams {
    unsigned n_events;
    unsigned clusters;        // T, host_total_number_of_velo_clusters
    unsigned tracks;          // host_number_of_reconstructed_velo_tracks
    unsigned track_hits;      // host_accumulated_number_of_hits_in_velo_tracks
    unsigned track_container; // entries of dev_tracks
    const unsigned* offsets_estimated_input_size;
    const unsigned* module_cluster_num;
    const char* sorted_container;
    const TrackHits* tracks_container;
    const unsigned* number_of_velo_tracks;
    const unsigned* offsets_all_velo_tracks;
    const unsigned* offsets_velo_track_hit_number;
    const char* velo_track_hits;
    unsigned* counts; // [VELO_CONTRACTS]
  };

  constexpr unsigned contract_threads = 256;
  constexpr uint32_t velo_id_type = 0x2;

  // (phi, id, x, y) of slot b strictly above that of slot a
  __device__ __forceinline__ bool increasing(const ClusterView& v, unsigned a, unsigned b)
  {
    const int16_t pa = v.phi(a), pb = v.phi(b);
    if (pb != pa) return pb > pa;
    const uint32_t ia = v.id(a), ib = v.id(b);
    if (ib != ia) return ib > ia;
    const float xa = v.x(a), xb = v.x(b);
    if (xb != xa) return xb > xa;
    return v.y(b) > v.y(a);
  }

  __global__ void __launch_bounds__(contract_threads) contracts_kernel(ContractParams p)
  {
    const ClusterView v {const_cast<char*>(p.sorted_container), p.clusters};
    unsigned outside = 0, unsorted = 0, too_long = 0, repeated = 0, zero = 0, not_velo = 0, offsets = 0;
    for (unsigned e = blockIdx.x; e < p.n_events; e += gridDim.x) {
      for (unsigned mp = 0; mp < n_module_pairs; ++mp) {
        const unsigned s0 = p.offsets_estimated_input_size[e * n_module_pairs + mp];
        unsigned num = p.module_cluster_num[e * n_module_pairs + mp];
        if (s0 > p.clusters || num > p.clusters - s0) {
          if (threadIdx.x == 0) ++outside; // a module pair beyond the container
          num = s0 > p.clusters ? 0u : p.clusters - s0;
        }
        for (unsigned k = threadIdx.x; k < num; k += blockDim.x) {
          const float x = v.x(s0 + k), y = v.y(s0 + k);
          if (!(x > -100.0f && x < 100.0f && y > -100.0f && y < 100.0f)) ++outside;
          if (k + 1 < num && !increasing(v, s0 + k, s0 + k + 1)) ++unsorted;
        }
      }
      const unsigned to = track_offset(p.offsets_estimated_input_size, e);
      const unsigned n = p.number_of_velo_tracks[e];
      const unsigned room = to < p.track_container ? p.track_container - to : 0u;
      if (n > room && threadIdx.x == 0) ++too_long; // tracks beyond the container
      for (unsigned t = threadIdx.x; t < min(n, room); t += blockDim.x) {
        const TrackHits& tr = p.tracks_container[to + t];
        if (tr.hits_num > max_track_size) ++too_long;
        const unsigned k = min(unsigned(tr.hits_num), max_track_size);
        bool twice = false;
        for (unsigned a = 1; a < k; ++a)
          for (unsigned b = 0; b < a; ++b)
            twice |= tr.hits[a] == tr.hits[b];
        repeated += twice ? 1u : 0u;
      }
    }
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (unsigned i = tid; i < p.n_events; i += stride)
      if (p.offsets_all_velo_tracks[i + 1] < p.offsets_all_velo_tracks[i]) ++offsets;
    for (unsigned i = tid; i < p.tracks; i += stride)
      if (p.offsets_velo_track_hit_number[i + 1] < p.offsets_velo_track_hit_number[i]) ++offsets;
    if (tid == 0) {
      if (p.offsets_all_velo_tracks[p.n_events] != p.tracks) ++offsets;
      if (p.offsets_velo_track_hit_number[p.tracks] != p.track_hits) ++offsets;
    }
    const uint32_t* ids = reinterpret_cast<const uint32_t*>(p.velo_track_hits);
    for (unsigned i = tid; i < p.track_hits; i += stride) {
      const uint32_t id = ids[i];
      if (id == 0) ++zero;
      if ((id >> 28) != velo_id_type) ++not_velo;
    }
    const unsigned mine[VELO_CONTRACTS] = {outside, unsorted, too_long, repeated, zero, not_velo, offsets};
#pragma unroll
    for (unsigned c = 0; c < VELO_CONTRACTS; ++c) {
      unsigned s = mine[c];
#pragma unroll
      for (unsigned o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
      if ((threadIdx.x & 31u) == 0 && s) atomicAdd(p.counts + c, s);
    }
  }

} // namespace velo

extern "C" VeloStatus velo_check_contracts(
  const VeloChainOutputs* outputs, const VeloChainTotals* totals, VeloStream stream, unsigned* dev_counts)
{
  if (!outputs || !totals || !dev_counts) {
    velo_host::set_last_error("velo_check_contracts: null argument");
    return VELO_ERR_ARGUMENT;
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(dev_counts, 0, VELO_CONTRACTS * sizeof(unsigned), s);
  if (e == cudaSuccess && totals->n_events > 0) {
    velo::ContractParams p {};
    p.n_events = totals->n_events;
    p.clusters = totals->host_total_number_of_velo_clusters;
    p.tracks = totals->host_number_of_reconstructed_velo_tracks;
    p.track_hits = totals->host_accumulated_number_of_hits_in_velo_tracks;
    p.track_container = totals->track_container_size;
    p.offsets_estimated_input_size = outputs->dev_offsets_estimated_input_size;
    p.module_cluster_num = outputs->dev_module_cluster_num;
    p.sorted_container = outputs->dev_sorted_velo_cluster_container;
    p.tracks_container = static_cast<const velo::TrackHits*>(outputs->dev_tracks);
    p.number_of_velo_tracks = outputs->dev_number_of_velo_tracks;
    p.offsets_all_velo_tracks = outputs->dev_offsets_all_velo_tracks;
    p.offsets_velo_track_hit_number = outputs->dev_offsets_velo_track_hit_number;
    p.velo_track_hits = outputs->dev_velo_track_hits;
    p.counts = dev_counts;
    if (!p.offsets_estimated_input_size || !p.module_cluster_num || !p.sorted_container || !p.tracks_container ||
        !p.number_of_velo_tracks || !p.offsets_all_velo_tracks || !p.offsets_velo_track_hit_number ||
        !p.velo_track_hits) {
      velo_host::set_last_error("velo_check_contracts: null output pointer");
      return VELO_ERR_ARGUMENT;
    }
    const unsigned grid = std::min(p.n_events, 2048u);
    velo::contracts_kernel<<<grid, velo::contract_threads, 0, s>>>(p);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    velo_host::set_last_error(std::string("velo_check_contracts: ") + cudaGetErrorString(e));
    return VELO_ERR_CUDA;
  }
  return VELO_OK;
}
