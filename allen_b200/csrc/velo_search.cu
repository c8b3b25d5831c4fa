// search_by_triplet (seeding + forwarding) and the three-hit filter on sm_100a,
// one event per CTA.
//
// Reference: device/velo/search_by_triplet/src/SearchByTriplet.cu:110-609 (kernel,
// find_forward_candidate, track_seeding, track_forwarding) and
// ThreeHitTracksFilter.cu:48-169.
//
// Design.  The event's sorted hits (id, x, y, z, phi) and the hit_used flags are staged
// in shared memory, together with the 2048-entry ring of tracks to follow and the
// tracklets, so the 24 barrier-separated steps run out of shared memory.  Within a step
// every seed candidate (h1) and every track to follow is independent: seeding only reads
// hit_used, forwarding only writes it, and each track to follow owns its track.  So each
// step runs one thread per item and then assigns output slots (ring entries, track numbers,
// three-hit entries) with a block-wide ordered scan, in item order.  That is the order the
// reference's sequential execution produces, so the track containers come out
// bit-identical to the reference CPU build, not merely equal as sets.
#include "velo_kernels.cuh"

namespace velo {

  constexpr unsigned seed_bit = 0x80000000u;
  constexpr unsigned track_number_mask = 0x0FFFFFFFu;
  constexpr unsigned skipped_mask = 0x70000000u;

  struct ModulePair {
    unsigned hit_start;
    unsigned hit_num;
    float z[2];
  };

  struct SearchShared {
    ModulePair md[3];
    unsigned warp_sums[33];
    unsigned ttf_counter; // atomics::tracks_to_follow
    unsigned n_three;     // atomics::number_of_three_hit_tracks
    unsigned local_hits;  // atomics::local_number_of_hits
    unsigned n_tracks;
    unsigned track_hits; // sum of hitsNum over the >= 4 hit tracks
    unsigned ttf[max_tracks_to_follow];
    TrackletHits tracklets[max_tracks_to_follow];
  };

  // Hits of one event: a cluster view with an index offset (0 in shared memory,
  // the event's hit offset in the global container).
  struct Hits {
    ClusterView v;
    unsigned offset;
    __device__ __forceinline__ float x(unsigned i) const { return v.x(offset + i); }
    __device__ __forceinline__ float y(unsigned i) const { return v.y(offset + i); }
    __device__ __forceinline__ float z(unsigned i) const { return v.z(offset + i); }
    __device__ __forceinline__ uint32_t id(unsigned i) const { return v.id(offset + i); }
    __device__ __forceinline__ int16_t phi(unsigned i) const { return v.phi(offset + i); }
    __device__ __forceinline__ const int16_t* phis() const { return v.phi_begin() + offset; }
  };

  struct Forward {
    int16_t candidate;
    int16_t phi;
  };

  // SearchByTriplet.cu:272-292
  __device__ __forceinline__ Forward find_forward_candidate(
    const Constants& k, const ModulePair& mp, const int16_t* phis, float h0x, float h0y, float tx, float ty, float dz)
  {
    const float predx = tx * dz;
    const float predy = ty * dz;
    const float xp = h0x + predx;
    const float yp = h0y + predy;
    Forward f;
    f.phi = hit_phi_16(k, xp, yp);
    f.candidate = static_cast<int16_t>(binary_search_leftmost(
      phis + mp.hit_start, mp.hit_num, static_cast<int16_t>(f.phi - static_cast<int16_t>(k.phi_tolerance_i16))));
    return f;
  }

  __device__ __forceinline__ bool phi_outside(int16_t phi, int16_t extrapolated, int16_t tol)
  {
    const int16_t diff = static_cast<int16_t>(phi - extrapolated);
    const int16_t abs_diff = static_cast<int16_t>(diff < 0 ? -diff : diff);
    return abs_diff > tol;
  }

  // One seed candidate h1 (SearchByTriplet.cu:325-445); returns true with the best
  // (h0, h2) when a triplet below max_scatter exists.
  __device__ __forceinline__ bool seed_one(
    const Constants& k,
    const Hits& h,
    const uint8_t* used,
    const ModulePair& prev,
    const ModulePair& next,
    unsigned h1,
    unsigned n_candidates,
    uint16_t& best_h0,
    uint16_t& best_h2)
  {
    const int16_t tol = static_cast<int16_t>(k.phi_tolerance_i16);
    float best_fit = k.max_scatter;
    best_h0 = 0;
    best_h2 = 0;
    const float h1x = h.x(h1), h1y = h.y(h1), h1z = h.z(h1);
    const int16_t h1_phi = h.phi(h1);
    const int16_t* phis = h.phis();
    int phi_index = binary_search_leftmost(phis + prev.hit_start, prev.hit_num, h1_phi);
    const float dz_next = next.z[0] - prev.z[0];
    unsigned found = 0;
    for (unsigned i = 0; i < prev.hit_num && found < n_candidates; ++i) {
      const int diff = (i & 1u) ? static_cast<int>(i) : -static_cast<int>(i);
      phi_index += diff;
      const unsigned in_bounds =
        phi_index < 0 ? static_cast<unsigned>(phi_index) + prev.hit_num :
                        (phi_index >= static_cast<int>(prev.hit_num) ?
                           static_cast<unsigned>(phi_index - static_cast<int>(prev.hit_num)) :
                           static_cast<unsigned>(phi_index));
      const unsigned h0 = prev.hit_start + in_bounds;
      if (used[h0]) continue;
      ++found;
      // the reference collects the candidates first and then visits them in the same order
      const float h0x = h.x(h0), h0y = h.y(h0), h0z = h.z(h0);
      const float td = __fdiv_rn(1.0f, h1z - h0z);
      const float txn = h1x - h0x;
      const float tyn = h1y - h0y;
      const float tx = txn * td;
      const float ty = tyn * td;
      const Forward f = find_forward_candidate(k, next, phis, h0x, h0y, tx, ty, dz_next);
      for (unsigned j = 0; j < next.hit_num; ++j) {
        const unsigned ib = (static_cast<unsigned>(static_cast<int>(f.candidate)) + j) % next.hit_num;
        const unsigned h2 = next.hit_start + ib;
        if (phi_outside(h.phi(h2), f.phi, tol)) break;
        if (used[h2]) continue;
        const float dz = h.z(h2) - h0z;
        const float predx = h0x + tx * dz;
        const float predy = h0y + ty * dz;
        const float dx = predx - h.x(h2);
        const float dy = predy - h.y(h2);
        const float scatter = dx * dx + dy * dy;
        if (scatter < best_fit) {
          best_fit = scatter;
          best_h0 = static_cast<uint16_t>(h0);
          best_h2 = static_cast<uint16_t>(h2);
        }
      }
    }
    return best_fit < k.max_scatter;
  }

  // Seeding over the current module pair (SearchByTriplet.cu:298-446).
  __device__ void seeding(SearchShared& s, const Constants& k, const Hits& h, const uint8_t* used, unsigned n_candidates)
  {
    const ModulePair prev = s.md[0], cur = s.md[1], next = s.md[2];
    for (unsigned c0 = 0; c0 < cur.hit_num; c0 += blockDim.x) {
      const unsigned r = c0 + threadIdx.x;
      bool ok = false;
      unsigned unused = 0;
      uint16_t bh0 = 0, bh2 = 0;
      const unsigned h1 = cur.hit_start + r;
      if (r < cur.hit_num && !used[h1]) {
        unused = 1;
        ok = seed_one(k, h, used, prev, next, h1, n_candidates, bh0, bh2);
      }
      unsigned total;
      const unsigned excl = block_exclusive_scan((ok ? 1u : 0u) | (unused << 16), s.warp_sums, &total);
      if (ok) {
        const unsigned tn = (s.ttf_counter + (excl & 0xFFFFu)) % max_tracks_to_follow;
        s.tracklets[tn].hits[0] = bh0;
        s.tracklets[tn].hits[1] = static_cast<uint16_t>(h1);
        s.tracklets[tn].hits[2] = bh2;
        s.ttf[tn] = seed_bit | tn;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        s.ttf_counter += total & 0xFFFFu;
        s.local_hits += total >> 16;
      }
      __syncthreads();
    }
  }

  // Forwarding of the tracks to follow (SearchByTriplet.cu:451-609).
  __device__ void forwarding(
    SearchShared& s,
    const Constants& k,
    const Hits& h,
    uint8_t* used,
    unsigned prev_ttf,
    unsigned diff_ttf,
    TrackHits* tracks,
    unsigned track_limit,
    TrackletHits* three_hit,
    unsigned three_limit,
    unsigned* status)
  {
    const ModulePair next = s.md[2];
    const int16_t tol = static_cast<int16_t>(k.phi_tolerance_i16);
    const int16_t* phis = h.phis();
    for (unsigned c0 = 0; c0 < diff_ttf; c0 += blockDim.x) {
      const unsigned kk = c0 + threadIdx.x;
      const bool active = kk < diff_ttf;
      unsigned full = 0, nh = 0, tn = 0;
      bool is_seed = false, found = false;
      int best_h2 = -1;
      uint16_t t0 = 0, t1 = 0, t2 = 0;
      if (active) {
        full = s.ttf[(prev_ttf + kk) % max_tracks_to_follow];
        is_seed = (full & seed_bit) == seed_bit;
        tn = full & track_number_mask;
        uint16_t h0n, h1n;
        if (is_seed) {
          const TrackletHits t = s.tracklets[tn];
          t0 = t.hits[0];
          t1 = t.hits[1];
          t2 = t.hits[2];
          nh = 3;
          h0n = t1;
          h1n = t2;
        }
        else if (tn < track_limit) {
          nh = tracks[tn].hits_num;
          if (nh < 2 || nh > max_track_size) nh = 2; // unreachable with consistent containers
          h0n = tracks[tn].hits[nh - 2];
          h1n = tracks[tn].hits[nh - 1];
        }
        else {
          // a track that did not fit its container (flagged when it was created)
          nh = 3;
          h0n = 0;
          h1n = 0;
        }
        const float h0x = h.x(h0n), h0y = h.y(h0n), h0z = h.z(h0n);
        const unsigned h0_module = ((h.id(h0n) & 0x3FC0000u) >> 18) / 4;
        const float h1x = h.x(h1n), h1y = h.y(h1n), h1z = h.z(h1n);
        const float td = __fdiv_rn(1.0f, h1z - h0z);
        const float txn = h1x - h0x;
        const float tyn = h1y - h0y;
        const float tx = txn * td;
        const float ty = tyn * td;
        float best_fit = k.max_scatter;
        const Forward f = find_forward_candidate(k, next, phis, h0x, h0y, tx, ty, next.z[h0_module % 2] - h0z);
        for (unsigned j = 0; j < next.hit_num; ++j) {
          const unsigned ib = (static_cast<unsigned>(static_cast<int>(f.candidate)) + j) % next.hit_num;
          const unsigned h2 = next.hit_start + ib;
          if (phi_outside(h.phi(h2), f.phi, tol)) break;
          const float dz = h.z(h2) - h0z;
          const float predx = h0x + tx * dz;
          const float predy = h0y + ty * dz;
          const float dx = predx - h.x(h2);
          const float dy = predy - h.y(h2);
          const float scatter = dx * dx + dy * dy;
          if (scatter < best_fit) {
            best_fit = scatter;
            best_h2 = static_cast<int>(h2);
          }
        }
        found = best_h2 != -1;
      }
      const unsigned skipped = (full & skipped_mask) >> 28;
      const bool new_track = active && found && is_seed;
      const bool enqueue =
        active && ((found && nh + 1 < max_track_size) || (!found && skipped < k.max_skipped_modules));
      const bool three = active && !found && !(skipped < k.max_skipped_modules) && nh == 3;
      unsigned total;
      const unsigned excl = block_exclusive_scan(
        (new_track ? 1u : 0u) | ((enqueue ? 1u : 0u) << 10) | ((three ? 1u : 0u) << 20), s.warp_sums, &total);
      if (active) {
        unsigned track_number = tn;
        if (found) {
          used[best_h2] = 1;
          if (is_seed) {
            used[t0] = 1;
            used[t1] = 1;
            used[t2] = 1;
            track_number = s.n_tracks + (excl & 0x3FFu);
            if (track_number < track_limit) {
              TrackHits& t = tracks[track_number];
              t.hits[0] = t0;
              t.hits[1] = t1;
              t.hits[2] = t2;
              t.hits[3] = static_cast<uint16_t>(best_h2);
              t.hits_num = 4;
            }
            else {
              set_error(status, err_track_capacity);
            }
          }
          else if (tn < track_limit) {
            tracks[tn].hits[nh] = static_cast<uint16_t>(best_h2);
            tracks[tn].hits_num = static_cast<uint8_t>(nh + 1);
          }
          atomicAdd(&s.track_hits, is_seed ? 4u : 1u);
        }
        if (enqueue) {
          const unsigned value =
            found ? track_number : (((skipped + 1) << 28) | (full & (seed_bit | track_number_mask)));
          s.ttf[(s.ttf_counter + ((excl >> 10) & 0x3FFu)) % max_tracks_to_follow] = value;
        }
        if (three) {
          const unsigned slot = s.n_three + ((excl >> 20) & 0x3FFu);
          if (slot < three_limit) three_hit[slot] = TrackletHits {{t0, t1, t2}};
          else set_error(status, err_track_capacity);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        s.n_tracks += total & 0x3FFu;
        s.ttf_counter += (total >> 10) & 0x3FFu;
        s.n_three += (total >> 20) & 0x3FFu;
      }
      __syncthreads();
    }
  }

  // ThreeHitTracksFilter.cu:48-107
  __device__ __forceinline__ float means_square_fit_chi2(const Hits& h, const TrackletHits& t)
  {
    const float w = 6400.f;
    float s0, sx, sz, sxz, sz2, u0, uy, uz, uyz, uz2;
    s0 = sx = sz = sxz = sz2 = 0.0f;
    u0 = uy = uz = uyz = uz2 = 0.0f;
#pragma unroll
    for (unsigned i = 0; i < 3; ++i) {
      const unsigned hn = t.hits[i];
      const float x = h.x(hn), y = h.y(hn), z = h.z(hn);
      const float wx_t_x = w * x, wx_t_z = w * z;
      s0 += w;
      sx += wx_t_x;
      sz += wx_t_z;
      sxz += wx_t_x * z;
      sz2 += wx_t_z * z;
      const float wy_t_y = w * y, wy_t_z = w * z;
      u0 += w;
      uy += wy_t_y;
      uz += wy_t_z;
      uyz += wy_t_y * z;
      uz2 += wy_t_z * z;
    }
    const float dens = __fdiv_rn(1.0f, sz2 * s0 - sz * sz);
    const float state_tx = (sxz * s0 - sx * sz) * dens;
    const float state_x = (sx * sz2 - sxz * sz) * dens;
    const float denu = __fdiv_rn(1.0f, uz2 * u0 - uz * uz);
    const float state_ty = (uyz * u0 - uy * uz) * denu;
    const float state_y = (uy * uz2 - uyz * uz) * denu;
    float chi2 = 0.0f;
#pragma unroll
    for (unsigned i = 0; i < 3; ++i) {
      const unsigned hn = t.hits[i];
      const float z = h.z(hn);
      const float x = state_x + state_tx * z;
      const float y = state_y + state_ty * z;
      const float dx = x - h.x(hn);
      const float dy = y - h.y(hn);
      chi2 += dx * dx * w + dy * dy * w;
    }
    return chi2 * 0.5f;
  }

  __device__ __forceinline__ void load_module_pairs(
    SearchShared& s, const Geometry* g, unsigned first, const unsigned* start, const unsigned* num, unsigned hit_offset)
  {
    if (threadIdx.x < 3) {
      const unsigned mp = first - threadIdx.x;
      s.md[threadIdx.x].hit_start = start[mp] - hit_offset;
      s.md[threadIdx.x].hit_num = num[mp];
      s.md[threadIdx.x].z[0] = __ldg(g->module_zs + 2 * mp);
      s.md[threadIdx.x].z[1] = __ldg(g->module_zs + 2 * mp + 1);
    }
  }

  __global__ void __launch_bounds__(search_threads) search_by_triplet_kernel(SearchParams p)
  {
    extern __shared__ __align__(128) unsigned char dsmem[];
    __shared__ SearchShared s;
    __shared__ unsigned filter_count;

    const unsigned e = blockIdx.x;
    const unsigned n = p.n_events;
    const unsigned* start = p.offsets_estimated_input_size + e * n_module_pairs;
    const unsigned* num = p.module_cluster_num + e * n_module_pairs;
    const unsigned hit_offset = start[0];
    const unsigned n_hits = start[n_module_pairs] - hit_offset;
    const unsigned T = p.offsets_estimated_input_size[n * n_module_pairs];
    const Constants k = p.k;
    if (T > p.cluster_capacity) return; // flagged by the clustering kernel
    if (n_hits > 65536u && threadIdx.x == 0) set_error(p.status, err_hits_per_event);

    // Track container size as SearchByTriplet.cu:23-27 computes it on the host.
    const float by_clusters = __uint2float_rn(T) * 0.34f;
    const unsigned track_container_size = by_clusters < __uint2float_rn(n * minimum_container_size) ?
                                            n * minimum_container_size :
                                            static_cast<unsigned>(by_clusters);
    const unsigned container = min(track_container_size, p.track_capacity);
    if (track_container_size > p.track_capacity && e == 0 && threadIdx.x == 0) set_error(p.status, err_input_capacity);
    const unsigned to = track_offset(p.offsets_estimated_input_size, e);
    const unsigned to_next = e + 1 < n ? track_offset(p.offsets_estimated_input_size, e + 1) : container;
    // Tracks may spill past the event's slice exactly as in the reference (no bound
    // there); writes stay inside the container and the spill is flagged.
    const unsigned track_limit = container > to ? container - to : 0u;
    TrackHits* tracks = p.tracks + to;
    TrackletHits* three_hit = p.three_hit_tracks + to;

    // Stage hits and hit_used flags
    const bool in_smem = n_hits <= p.smem_hit_capacity;
    Hits h;
    uint8_t* used;
    if (in_smem) {
      h.v = ClusterView {reinterpret_cast<char*>(dsmem), n_hits};
      h.offset = 0;
      used = dsmem + ((size_t(n_hits) * element_size + 15) & ~size_t(15));
      const ClusterView g {const_cast<char*>(p.sorted_container), T};
      for (unsigned i = threadIdx.x; i < n_hits; i += blockDim.x) {
        h.v.id(i) = g.id(hit_offset + i);
        h.v.phi(i) = g.phi(hit_offset + i);
        used[i] = 0;
      }
      const float* src = &g.x(hit_offset);
      float* dst = &h.v.x(0);
      for (unsigned i = threadIdx.x; i < 3 * n_hits; i += blockDim.x)
        dst[i] = src[i];
    }
    else {
      h.v = ClusterView {const_cast<char*>(p.sorted_container), T};
      h.offset = hit_offset;
      used = reinterpret_cast<uint8_t*>(p.hit_used) + hit_offset;
      for (unsigned i = threadIdx.x; i < n_hits; i += blockDim.x)
        used[i] = 0;
    }
    if (threadIdx.x == 0) {
      s.ttf_counter = 0;
      s.n_three = 0;
      s.local_hits = 0;
      s.n_tracks = 0;
      s.track_hits = 0;
    }
    unsigned first = n_module_pairs - 1;
    load_module_pairs(s, p.geo, first, start, num, hit_offset);
    __syncthreads();

    seeding(s, k, h, used, 8);

    unsigned last_ttf = 0;
    --first;
    while (first > 1) {
      load_module_pairs(s, p.geo, first, start, num, hit_offset);
      const unsigned prev_ttf = last_ttf;
      last_ttf = s.ttf_counter;
      const unsigned diff = last_ttf - prev_ttf;
      if (threadIdx.x == 0) s.local_hits = 0;
      __syncthreads();
      forwarding(s, k, h, used, prev_ttf, diff, tracks, track_limit, three_hit, track_limit, p.status);
      // The ring holds 2048 entries; beyond that the reference overwrites entries it has
      // not read yet, an order-dependent outcome this kernel does not reproduce.
      if (threadIdx.x == 0 && s.ttf_counter - prev_ttf > max_tracks_to_follow) set_error(p.status, err_ttf_overflow);
      seeding(s, k, h, used, 4);
      if (threadIdx.x == 0 && s.ttf_counter - last_ttf > max_tracks_to_follow) set_error(p.status, err_ttf_overflow);
      --first;
    }

    // Tail: seeds still in flight become three-hit tracks (SearchByTriplet.cu:247-264)
    {
      const unsigned prev_ttf = last_ttf;
      last_ttf = s.ttf_counter;
      const unsigned diff = last_ttf - prev_ttf;
      for (unsigned c0 = 0; c0 < diff; c0 += blockDim.x) {
        const unsigned kk = c0 + threadIdx.x;
        unsigned full = 0;
        bool seed = false;
        if (kk < diff) {
          full = s.ttf[(prev_ttf + kk) % max_tracks_to_follow];
          seed = (full & seed_bit) == seed_bit;
        }
        unsigned total;
        const unsigned excl = block_exclusive_scan(seed ? 1u : 0u, s.warp_sums, &total);
        if (seed) {
          const unsigned slot = s.n_three + excl;
          if (slot < track_limit) three_hit[slot] = s.tracklets[full & track_number_mask];
          else set_error(p.status, err_track_capacity);
        }
        __syncthreads();
        if (threadIdx.x == 0) s.n_three += total;
        __syncthreads();
      }
    }

    if (threadIdx.x == 0) {
      unsigned* atomics = p.atomics_velo + 3 * e;
      atomics[0] = s.n_three;
      atomics[1] = s.ttf_counter;
      atomics[2] = s.local_hits;
      p.number_of_velo_tracks[e] = s.n_tracks;
      if (s.n_tracks > to_next - to) set_error(p.status, err_track_capacity);
      filter_count = 0;
    }
    if (in_smem) {
      uint8_t* g_used = reinterpret_cast<uint8_t*>(p.hit_used) + hit_offset;
      for (unsigned i = threadIdx.x; i < n_hits; i += blockDim.x)
        g_used[i] = used[i];
    }
    __syncthreads();

    // Three-hit filter (ThreeHitTracksFilter.cu:109-130), input order preserved
    const unsigned n_in = min(s.n_three, track_limit);
    TrackletHits* out = p.three_hit_tracks_output + to;
    for (unsigned c0 = 0; c0 < n_in; c0 += blockDim.x) {
      const unsigned i = c0 + threadIdx.x;
      bool keep = false;
      TrackletHits t {};
      if (i < n_in) {
        t = three_hit[i];
        const bool any_used = used[t.hits[0]] || used[t.hits[1]] || used[t.hits[2]];
        const float chi2 = means_square_fit_chi2(h, t);
        keep = !any_used && chi2 < k.max_chi2;
      }
      unsigned total;
      const unsigned excl = block_exclusive_scan(keep ? 1u : 0u, s.warp_sums, &total);
      if (keep) out[filter_count + excl] = t;
      __syncthreads();
      if (threadIdx.x == 0) filter_count += total;
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      p.number_of_three_hit_tracks_output[e] = filter_count;
      p.event_track_hits[e] = s.track_hits + 3 * filter_count;
    }
  }

} // namespace velo
