// search_by_triplet (seeding + forwarding) and the three-hit filter on sm_100a,
// one event per CTA.
//
// Reference: device/velo/search_by_triplet/src/SearchByTriplet.cu:110-609 (kernel,
// find_forward_candidate, track_seeding, track_forwarding) and
// ThreeHitTracksFilter.cu:48-169.
//
// Design.
//  * The event's sorted hits are staged once as structure-of-arrays (x, y, z, phi and a
//    flag byte holding hit_used and the module parity that forwarding needs) in shared
//    memory: 15 bytes per hit.  Events above the shared-memory capacity use the same
//    layout in a global scratch slice, through the same generic pointers.
//  * Within a step every seed candidate (h1) and every track to follow is independent:
//    seeding only reads hit_used, forwarding only writes it, and each track to follow
//    owns its track.  Seeding runs LPH lanes per h1: the lanes walk the pendulum of h0
//    candidates together (ballot), each lane extrapolates its own candidates, and a
//    shuffle reduction keeps the best (scatter, candidate order) - the same choice as the
//    reference's sequential loop.  Forwarding runs one thread per track.
//  * Output slots (ring entries, track numbers, three-hit entries) are assigned by a
//    block-wide ordered scan in item order, which is the reference's sequential order, so
//    the track containers come out bit-identical to the reference CPU build.
//  * The ring of tracks to follow (2048 entries, as the reference) keeps a seed's three
//    hits in the entry itself; each track's last two hits and hit count live in shared
//    memory, so forwarding reads no global memory.  Tracks are written to dev_tracks
//    as they grow.
//  * Leftmost binary searches over a module pair's phi go through a 128-bucket table
//    per module pair, built once per event, plus a short scan: same index, fewer loads.
#include <type_traits>

#include "velo_kernels.cuh"

namespace velo {

  constexpr uint64_t seed_flag = 1ull << 63;
  constexpr unsigned skipped_shift = 60;
  constexpr uint64_t track_number_mask64 = 0x0FFFFFFFull;
  constexpr unsigned max_tail_tracks = 512; // tracks whose tail lives in shared memory (the others: their container)
  constexpr unsigned n_buckets = 128;
  constexpr uint8_t flag_used = 1;
  constexpr uint8_t flag_odd_module = 2;
  constexpr unsigned flat_slots = 1024; // (h1, h0 candidate) slots per chunk of the flat seeding

  struct ModulePair {
    unsigned hit_start;
    unsigned hit_num;
    float z[2];
    unsigned mp;
  };

  struct SearchShared {
    unsigned scan_sums[2][32]; // double-buffered warp totals of the block scans
    unsigned track_hits;       // sum of hitsNum over the >= 4 hit tracks
    uint32_t tail[max_tail_tracks]; // last two hits of a track (hit[n-2] | hit[n-1] << 16)
    uint8_t tail_n[max_tail_tracks];
    uint16_t bucket[n_module_pairs][n_buckets + 1];
  };

  // Shared state of the flat seeding variant: one slot per (h1, candidate order).
  // SLOTS doublets per chunk; MLP adds the seed pruner's staging rows (learned kernel).
  template<unsigned SLOTS, bool MLP>
  struct SearchSharedFlatT : SearchShared {
    static constexpr unsigned slots = SLOTS;
    // (h0, h1) doublets of a chunk, packed by pack_doublet(), then overwritten in place
    // with the best scatter found for the doublet
    union {
      uint32_t doublet;
      float fit;
    } slot[SLOTS];
    union alignas(16) { // ldmatrix reads 16-byte rows of mlp_rows
      uint16_t res_h2[SLOTS];
      uint32_t mlp_rows[MLP ? 8 : 1][16][8]; // per warp: 16 doublets x 16 bf16 inputs (learned mode)
    };
  };
  using SearchSharedFlat = SearchSharedFlatT<flat_slots, true>;
  // plain flat-seeding kernels: 512 slots for 128 threads (chunks of 64 or 128 h1), which with
  // the ring in global scratch leaves room for twelve CTAs per SM
  template<unsigned THREADS>
  using SearchSharedFlatPlain =
    SearchSharedFlatT<(THREADS <= 64 ? flat_slots / 4 : (THREADS <= 128 ? flat_slots / 2 : flat_slots)), false>;

  // Packed doublet: h0 | h1 index in the chunk << 16 | rank << 25 | (found - 1) << 28 | keep << 31
  __device__ __forceinline__ uint32_t pack_doublet(unsigned h0, unsigned h1_local, unsigned rank, unsigned found)
  {
    return h0 | (h1_local << 16) | (rank << 25) | ((found - 1u) << 28);
  }
  constexpr uint32_t doublet_keep = 1u << 31;

  struct HitsSoA {
    const float* x;
    const float* y;
    const float* z;
    const int16_t* phi;
    uint8_t* flags;
  };

  // The event's counters (the reference's dev_atomics_velo and track count), kept in
  // registers: every thread holds the same values and advances them by scan totals.
  struct Counters {
    unsigned ttf;        // atomics::tracks_to_follow
    unsigned n_three;    // atomics::number_of_three_hit_tracks
    unsigned local_hits; // atomics::local_number_of_hits
    unsigned n_tracks;   // dev_number_of_velo_tracks
    unsigned scan_parity;
    unsigned doublets;   // (h0, h1) doublets formed by the flat seeding
    unsigned kept;       // doublets whose h2 window was scanned
  };

  // Block-wide exclusive scan with a single barrier: warp totals go to one of two
  // buffers, alternating per call, so a call never overwrites totals still being read.
  __device__ __forceinline__ unsigned scan1(SearchShared& s, Counters& c, unsigned v, unsigned& total)
  {
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    unsigned incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= static_cast<unsigned>(o)) incl += t;
    }
    unsigned* buf = s.scan_sums[c.scan_parity];
    c.scan_parity ^= 1u;
    if (lane == 31) buf[warp] = incl;
    __syncthreads();
    unsigned before = 0, all = 0;
    for (unsigned w = 0; w < n_warps; ++w) {
      const unsigned t = buf[w];
      before += w < warp ? t : 0u;
      all += t;
    }
    total = all;
    return before + incl - v;
  }

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

  __device__ __forceinline__ bool phi_outside(int16_t phi, int16_t extrapolated, int16_t tol)
  {
    const int16_t diff = static_cast<int16_t>(phi - extrapolated);
    const int16_t abs_diff = static_cast<int16_t>(diff < 0 ? -diff : diff);
    return abs_diff > tol;
  }

  struct Extrapolation {
    int start;   // first h2 candidate (find_forward_candidate, SearchByTriplet.cu:272-292)
    int16_t phi; // extrapolated phi
  };

  __device__ __forceinline__ Extrapolation extrapolate(
    const Constants& k,
    const SearchShared& s,
    const HitsSoA& h,
    const ModulePair& next,
    float h0x,
    float h0y,
    float tx,
    float ty,
    float dz)
  {
    const float predx = tx * dz;
    const float predy = ty * dz;
    const float xp = h0x + predx;
    const float yp = h0y + predy;
    Extrapolation x;
    x.phi = hit_phi_16(k, xp, yp);
    const int16_t lo = static_cast<int16_t>(x.phi - static_cast<int16_t>(k.phi_tolerance_i16));
    // find_forward_candidate returns the index as int16
    x.start = static_cast<int16_t>(leftmost(s.bucket[next.mp], h.phi + next.hit_start, next.hit_num, lo));
    return x;
  }

  // One h0 candidate of a seed (SearchByTriplet.cu:374-432): updates (best_fit, best_c,
  // best_h0, best_h2) with strict improvement, in window order.
  __device__ __forceinline__ void seed_candidate(
    const Constants& k,
    const SearchShared& s,
    const HitsSoA& h,
    const ModulePair& prev,
    const ModulePair& next,
    float h1x,
    float h1y,
    float h1z,
    unsigned h0,
    unsigned c,
    float& best_fit,
    unsigned& best_c,
    unsigned& best_h0,
    unsigned& best_h2)
  {
    const int16_t tol = static_cast<int16_t>(k.phi_tolerance_i16);
    const float h0x = h.x[h0], h0y = h.y[h0], h0z = h.z[h0];
    const float td = __fdiv_rn(1.0f, h1z - h0z);
    const float txn = h1x - h0x;
    const float tyn = h1y - h0y;
    const float tx = txn * td;
    const float ty = tyn * td;
    const Extrapolation f = extrapolate(k, s, h, next, h0x, h0y, tx, ty, next.z[0] - prev.z[0]);
    // circular walk from the candidate: index (start + j) % n without a division per step
    unsigned idx = next.hit_num ? static_cast<unsigned>(f.start) % next.hit_num : 0u;
    for (unsigned j = 0; j < next.hit_num; ++j, idx = (idx + 1 == next.hit_num) ? 0u : idx + 1) {
      const unsigned h2 = next.hit_start + idx;
      if (phi_outside(h.phi[h2], f.phi, tol)) break;
      if (h.flags[h2] & flag_used) continue;
      const float dz = h.z[h2] - h0z;
      const float predx = h0x + tx * dz;
      const float predy = h0y + ty * dz;
      const float dx = predx - h.x[h2];
      const float dy = predy - h.y[h2];
      const float scatter = dx * dx + dy * dy;
      if (scatter < best_fit) {
        best_fit = scatter;
        best_c = c;
        best_h0 = h0;
        best_h2 = h2;
      }
    }
  }

  // Seeding over the current module pair (SearchByTriplet.cu:298-446), LPH lanes per h1.
  template<unsigned LPH>
  __device__ __forceinline__ void seeding(
    SearchShared& s, uint64_t* ring, Counters& cnt, const Constants& k, const HitsSoA& h, const ModulePair* md,
    unsigned n_candidates)
  {
    const ModulePair prev = md[0], cur = md[1], next = md[2];
    const unsigned groups = blockDim.x / LPH;
    const unsigned g = threadIdx.x / LPH;
    const unsigned l = threadIdx.x % LPH;
    const unsigned lane0 = (threadIdx.x & 31u) & ~(LPH - 1);
    const unsigned gmask = (LPH == 32 ? 0xFFFFFFFFu : ((1u << LPH) - 1u)) << lane0;
    for (unsigned c0 = 0; c0 < cur.hit_num; c0 += groups) {
      const unsigned r = c0 + g;
      const unsigned h1 = cur.hit_start + r;
      const bool valid = r < cur.hit_num && !(h.flags[h1] & flag_used);
      float best_fit = k.max_scatter;
      unsigned best_c = 0xFFFFFFFFu, best_h0 = 0, best_h2 = 0;
      if (valid) {
        const float h1x = h.x[h1], h1y = h.y[h1], h1z = h.z[h1];
        const int p0 = leftmost(s.bucket[prev.mp], h.phi + prev.hit_start, prev.hit_num, h.phi[h1]);
        const int n_prev = static_cast<int>(prev.hit_num);
        unsigned found = 0;
        for (unsigned i0 = 0; i0 < prev.hit_num && found < n_candidates; i0 += LPH) {
          const unsigned i = i0 + l;
          bool ok = false;
          unsigned h0 = 0;
          if (i < prev.hit_num) {
            // pendulum p0, p0 + 1, p0 - 1, p0 + 2, ... with one wrap (SearchByTriplet.cu:351-370)
            const int pos = p0 + ((i & 1u) ? static_cast<int>((i + 1) / 2) : -static_cast<int>(i / 2));
            const int in_bounds = pos < 0 ? pos + n_prev : (pos >= n_prev ? pos - n_prev : pos);
            h0 = prev.hit_start + static_cast<unsigned>(in_bounds);
            ok = !(h.flags[h0] & flag_used);
          }
          const unsigned ballot = (__ballot_sync(gmask, ok) & gmask) >> lane0;
          const unsigned rank = __popc(ballot & ((1u << l) - 1u));
          if (ok && found + rank < n_candidates) {
            seed_candidate(k, s, h, prev, next, h1x, h1y, h1z, h0, found + rank, best_fit, best_c, best_h0, best_h2);
          }
          found += __popc(ballot);
        }
#pragma unroll
        for (unsigned o = LPH / 2; o >= 1; o /= 2) {
          const float of = __shfl_xor_sync(gmask, best_fit, o);
          const unsigned oc = __shfl_xor_sync(gmask, best_c, o);
          const unsigned o0 = __shfl_xor_sync(gmask, best_h0, o);
          const unsigned o2 = __shfl_xor_sync(gmask, best_h2, o);
          if (of < best_fit || (of == best_fit && oc < best_c)) {
            best_fit = of;
            best_c = oc;
            best_h0 = o0;
            best_h2 = o2;
          }
        }
      }
      const bool ok = valid && l == 0 && best_fit < k.max_scatter;
      const unsigned unused = (valid && l == 0) ? 1u : 0u;
      unsigned total;
      const unsigned excl = scan1(s, cnt, (ok ? 1u : 0u) | (unused << 16), total);
      if (ok) {
        const unsigned tn = (cnt.ttf + (excl & 0xFFFFu)) % max_tracks_to_follow;
        ring[tn] = seed_flag | (uint64_t(best_h0 & 0xFFFFu)) | (uint64_t(h1 & 0xFFFFu) << 16) |
                     (uint64_t(best_h2 & 0xFFFFu) << 32);
      }
      cnt.ttf += total & 0xFFFFu;
      cnt.local_hits += total >> 16;
    }
  }

  __device__ __forceinline__ unsigned candidate_h0(uint64_t lo, uint64_t hi, unsigned c)
  {
    return static_cast<unsigned>((c < 4 ? lo >> (16 * c) : hi >> (16 * (c - 4))) & 0xFFFFu);
  }

  // Learned mode: scores the n doublets of the list with the network and sets the keep bit
  // of those above the threshold.  Warps 0..7 take 16-doublet tiles; lanes 0..15 compute one
  // doublet's inputs each into the warp's staging rows, ldmatrix forms the A fragment.
  __device__ __forceinline__ void score_doublets(
    SearchSharedFlat& s, const MlpModelDevice* m, const HitsSoA& h, unsigned h1_base, unsigned n)
  {
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const unsigned n_warps = min(blockDim.x >> 5, 8u);
    if (warp >= n_warps) return;
    uint32_t(*rows)[8] = s.mlp_rows[warp];
    for (unsigned t = warp; 16 * t < n; t += n_warps) {
      if (lane < 16) {
        const unsigned q = 16 * t + lane;
        uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (q < n) {
          const uint32_t d = s.slot[q].doublet;
          const unsigned h0 = d & 0xFFFFu, h1 = h1_base + ((d >> 16) & 0x1FFu);
          float f[mlp_features];
          doublet_features(h.x[h0], h.y[h0], h.z[h0], h.phi[h0], h.x[h1], h.y[h1], h.z[h1], h.phi[h1], (d >> 25) & 7u,
                           ((d >> 28) & 7u) + 1u, f);
          standardise_pairs(*m, f, w);
        }
#pragma unroll
        for (unsigned i = 0; i < 8; ++i)
          rows[lane][i] = w[i];
      }
      __syncwarp();
      uint32_t a[4];
      ldmatrix_x4(a, &rows[lane & 15u][(lane >> 4) * 4]);
      float lg, lg8;
      mlp_forward_tile(m, a, lg, lg8);
      if ((lane & 3u) == 0) {
        const float thr = __ldg(&m->threshold_logit);
        const unsigned q0 = 16 * t + (lane >> 2), q1 = q0 + 8;
        if (q0 < n && lg > thr) s.slot[q0].doublet |= doublet_keep;
        if (q1 < n && lg8 > thr) s.slot[q1].doublet |= doublet_keep;
      }
      __syncwarp();
    }
  }

  // Seeding with the candidates flattened (SearchByTriplet.cu:298-446).  Phase A, one
  // thread per h1, walks the pendulum and keeps its first n_candidates unused h0 in
  // registers; a block scan packs all (h0, h1) doublets of the chunk into one list.
  // Phase B, one thread per doublet, extrapolates and scans the h2 window.  Phase C, one
  // thread per h1, keeps the first strictly best of its doublets in candidate order (the
  // reference's sequential choice) and queues the seed in h1 order.  Phase B runs the same
  // path on every lane and has no idle slots for h1 with fewer than n_candidates doublets.
  // LEARNED kernels can also score the doublets with the seed pruner (only kept doublets
  // reach phase B) and record training doublets.
  template<bool LEARNED, typename Flat>
  __device__ __forceinline__ void seeding_flat(
    Flat& s,
    uint64_t* ring,
    Counters& cnt,
    const Constants& k,
    const HitsSoA& h,
    const ModulePair* md,
    unsigned n_candidates,
    const SearchParams& p,
    bool learned,
    unsigned event,
    unsigned hit_offset)
  {
    const ModulePair prev = md[0], cur = md[1], next = md[2];
    const unsigned per_chunk = min(blockDim.x, Flat::slots / n_candidates);
    const int n_prev = static_cast<int>(prev.hit_num);
    const int16_t tol = static_cast<int16_t>(k.phi_tolerance_i16);
    for (unsigned c0 = 0; c0 < cur.hit_num; c0 += per_chunk) {
      const unsigned n_h1 = min(per_chunk, cur.hit_num - c0);
      // Phase A: candidates c < 4 in the 16-bit fields of cand_lo, 4..7 in cand_hi
      const unsigned h1 = cur.hit_start + c0 + threadIdx.x;
      const bool valid = threadIdx.x < n_h1 && !(h.flags[h1] & flag_used);
      uint64_t cand_lo = 0, cand_hi = 0;
      unsigned found = 0;
      if (valid) {
        const int p0 = leftmost(s.bucket[prev.mp], h.phi + prev.hit_start, prev.hit_num, h.phi[h1]);
        int pos = p0;
        for (unsigned i = 0; i < prev.hit_num && found < n_candidates; ++i) {
          pos += (i & 1u) ? static_cast<int>(i) : -static_cast<int>(i);
          const int in_bounds = pos < 0 ? pos + n_prev : (pos >= n_prev ? pos - n_prev : pos);
          const unsigned h0 = prev.hit_start + static_cast<unsigned>(in_bounds);
          if (!(h.flags[h0] & flag_used)) {
            if (found < 4) cand_lo |= uint64_t(h0) << (16 * found);
            else cand_hi |= uint64_t(h0) << (16 * (found - 4));
            ++found;
          }
        }
      }
      unsigned n_doublets;
      unsigned first = scan1(s, cnt, found, n_doublets);
      for (unsigned c = 0; c < found; ++c)
        s.slot[first + c].doublet = pack_doublet(candidate_h0(cand_lo, cand_hi, c), threadIdx.x, c, found);
      __syncthreads();
      cnt.doublets += n_doublets;
      // keep_mask bit c: the h2 window of doublet c is scanned (always, in the plain search)
      unsigned keep_mask = (1u << found) - 1u;
      if constexpr (LEARNED) if (learned) {
        score_doublets(s, p.seed_model, h, cur.hit_start + c0, n_doublets);
        __syncthreads();
        keep_mask = 0;
        for (unsigned c = 0; c < found; ++c)
          keep_mask |= (s.slot[first + c].doublet >> 31) << c;
        // pack the kept doublets (reads above, writes after the scan's barrier)
        first = scan1(s, cnt, __popc(keep_mask), n_doublets);
        unsigned at = first;
        for (unsigned c = 0; c < found; ++c)
          if (keep_mask & (1u << c))
            s.slot[at++].doublet = pack_doublet(candidate_h0(cand_lo, cand_hi, c), threadIdx.x, c, found);
        __syncthreads();
      }
      cnt.kept += n_doublets;
      // Phase B
      for (unsigned q = threadIdx.x; q < n_doublets; q += blockDim.x) {
        const uint32_t d = s.slot[q].doublet;
        const unsigned h0 = d & 0xFFFFu;
        const unsigned hh1 = cur.hit_start + c0 + ((d >> 16) & 0x1FFu);
        float best_fit = k.max_scatter;
        unsigned best_h2 = 0xFFFFu;
        const float h1x = h.x[hh1], h1y = h.y[hh1], h1z = h.z[hh1];
        const float h0x = h.x[h0], h0y = h.y[h0], h0z = h.z[h0];
        const float td = __fdiv_rn(1.0f, h1z - h0z);
        const float txn = h1x - h0x;
        const float tyn = h1y - h0y;
        const float tx = txn * td;
        const float ty = tyn * td;
        const Extrapolation f = extrapolate(k, s, h, next, h0x, h0y, tx, ty, next.z[0] - prev.z[0]);
        unsigned idx = next.hit_num ? static_cast<unsigned>(f.start) % next.hit_num : 0u;
        for (unsigned j = 0; j < next.hit_num; ++j, idx = (idx + 1 == next.hit_num) ? 0u : idx + 1) {
          const unsigned h2 = next.hit_start + idx;
          if (phi_outside(h.phi[h2], f.phi, tol)) break;
          if (h.flags[h2] & flag_used) continue;
          const float dz = h.z[h2] - h0z;
          const float predx = h0x + tx * dz;
          const float predy = h0y + ty * dz;
          const float dx = predx - h.x[h2];
          const float dy = predy - h.y[h2];
          const float scatter = dx * dx + dy * dy;
          if (scatter < best_fit) {
            best_fit = scatter;
            best_h2 = h2;
          }
        }
        s.slot[q].fit = best_fit;
        s.res_h2[q] = static_cast<uint16_t>(best_h2);
      }
      __syncthreads();
      // Phase C
      bool ok = false;
      unsigned best_h0 = 0, best_h2 = 0, best_c = 0xFFFFFFFFu;
      if (valid) {
        float best_fit = k.max_scatter;
        unsigned at = first;
        for (unsigned c = 0; c < found; ++c) {
          if (!(keep_mask & (1u << c))) continue;
          const float fit = s.slot[at].fit;
          if (fit < best_fit) {
            best_fit = fit;
            best_c = c;
            best_h0 = candidate_h0(cand_lo, cand_hi, c);
            best_h2 = s.res_h2[at];
          }
          ++at;
        }
        ok = best_fit < k.max_scatter;
        // training doublets: every candidate of one h1 in record_every, labelled by the choice
        if (LEARNED && p.records != nullptr && found > 0 &&
            ((event * 0x9E3779B1u) ^ ((hit_offset + h1) * 0x85EBCA77u)) % p.record_every == 0) {
          const unsigned slot0 = atomicAdd(p.record_count, found);
          for (unsigned c = 0; c < found && slot0 + found <= p.record_capacity; ++c) {
            const unsigned h0 = candidate_h0(cand_lo, cand_hi, c);
            DoubletRecord r;
            doublet_features(h.x[h0], h.y[h0], h.z[h0], h.phi[h0], h.x[h1], h.y[h1], h.z[h1], h.phi[h1], c, found, r.f);
            r.label = (ok && c == best_c) ? 1.0f : 0.0f;
            r.event = event;
            r.h0 = hit_offset + h0;
            r.h1 = hit_offset + h1;
            p.records[slot0 + c] = r;
          }
        }
      }
      unsigned total;
      const unsigned excl = scan1(s, cnt, (ok ? 1u : 0u) | ((valid ? 1u : 0u) << 16), total);
      if (ok) {
        const unsigned tn = (cnt.ttf + (excl & 0xFFFFu)) % max_tracks_to_follow;
        ring[tn] = seed_flag | (uint64_t(best_h0 & 0xFFFFu)) | (uint64_t(h1 & 0xFFFFu) << 16) |
                     (uint64_t(best_h2 & 0xFFFFu) << 32);
      }
      cnt.ttf += total & 0xFFFFu;
      cnt.local_hits += total >> 16;
    }
  }

  // Forwarding of the tracks to follow (SearchByTriplet.cu:451-609), one thread per track.
  __device__ __forceinline__ void forwarding(
    SearchShared& s,
    uint64_t* ring,
    Counters& cnt,
    const Constants& k,
    const HitsSoA& h,
    const ModulePair& next,
    unsigned prev_ttf,
    unsigned diff_ttf,
    TrackHits* tracks,
    unsigned track_limit,
    TrackletHits* three_hit,
    unsigned* status)
  {
    const int16_t tol = static_cast<int16_t>(k.phi_tolerance_i16);
    for (unsigned c0 = 0; c0 < diff_ttf; c0 += blockDim.x) {
      const unsigned kk = c0 + threadIdx.x;
      const bool active = kk < diff_ttf;
      uint64_t entry = 0;
      unsigned nh = 0, tn = 0, h0n = 0, h1n = 0;
      bool is_seed = false, found = false;
      unsigned best_h2 = 0;
      if (active) {
        entry = ring[(prev_ttf + kk) % max_tracks_to_follow];
        is_seed = (entry & seed_flag) != 0;
        if (is_seed) {
          nh = 3;
          h0n = static_cast<unsigned>(entry >> 16) & 0xFFFFu;
          h1n = static_cast<unsigned>(entry >> 32) & 0xFFFFu;
        }
        else {
          tn = static_cast<unsigned>(entry & track_number_mask64);
          if (tn < max_tail_tracks) {
            nh = s.tail_n[tn];
            h0n = s.tail[tn] & 0xFFFFu;
            h1n = s.tail[tn] >> 16;
          }
          else if (tn < track_limit) {
            nh = tracks[tn].hits_num;
            if (nh < 2 || nh > max_track_size) nh = 2;
            h0n = tracks[tn].hits[nh - 2];
            h1n = tracks[tn].hits[nh - 1];
          }
          else {
            nh = 3; // a track that did not fit its container, flagged when created
          }
        }
        const float h0x = h.x[h0n], h0y = h.y[h0n], h0z = h.z[h0n];
        const unsigned odd = (h.flags[h0n] & flag_odd_module) ? 1u : 0u;
        const float h1x = h.x[h1n], h1y = h.y[h1n], h1z = h.z[h1n];
        const float td = __fdiv_rn(1.0f, h1z - h0z);
        const float txn = h1x - h0x;
        const float tyn = h1y - h0y;
        const float tx = txn * td;
        const float ty = tyn * td;
        float best_fit = k.max_scatter;
        const Extrapolation f = extrapolate(k, s, h, next, h0x, h0y, tx, ty, next.z[odd] - h0z);
        unsigned idx = next.hit_num ? static_cast<unsigned>(f.start) % next.hit_num : 0u;
        for (unsigned j = 0; j < next.hit_num; ++j, idx = (idx + 1 == next.hit_num) ? 0u : idx + 1) {
          const unsigned h2 = next.hit_start + idx;
          if (phi_outside(h.phi[h2], f.phi, tol)) break;
          const float dz = h.z[h2] - h0z;
          const float predx = h0x + tx * dz;
          const float predy = h0y + ty * dz;
          const float dx = predx - h.x[h2];
          const float dy = predy - h.y[h2];
          const float scatter = dx * dx + dy * dy;
          if (scatter < best_fit) {
            best_fit = scatter;
            best_h2 = h2;
            found = true;
          }
        }
      }
      const unsigned skipped = static_cast<unsigned>(entry >> skipped_shift) & 0x7u;
      const bool new_track = active && found && is_seed;
      const bool enqueue =
        active && ((found && nh + 1 < max_track_size) || (!found && skipped < k.max_skipped_modules));
      const bool three = active && !found && !(skipped < k.max_skipped_modules) && nh == 3 && is_seed;
      unsigned total;
      const unsigned excl =
        scan1(s, cnt, (new_track ? 1u : 0u) | ((enqueue ? 1u : 0u) << 10) | ((three ? 1u : 0u) << 20), total);
      if (active) {
        unsigned track_number = tn;
        if (found) {
          h.flags[best_h2] |= flag_used;
          if (is_seed) {
            const unsigned t0 = static_cast<unsigned>(entry) & 0xFFFFu;
            h.flags[t0] |= flag_used;
            h.flags[h0n] |= flag_used;
            h.flags[h1n] |= flag_used;
            track_number = cnt.n_tracks + (excl & 0x3FFu);
            if (track_number < track_limit) {
              TrackHits& t = tracks[track_number];
              t.hits[0] = static_cast<uint16_t>(t0);
              t.hits[1] = static_cast<uint16_t>(h0n);
              t.hits[2] = static_cast<uint16_t>(h1n);
              t.hits[3] = static_cast<uint16_t>(best_h2);
              t.hits_num = 4;
            }
            else {
              set_error(status, err_track_capacity);
            }
            if (track_number < max_tail_tracks) {
              s.tail[track_number] = h1n | (best_h2 << 16);
              s.tail_n[track_number] = 4;
            }
          }
          else {
            if (tn < track_limit) {
              tracks[tn].hits[nh] = static_cast<uint16_t>(best_h2);
              tracks[tn].hits_num = static_cast<uint8_t>(nh + 1);
            }
            if (tn < max_tail_tracks) {
              s.tail[tn] = h1n | (best_h2 << 16);
              s.tail_n[tn] = static_cast<uint8_t>(nh + 1);
            }
          }
          atomicAdd(&s.track_hits, is_seed ? 4u : 1u);
        }
        if (enqueue) {
          // requeued entries keep the seed's hits or the track number, with skipped + 1
          const uint64_t value =
            found ? uint64_t(track_number) :
                    ((entry & ~(uint64_t(0x7) << skipped_shift)) | (uint64_t(skipped + 1) << skipped_shift));
          ring[(cnt.ttf + ((excl >> 10) & 0x3FFu)) % max_tracks_to_follow] = value;
        }
        if (three) {
          const unsigned slot = cnt.n_three + ((excl >> 20) & 0x3FFu);
          if (slot < track_limit) {
            three_hit[slot] = TrackletHits {
              {static_cast<uint16_t>(entry & 0xFFFFu), static_cast<uint16_t>(h0n), static_cast<uint16_t>(h1n)}};
          }
          else {
            set_error(status, err_track_capacity);
          }
        }
      }
      cnt.n_tracks += total & 0x3FFu;
      cnt.ttf += (total >> 10) & 0x3FFu;
      cnt.n_three += (total >> 20) & 0x3FFu;
    }
  }

  // ThreeHitTracksFilter.cu:48-107
  __device__ __forceinline__ float means_square_fit_chi2(const HitsSoA& h, const TrackletHits& t)
  {
    const float w = 6400.f;
    float s0, sx, sz, sxz, sz2, u0, uy, uz, uyz, uz2;
    s0 = sx = sz = sxz = sz2 = 0.0f;
    u0 = uy = uz = uyz = uz2 = 0.0f;
#pragma unroll
    for (unsigned i = 0; i < 3; ++i) {
      const unsigned hn = t.hits[i];
      const float x = h.x[hn], y = h.y[hn], z = h.z[hn];
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
      const float z = h.z[hn];
      const float x = state_x + state_tx * z;
      const float y = state_y + state_ty * z;
      const float dx = x - h.x[hn];
      const float dy = y - h.y[hn];
      chi2 += dx * dx * w + dy * dy * w;
    }
    return chi2 * 0.5f;
  }

  // The three module pairs of a step (first, first - 1, first - 2), read by every thread.
  __device__ __forceinline__ void module_pairs(
    ModulePair* md, const Geometry* g, unsigned first, const unsigned* start, const unsigned* num, unsigned hit_offset)
  {
#pragma unroll
    for (unsigned i = 0; i < 3; ++i) {
      const unsigned mp = first - i;
      md[i].hit_start = start[mp] - hit_offset;
      md[i].hit_num = num[mp];
      md[i].z[0] = __ldg(g->module_zs + 2 * mp);
      md[i].z[1] = __ldg(g->module_zs + 2 * mp + 1);
      md[i].mp = mp;
    }
  }

  // Seeding, forwarding and the tail of one event over staged hits (hit_used clear):
  // SearchByTriplet.cu:165-264.  Returns the event's counters; the track containers hold
  // its tracks and three-hit tracks.
  template<unsigned LPH, bool LEARNED, typename Shared>
  __device__ __forceinline__ Counters search_pass(
    const SearchParams& p,
    Shared& s,
    uint64_t* ring,
    const Constants& k,
    const HitsSoA& h,
    const unsigned* start,
    const unsigned* num,
    unsigned hit_offset,
    unsigned e,
    TrackHits* tracks,
    unsigned track_limit,
    TrackletHits* three_hit,
    bool learned)
  {
    if (threadIdx.x == 0) s.track_hits = 0;
    Counters cnt {0, 0, 0, 0, 0, 0, 0};
    __syncthreads();
    unsigned first = n_module_pairs - 1;
    ModulePair md[3];
    module_pairs(md, p.geo, first, start, num, hit_offset);
    __syncthreads(); // bucket tables

    if constexpr (LPH == 0) seeding_flat<LEARNED>(s, ring, cnt, k, h, md, 8, p, learned, e, hit_offset);
    else seeding<LPH>(s, ring, cnt, k, h, md, 8);

    unsigned last_ttf = 0;
    --first;
    while (first > 1) {
      module_pairs(md, p.geo, first, start, num, hit_offset);
      const unsigned prev_ttf = last_ttf;
      last_ttf = cnt.ttf;
      const unsigned diff = last_ttf - prev_ttf;
      cnt.local_hits = 0;
      __syncthreads(); // ring entries of the last seeding
      forwarding(s, ring, cnt, k, h, md[2], prev_ttf, diff, tracks, track_limit, three_hit, p.status);
      // The ring holds 2048 entries; beyond that the reference overwrites entries it has
      // not read yet, an order-dependent outcome this kernel does not reproduce.
      if (threadIdx.x == 0 && cnt.ttf - prev_ttf > max_tracks_to_follow) set_error(p.status, err_ttf_overflow);
      __syncthreads(); // hit_used flags written by forwarding
      if constexpr (LPH == 0) seeding_flat<LEARNED>(s, ring, cnt, k, h, md, 4, p, learned, e, hit_offset);
      else seeding<LPH>(s, ring, cnt, k, h, md, 4);
      if (threadIdx.x == 0 && cnt.ttf - last_ttf > max_tracks_to_follow) set_error(p.status, err_ttf_overflow);
      --first;
    }
    __syncthreads(); // ring entries of the last seeding

    // Tail: seeds still in flight become three-hit tracks (SearchByTriplet.cu:247-264)
    {
      const unsigned prev_ttf = last_ttf;
      last_ttf = cnt.ttf;
      const unsigned diff = last_ttf - prev_ttf;
      for (unsigned c0 = 0; c0 < diff; c0 += blockDim.x) {
        const unsigned kk = c0 + threadIdx.x;
        uint64_t entry = 0;
        bool seed = false;
        if (kk < diff) {
          entry = ring[(prev_ttf + kk) % max_tracks_to_follow];
          seed = (entry & seed_flag) != 0;
        }
        unsigned total;
        const unsigned excl = scan1(s, cnt, seed ? 1u : 0u, total);
        if (seed) {
          const unsigned slot = cnt.n_three + excl;
          if (slot < track_limit) {
            three_hit[slot] = TrackletHits {{static_cast<uint16_t>(entry & 0xFFFFu),
                                             static_cast<uint16_t>((entry >> 16) & 0xFFFFu),
                                             static_cast<uint16_t>((entry >> 32) & 0xFFFFu)}};
          }
          else {
            set_error(p.status, err_track_capacity);
          }
        }
        cnt.n_three += total;
      }
    }

    return cnt;
  }

  template<unsigned LPH, bool SMEM, bool LEARNED, typename Shared>
  __device__ __forceinline__ void
  search_event(const SearchParams& p, Shared& s, uint64_t* ring, unsigned char* dsmem, unsigned e)
  {
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

    // Stage the hits as SoA: shared memory when they fit (SMEM), else the event's global
    // slice (16 bytes per estimated hit, so every slice starts 16-byte aligned).
    unsigned char* base = SMEM ? dsmem : reinterpret_cast<unsigned char*>(p.hit_scratch) + size_t(16) * hit_offset;
    const unsigned cap = SMEM ? p.smem_hit_capacity : n_hits;
    float* xs = reinterpret_cast<float*>(base);
    float* ys = xs + cap;
    float* zs = ys + cap;
    int16_t* phis = reinterpret_cast<int16_t*>(zs + cap);
    uint8_t* flags = reinterpret_cast<uint8_t*>(phis + cap);
    {
      const ClusterView g {const_cast<char*>(p.sorted_container), T};
      for (unsigned i = threadIdx.x; i < n_hits; i += blockDim.x) {
        const unsigned gi = hit_offset + i;
        xs[i] = g.x(gi);
        ys[i] = g.y(gi);
        zs[i] = g.z(gi);
        phis[i] = g.phi(gi);
        const unsigned module = ((g.id(gi) & 0x3FC0000u) >> 18) / 4;
        flags[i] = (module & 1u) ? flag_odd_module : 0;
      }
    }
    const HitsSoA h {xs, ys, zs, phis, flags};
    // bucket tables: bucket[mp][b] = first index of the module pair with phi >= b * 512 - 32768
    for (unsigned mp = 0; mp < n_module_pairs; ++mp) {
      const unsigned s0 = start[mp] - hit_offset;
      const unsigned cnt = num[mp];
      uint16_t* table = s.bucket[mp];
      for (unsigned i = threadIdx.x; i <= cnt; i += blockDim.x) {
        const unsigned lo = i == 0 ? 0u : bucket_of(phis[s0 + i - 1]) + 1;
        const unsigned hi = i == cnt ? n_buckets : bucket_of(phis[s0 + i]);
        for (unsigned b = lo; b <= hi; ++b)
          table[b] = static_cast<uint16_t>(i);
      }
    }

    // Learned mode: the pruned search first; an event whose fraction of kept doublets falls
    // outside the model's bounds is searched again by the plain search, from scratch.
    const bool learned = LEARNED && p.seed_model != nullptr;
    Counters cnt =
      search_pass<LPH, LEARNED>(p, s, ring, k, h, start, num, hit_offset, e, tracks, track_limit, three_hit, learned);
    unsigned mode = learned ? seed_mode_learned : seed_mode_plain;
    const unsigned doublets = cnt.doublets, kept = cnt.kept;
    if (learned && doublets > 0) {
      const float frac = __fdiv_rn(__uint2float_rn(kept), __uint2float_rn(doublets));
      if (frac < __ldg(&p.seed_model->kept_lo) || frac > __ldg(&p.seed_model->kept_hi)) {
        mode = seed_mode_fallback;
        __syncthreads();
        for (unsigned i = threadIdx.x; i < n_hits; i += blockDim.x)
          flags[i] &= static_cast<uint8_t>(~flag_used);
        cnt = search_pass<LPH, LEARNED>(p, s, ring, k, h, start, num, hit_offset, e, tracks, track_limit, three_hit, false);
      }
    }
    if (p.seed_stats != nullptr && threadIdx.x == 0) {
      p.seed_stats[3 * e] = doublets;
      p.seed_stats[3 * e + 1] = kept;
      p.seed_stats[3 * e + 2] = mode;
    }

    if (threadIdx.x == 0) {
      unsigned* atomics = p.atomics_velo + 3 * e;
      atomics[0] = cnt.n_three;
      atomics[1] = cnt.ttf;
      atomics[2] = cnt.local_hits;
      p.number_of_velo_tracks[e] = cnt.n_tracks;
      if (cnt.n_tracks > to_next - to) set_error(p.status, err_track_capacity);
    }
    {
      uint8_t* g_used = reinterpret_cast<uint8_t*>(p.hit_used) + hit_offset;
      for (unsigned i = threadIdx.x; i < n_hits; i += blockDim.x)
        g_used[i] = flags[i] & flag_used;
    }
    __syncthreads();

    // Three-hit filter (ThreeHitTracksFilter.cu:109-130), input order preserved
    const unsigned n_in = min(cnt.n_three, track_limit);
    TrackletHits* out = p.three_hit_tracks_output + to;
    unsigned filter_count = 0;
    for (unsigned c0 = 0; c0 < n_in; c0 += blockDim.x) {
      const unsigned i = c0 + threadIdx.x;
      bool keep = false;
      TrackletHits t {};
      if (i < n_in) {
        t = three_hit[i];
        const bool any_used =
          (flags[t.hits[0]] & flag_used) || (flags[t.hits[1]] & flag_used) || (flags[t.hits[2]] & flag_used);
        const float chi2 = means_square_fit_chi2(h, t);
        keep = !any_used && chi2 < k.max_chi2;
      }
      unsigned total;
      const unsigned excl = scan1(s, cnt, keep ? 1u : 0u, total);
      if (keep) out[filter_count + excl] = t;
      filter_count += total;
    }
    if (threadIdx.x == 0) {
      p.number_of_three_hit_tracks_output[e] = filter_count;
      p.event_track_hits[e] = s.track_hits + 3 * filter_count;
    }
  }

  // One instantiation per (block size, lanes per seed, ring place); the chain launches the one
  // its launch configuration names (autotuned).  Events whose hits fit the shared-memory
  // capacity run the shared-memory body, the others the global-scratch body.  The ring of
  // tracks to follow (2048 entries, 16 KiB) sits in shared memory, or with RING = 1 in this
  // CTA's slice of a global scratch (persistent launches only: the slice is the CTA's index),
  // which leaves room for more resident CTAs per SM.
  // Flat-seeding kernels are register-capped for 1536 threads per SM (40 registers, a few
  // spills): with the hits and the ring staged through L2 shared memory no longer limits the
  // CTAs per SM, and the extra resident events hide more latency than the spills cost
  // (measured per 16000-event launch: 5.87 / 5.72 ms at five / six 256-thread CTAs, 3.94 ms at
  // twelve 128-thread CTAs; sixteen at 32 registers, 4.13 ms).
  template<unsigned THREADS, unsigned LPH, unsigned RING>
  __global__ void __launch_bounds__(THREADS, LPH == 0 ? 1536 / THREADS : 1) search_by_triplet_kernel(SearchParams p)
  {
    extern __shared__ __align__(128) unsigned char dsmem[];
    __shared__ std::conditional_t<LPH == 0, SearchSharedFlatPlain<THREADS>, SearchShared> s;
    __shared__ uint64_t ring_smem[RING ? 1 : max_tracks_to_follow];
    uint64_t* ring = RING ? p.ring_scratch + size_t(blockIdx.x) * max_tracks_to_follow : ring_smem;
    for_each_event(p.queue, p.n_events, [&](unsigned e, unsigned) {
      const unsigned* start = p.offsets_estimated_input_size + e * n_module_pairs;
      const unsigned n_hits = start[n_module_pairs] - start[0];
      if (n_hits <= p.smem_hit_capacity) search_event<LPH, true, false>(p, s, ring, dsmem, e);
      else search_event<LPH, false, false>(p, s, ring, dsmem, e);
    });
  }

  // The learned search (flat seeding with the seed pruner; with seed_model null, the plain
  // search, recording training doublets when asked) is a kernel of its own, so the plain
  // kernels keep their register budget.
  template<unsigned THREADS, unsigned RING>
  __global__ void __launch_bounds__(THREADS, 1024 / THREADS) search_by_triplet_learned_kernel(SearchParams p)
  {
    extern __shared__ __align__(128) unsigned char dsmem[];
    __shared__ SearchSharedFlat s;
    __shared__ uint64_t ring_smem[RING ? 1 : max_tracks_to_follow];
    uint64_t* ring = RING ? p.ring_scratch + size_t(blockIdx.x) * max_tracks_to_follow : ring_smem;
    for_each_event(p.queue, p.n_events, [&](unsigned e, unsigned) {
      const unsigned* start = p.offsets_estimated_input_size + e * n_module_pairs;
      const unsigned n_hits = start[n_module_pairs] - start[0];
      if (n_hits <= p.smem_hit_capacity) search_event<0, true, true>(p, s, ring, dsmem, e);
      else search_event<0, false, true>(p, s, ring, dsmem, e);
    });
  }

#define VELO_SEARCH_CONFIG(T, L, R)                                              \
  template __global__ void search_by_triplet_kernel<T, L, R>(SearchParams p);
  VELO_SEARCH_CONFIGS(VELO_SEARCH_CONFIG)
#undef VELO_SEARCH_CONFIG
  template __global__ void search_by_triplet_learned_kernel<128, 0>(SearchParams p);
  template __global__ void search_by_triplet_learned_kernel<256, 0>(SearchParams p);
  template __global__ void search_by_triplet_learned_kernel<512, 0>(SearchParams p);
  template __global__ void search_by_triplet_learned_kernel<128, 1>(SearchParams p);
  template __global__ void search_by_triplet_learned_kernel<256, 1>(SearchParams p);

} // namespace velo
