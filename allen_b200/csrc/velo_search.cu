// search_by_triplet (seeding + forwarding) and the three-hit filter on sm_100a,
// one event per CTA.
//
// Reference: device/velo/search_by_triplet/src/SearchByTriplet.cu:110-609 (kernel,
// find_forward_candidate, track_seeding, track_forwarding) and
// ThreeHitTracksFilter.cu:48-169.
//
// Design.
//  * The event's sorted hits are staged once as 16-byte records (x, y, z, phi and a flag
//    byte holding hit_used and the module parity that forwarding needs), so that every
//    hit a walk visits costs one vector load: in shared memory, or for events above the
//    shared-memory capacity (and in the tuned launch, every event) in a global scratch
//    slice that stays in L2, through the same code.
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
  constexpr uint8_t flag_used = 1;
  constexpr uint8_t flag_odd_module = 2;
  constexpr unsigned flat_slots = 1024; // (h1, h0 candidate) slots per chunk of the flat seeding
  constexpr unsigned pendulum_capacity = 512; // module pairs of up to this many hits get the unused-hit index

  struct ModulePair {
    unsigned hit_start;
    unsigned hit_num;
    float z[2];
    unsigned table; // slot of its bucket table: the module pair's index % 3
  };

  struct SearchShared {
    alignas(16) unsigned scan_sums[2][32]; // double-buffered warp totals of the block scans (0 past the last warp)
    unsigned track_hits;       // sum of hitsNum over the >= 4 hit tracks
    // counters only reported (thread 0 keeps them): atomics::local_number_of_hits, the unused
    // h1 met by the seeding (seed candidates), the candidates whose h0 and h2 windows were
    // searched (the gate let through)
    unsigned local_hits, candidates, searched;
    uint32_t tail[max_tail_tracks]; // last two hits of a track (hit[n-2] | hit[n-1] << 16)
    uint8_t tail_n[max_tail_tracks];
    // bucket tables of the three module pairs a step reads, built one per step
    uint16_t bucket[3][n_buckets + 1];
    // the event's module pairs, last first: a step's three are mps[25 - first] onwards
    ModulePair mps[n_module_pairs];
  };

  // Shared state of the flat seeding variant: one slot per (h1, candidate order).
  template<unsigned SLOTS>
  struct SearchSharedFlatBase : SearchShared {
    static constexpr unsigned slots = SLOTS;
    // (h0, h1) doublets of a chunk, packed by pack_doublet(), then overwritten in place
    // with the best scatter found for the doublet
    union {
      uint32_t doublet;
      float fit;
    } slot[SLOTS];
    uint16_t res_h2[SLOTS];
    // The unused hits of the seeding's previous module pair: how many lie before each
    // position (the last entry: all of them), and their positions in phi order
    uint16_t unused_before[pendulum_capacity + 1];
    uint16_t unused_at[pendulum_capacity];
  };
  template<unsigned SLOTS, bool GATED>
  struct SearchSharedFlatT : SearchSharedFlatBase<SLOTS> {};
  template<unsigned SLOTS>
  struct SearchSharedFlatT<SLOTS, true> : SearchSharedFlatBase<SLOTS> {
    uint16_t cand_list[SLOTS]; // the window's searched candidates (index in the window), h1 order
  };
  // flat-seeding kernels: 512 slots for 128 threads (chunks of 64 or 128 h1), which with the
  // ring in global scratch leaves room for sixteen CTAs per SM
  template<unsigned THREADS, bool GATED = false>
  using SearchSharedFlatPlain =
    SearchSharedFlatT<(THREADS <= 64 ? flat_slots / 4 : (THREADS <= 128 ? flat_slots / 2 : flat_slots)), GATED>;

  // Packed doublet: h0 | h1 index in the chunk << 16 | rank << 25 | (found - 1) << 28
  __device__ __forceinline__ uint32_t pack_doublet(unsigned h0, unsigned h1_local, unsigned rank, unsigned found)
  {
    return h0 | (h1_local << 16) | (rank << 25) | ((found - 1u) << 28);
  }

  // A staged hit, unpacked from its 16-byte record.
  struct Hit {
    float x, y, z;
    int16_t phi;
    unsigned flags;
  };

  // The event's staged hits: one 16-byte record per hit (x, y, z as fp32 bits, then phi in
  // bits 0-15 and the flags in bits 16-23 of the fourth word), so that a candidate costs
  // one vector load instead of one load per field.
  struct Hits {
    uint4* r;
    __device__ __forceinline__ Hit operator[](unsigned i) const
    {
      const uint4 v = r[i];
      return Hit {__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z), static_cast<int16_t>(v.w & 0xFFFFu),
                  (v.w >> 16) & 0xFFu};
    }
    __device__ __forceinline__ int16_t phi(unsigned i) const { return reinterpret_cast<const int16_t*>(r + i)[6]; }
    __device__ __forceinline__ unsigned flags(unsigned i) const { return reinterpret_cast<const uint8_t*>(r + i)[14]; }
    __device__ __forceinline__ void mark_used(unsigned i) const { reinterpret_cast<uint8_t*>(r + i)[14] |= flag_used; }
  };

  // Position i < n of the pendulum around p0 in [0, n]: p0, p0 + 1, p0 - 1, p0 + 2, ...
  // with one wrap (SearchByTriplet.cu:351-370).
  __device__ __forceinline__ unsigned pendulum(int p0, unsigned i, int n)
  {
    const int pos = p0 + ((i & 1u) ? static_cast<int>((i + 1) / 2) : -static_cast<int>(i / 2));
    return static_cast<unsigned>(pos < 0 ? pos + n : (pos >= n ? pos - n : pos));
  }

  // The first h2 of the circular window walk: start % n (0 for an empty module pair), without
  // a division for start in [0, n], leftmost()'s range.
  __device__ __forceinline__ unsigned first_candidate(int16_t start, unsigned n)
  {
    const unsigned x = static_cast<unsigned>(start);
    return x < n ? x : (x == n || n == 0 ? 0u : x % n);
  }

  // leftmost() over the staged hits [start, start + n) of a module pair.
  __device__ __forceinline__ int leftmost_hit(const uint16_t* table, const Hits& h, unsigned start, unsigned n, int16_t value)
  {
    unsigned i = table[bucket_of(value)];
    while (i < n && h.phi(start + i) < value)
      ++i;
    return static_cast<int>(i);
  }

  // The event's counters that place items (the reference's dev_atomics_velo and track
  // count), kept in registers: every thread holds the same values and advances them by scan
  // totals.
  struct Counters {
    unsigned ttf;      // atomics::tracks_to_follow
    unsigned n_three;  // atomics::number_of_three_hit_tracks
    unsigned n_tracks; // dev_number_of_velo_tracks
    unsigned scan_parity;
  };

  // The block-wide part of an exclusive scan, with a single barrier: warp totals go to one
  // of two buffers, alternating per call, so a call never overwrites totals still being
  // read.  incl: the warp-inclusive sum of v.
  __device__ __forceinline__ unsigned scan_block(SearchShared& s, Counters& c, unsigned incl, unsigned v, unsigned& total)
  {
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    unsigned* buf = s.scan_sums[c.scan_parity];
    c.scan_parity ^= 1u;
    if (lane == 31) buf[warp] = incl;
    __syncthreads();
    unsigned before = 0, all = 0;
    if (n_warps <= 4) { // one vector read of the four totals (those past the last warp stay 0)
      const uint4 t = *reinterpret_cast<const uint4*>(buf);
      all = t.x + t.y + t.z + t.w;
      before = (warp > 0 ? t.x : 0u) + (warp > 1 ? t.y : 0u) + (warp > 2 ? t.z : 0u);
    }
    else {
      for (unsigned w = 0; w < n_warps; ++w) {
        const unsigned t = buf[w];
        before += w < warp ? t : 0u;
        all += t;
      }
    }
    total = all;
    return before + incl - v;
  }

  // Block-wide exclusive scan of v (every thread of the block calls it).
  __device__ __forceinline__ unsigned scan1(SearchShared& s, Counters& c, unsigned v, unsigned& total)
  {
    const unsigned lane = threadIdx.x & 31u;
    unsigned incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= static_cast<unsigned>(o)) incl += t;
    }
    return scan_block(s, c, incl, v, total);
  }

  // scan1() of up to three 0/1 flags packed at bits 0, S1 and S2 (each field wide enough for
  // a block total), the warp part by ballots.
  template<unsigned NF, unsigned S1 = 16, unsigned S2 = 32>
  __device__ __forceinline__ unsigned scan_flags(SearchShared& s, Counters& c, bool f0, bool f1, bool f2, unsigned& total)
  {
    const unsigned le = 0xFFFFFFFFu >> (31u - (threadIdx.x & 31u)); // this lane and those below
    unsigned incl = __popc(__ballot_sync(0xFFFFFFFFu, f0) & le);
    unsigned v = f0 ? 1u : 0u;
    if constexpr (NF > 1) {
      incl |= static_cast<unsigned>(__popc(__ballot_sync(0xFFFFFFFFu, f1) & le)) << S1;
      v |= (f1 ? 1u : 0u) << S1;
    }
    if constexpr (NF > 2) {
      incl |= static_cast<unsigned>(__popc(__ballot_sync(0xFFFFFFFFu, f2) & le)) << S2;
      v |= (f2 ? 1u : 0u) << S2;
    }
    return scan_block(s, c, incl, v, total);
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
    const Hits& h,
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
    x.start = static_cast<int16_t>(leftmost_hit(s.bucket[next.table], h, next.hit_start, next.hit_num, lo));
    return x;
  }

  // One h0 candidate of a seed (SearchByTriplet.cu:374-432): updates (best_fit, best_c,
  // best_h0, best_h2) with strict improvement, in window order.
  __device__ __forceinline__ void seed_candidate(
    const Constants& k,
    const SearchShared& s,
    const Hits& h,
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
    const Hit a = h[h0];
    const float h0x = a.x, h0y = a.y, h0z = a.z;
    const float td = __fdiv_rn(1.0f, h1z - h0z);
    const float txn = h1x - h0x;
    const float tyn = h1y - h0y;
    const float tx = txn * td;
    const float ty = tyn * td;
    const Extrapolation f = extrapolate(k, s, h, next, h0x, h0y, tx, ty, next.z[0] - prev.z[0]);
    // circular walk from the candidate: index (start + j) % n without a division per step
    unsigned idx = first_candidate(f.start, next.hit_num);
    for (unsigned j = 0; j < next.hit_num; ++j, idx = (idx + 1 == next.hit_num) ? 0u : idx + 1) {
      const unsigned h2 = next.hit_start + idx;
      const Hit b = h[h2];
      if (phi_outside(b.phi, f.phi, tol)) break;
      if (b.flags & flag_used) continue;
      const float dz = b.z - h0z;
      const float predx = h0x + tx * dz;
      const float predy = h0y + ty * dz;
      const float dx = predx - b.x;
      const float dy = predy - b.y;
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
    SearchShared& s, uint64_t* ring, Counters& cnt, const Constants& k, const Hits& h, const ModulePair* md,
    unsigned n_candidates)
  {
    const ModulePair &prev = md[0], &cur = md[1], &next = md[2];
    const unsigned groups = blockDim.x / LPH;
    const unsigned g = threadIdx.x / LPH;
    const unsigned l = threadIdx.x % LPH;
    const unsigned lane0 = (threadIdx.x & 31u) & ~(LPH - 1);
    const unsigned gmask = (LPH == 32 ? 0xFFFFFFFFu : ((1u << LPH) - 1u)) << lane0;
    for (unsigned c0 = 0; c0 < cur.hit_num; c0 += groups) {
      const unsigned r = c0 + g;
      const unsigned h1 = cur.hit_start + r;
      const bool valid = r < cur.hit_num && !(h.flags(h1) & flag_used);
      float best_fit = k.max_scatter;
      unsigned best_c = 0xFFFFFFFFu, best_h0 = 0, best_h2 = 0;
      if (valid) {
        const Hit b = h[h1];
        const float h1x = b.x, h1y = b.y, h1z = b.z;
        const int p0 = leftmost_hit(s.bucket[prev.table], h, prev.hit_start, prev.hit_num, b.phi);
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
            ok = !(h.flags(h0) & flag_used);
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
      const unsigned excl = scan_flags<2>(s, cnt, ok, unused != 0, false, total);
      if (ok) {
        const unsigned tn = (cnt.ttf + (excl & 0xFFFFu)) % max_tracks_to_follow;
        ring[tn] = seed_flag | (uint64_t(best_h0 & 0xFFFFu)) | (uint64_t(h1 & 0xFFFFu) << 16) |
                     (uint64_t(best_h2 & 0xFFFFu) << 32);
      }
      cnt.ttf += total & 0xFFFFu;
      if (threadIdx.x == 0) s.local_hits += total >> 16;
    }
  }

  __device__ __forceinline__ unsigned candidate_h0(uint64_t lo, uint64_t hi, unsigned c)
  {
    return static_cast<unsigned>((c < 4 ? lo >> (16 * c) : hi >> (16 * (c - 4))) & 0xFFFFu);
  }

  // Seeding with the candidates flattened (SearchByTriplet.cu:298-446).  The window's unused
  // h1 are first compacted to threads 0, 1, ... in h1 order.  Phase A, one thread per h1,
  // walks the pendulum and keeps its first n_candidates unused h0 in registers; a block scan
  // packs all (h0, h1) doublets of the chunk into one list.
  // Phase B, one thread per doublet, extrapolates and scans the h2 window.  Phase C, one
  // thread per h1, keeps the first strictly best of its doublets in candidate order (the
  // reference's sequential choice) and queues the seed in h1 order.  Phase B runs the same
  // path on every lane and has no idle slots for h1 with fewer than n_candidates doublets.
  // GATED kernels take the learned seed gate (gate, event-relative, or null): an unused h1
  // whose gate byte is 0 is not searched; and, for training, record each unused h1's
  // outcome (outcome: 1 no seed, 2 seed; null = off).
  template<bool GATED, typename Flat>
  __device__ __forceinline__ void seeding_flat(
    Flat& s,
    uint64_t* ring,
    Counters& cnt,
    const Constants& k,
    const Hits& h,
    const ModulePair* md,
    unsigned n_candidates,
    const uint8_t* gate,
    uint8_t* outcome)
  {
    const ModulePair &prev = md[0], &cur = md[1], &next = md[2];
    const unsigned per_chunk = min(blockDim.x, Flat::slots / n_candidates);
    const int n_prev = static_cast<int>(prev.hit_num);
    const int16_t tol = static_cast<int16_t>(k.phi_tolerance_i16);
    // The unused-hit index of the previous module pair (its used flags do not change
    // during the seeding), when a module pair has hits to seed and fits the index
    const bool indexed = cur.hit_num > 0 && prev.hit_num <= pendulum_capacity;
    unsigned n_unused = 0;
    if (indexed) {
      for (unsigned i0 = 0; i0 < prev.hit_num; i0 += blockDim.x) {
        const unsigned i = i0 + threadIdx.x;
        const bool unused = i < prev.hit_num && !(h.flags(prev.hit_start + i) & flag_used);
        unsigned total;
        const unsigned before = n_unused + scan_flags<1>(s, cnt, unused, false, false, total);
        if (i < prev.hit_num) s.unused_before[i] = static_cast<uint16_t>(before);
        if (unused) s.unused_at[before] = static_cast<uint16_t>(i);
        n_unused += total;
      }
      if (threadIdx.x == 0) s.unused_before[prev.hit_num] = static_cast<uint16_t>(n_unused);
      __syncthreads();
    }
    for (unsigned c0 = 0; c0 < cur.hit_num; c0 += per_chunk) {
      const unsigned n_h1 = min(per_chunk, cur.hit_num - c0);
      // Gated: the window's candidates compacted in h1 order (its unused hits that the gate
      // lets through, one per thread from thread 0 on), so that the phases below run on as
      // few warps as there are candidates.  Plain: thread i takes the window's hit i (the
      // compaction's scan and barrier cost the plain search more than they save).
      bool searched;
      unsigned hl;
      if constexpr (GATED) {
        unsigned n_searched;
        {
          const unsigned hw = cur.hit_start + c0 + threadIdx.x;
          const bool valid = threadIdx.x < n_h1 && !(h.flags(hw) & flag_used);
          const bool pass = valid && (gate == nullptr || gate[hw] != 0);
          unsigned total;
          const unsigned excl = scan_flags<2>(s, cnt, pass, valid, false, total);
          if (pass) s.cand_list[excl & 0xFFFFu] = static_cast<uint16_t>(threadIdx.x);
          n_searched = total & 0xFFFFu;
          if (threadIdx.x == 0) {
            s.local_hits += total >> 16;
            s.candidates += total >> 16;
            s.searched += n_searched;
          }
        }
        __syncthreads();
        searched = threadIdx.x < n_searched;
        hl = searched ? s.cand_list[threadIdx.x] : 0u;
      }
      else {
        hl = threadIdx.x;
        searched = threadIdx.x < n_h1 && !(h.flags(cur.hit_start + c0 + hl) & flag_used);
      }
      const unsigned h1 = cur.hit_start + c0 + hl;
      // Phase A: candidates c < 4 in the 16-bit fields of cand_lo, 4..7 in cand_hi, the first
      // n_candidates unused h0 of the pendulum p0, p0 + 1, p0 - 1, p0 + 2, ... (one wrap).
      // With the unused-hit index, the pendulum's unused hits are the merge of the index's
      // run from p0 upwards (pendulum step 2d - 1 at offset d > 0, 0 at p0) and its run below
      // p0 (step 2d at offset d), each wrapping once, taken while the step is below n.
      uint64_t cand_lo = 0, cand_hi = 0;
      unsigned found = 0;
      if (searched) {
        const int p0 = leftmost_hit(s.bucket[prev.table], h, prev.hit_start, prev.hit_num, h.phi(h1));
        if (indexed) {
          const int u = static_cast<int>(n_unused);
          const int r = s.unused_before[p0];
          // step and position of the k-th unused hit upwards (k >= r) and downwards (k < r)
          auto up = [&](int kk, unsigned& pos) {
            if (kk >= 2 * u) return static_cast<unsigned>(n_prev);
            const int q = s.unused_at[kk < u ? kk : kk - u];
            pos = static_cast<unsigned>(q);
            const int d = (kk < u ? q : q + n_prev) - p0;
            return d == 0 ? 0u : static_cast<unsigned>(2 * d - 1);
          };
          auto down = [&](int kk, unsigned& pos) {
            if (kk < -u) return static_cast<unsigned>(n_prev);
            const int q = s.unused_at[kk >= 0 ? kk : kk + u];
            pos = static_cast<unsigned>(q);
            return static_cast<unsigned>(2 * (p0 - (kk >= 0 ? q : q - n_prev)));
          };
          int ku = r, kd = r - 1;
          unsigned pu = 0, pd = 0;
          unsigned iu = up(ku, pu), id = down(kd, pd);
          while (found < n_candidates) {
            const bool upward = iu < id;
            if ((upward ? iu : id) >= prev.hit_num) break;
            const unsigned h0 = prev.hit_start + (upward ? pu : pd);
            if (found < 4) cand_lo |= uint64_t(h0) << (16 * found);
            else cand_hi |= uint64_t(h0) << (16 * (found - 4));
            ++found;
            if (upward) iu = up(++ku, pu);
            else id = down(--kd, pd);
          }
        }
        else {
          for (unsigned i = 0; i < prev.hit_num && found < n_candidates; ++i) {
            const unsigned h0 = prev.hit_start + pendulum(p0, i, n_prev);
            if (!(h.flags(h0) & flag_used)) {
              if (found < 4) cand_lo |= uint64_t(h0) << (16 * found);
              else cand_hi |= uint64_t(h0) << (16 * (found - 4));
              ++found;
            }
          }
        }
      }
      unsigned n_doublets;
      const unsigned first = scan1(s, cnt, found, n_doublets);
      for (unsigned c = 0; c < found; ++c)
        s.slot[first + c].doublet = pack_doublet(candidate_h0(cand_lo, cand_hi, c), hl, c, found);
      __syncthreads();
      // keep_mask bit c: doublet c's slot in the packed list (every doublet is scanned)
      const unsigned keep_mask = (1u << found) - 1u;
      // Phase B
      for (unsigned q = threadIdx.x; q < n_doublets; q += blockDim.x) {
        const uint32_t d = s.slot[q].doublet;
        const unsigned h0 = d & 0xFFFFu;
        const unsigned hh1 = cur.hit_start + c0 + ((d >> 16) & 0x1FFu);
        float best_fit = k.max_scatter;
        unsigned best_h2 = 0xFFFFu;
        const Hit a = h[h0], b = h[hh1];
        const float h1x = b.x, h1y = b.y, h1z = b.z;
        const float h0x = a.x, h0y = a.y, h0z = a.z;
        const float td = __fdiv_rn(1.0f, h1z - h0z);
        const float txn = h1x - h0x;
        const float tyn = h1y - h0y;
        const float tx = txn * td;
        const float ty = tyn * td;
        const Extrapolation f = extrapolate(k, s, h, next, h0x, h0y, tx, ty, next.z[0] - prev.z[0]);
        unsigned idx = first_candidate(f.start, next.hit_num);
        for (unsigned j = 0; j < next.hit_num; ++j, idx = (idx + 1 == next.hit_num) ? 0u : idx + 1) {
          const unsigned h2 = next.hit_start + idx;
          const Hit c = h[h2];
          if (phi_outside(c.phi, f.phi, tol)) break;
          if (c.flags & flag_used) continue;
          const float dz = c.z - h0z;
          const float predx = h0x + tx * dz;
          const float predy = h0y + ty * dz;
          const float dx = predx - c.x;
          const float dy = predy - c.y;
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
      if (searched) {
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
        if (GATED && outcome != nullptr) outcome[h1] = ok ? 2 : 1;
      }
      unsigned total;
      const unsigned excl = scan_flags<GATED ? 1 : 2>(s, cnt, ok, !GATED && searched, false, total);
      if (ok) {
        const unsigned tn = (cnt.ttf + (excl & 0xFFFFu)) % max_tracks_to_follow;
        ring[tn] = seed_flag | (uint64_t(best_h0 & 0xFFFFu)) | (uint64_t(h1 & 0xFFFFu) << 16) |
                     (uint64_t(best_h2 & 0xFFFFu) << 32);
      }
      cnt.ttf += total & 0xFFFFu;
      if (!GATED && threadIdx.x == 0) {
        s.local_hits += total >> 16;
        s.candidates += total >> 16;
        s.searched += total >> 16;
      }
    }
  }

  // Forwarding of the tracks to follow (SearchByTriplet.cu:451-609), one thread per track.
  __device__ __forceinline__ void forwarding(
    SearchShared& s,
    uint64_t* ring,
    Counters& cnt,
    const Constants& k,
    const Hits& h,
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
        const Hit a = h[h0n], b = h[h1n];
        const float h0x = a.x, h0y = a.y, h0z = a.z;
        const unsigned odd = (a.flags & flag_odd_module) ? 1u : 0u;
        const float h1x = b.x, h1y = b.y, h1z = b.z;
        const float td = __fdiv_rn(1.0f, h1z - h0z);
        const float txn = h1x - h0x;
        const float tyn = h1y - h0y;
        const float tx = txn * td;
        const float ty = tyn * td;
        float best_fit = k.max_scatter;
        const Extrapolation f = extrapolate(k, s, h, next, h0x, h0y, tx, ty, next.z[odd] - h0z);
        unsigned idx = first_candidate(f.start, next.hit_num);
        for (unsigned j = 0; j < next.hit_num; ++j, idx = (idx + 1 == next.hit_num) ? 0u : idx + 1) {
          const unsigned h2 = next.hit_start + idx;
          const Hit c = h[h2];
          if (phi_outside(c.phi, f.phi, tol)) break;
          const float dz = c.z - h0z;
          const float predx = h0x + tx * dz;
          const float predy = h0y + ty * dz;
          const float dx = predx - c.x;
          const float dy = predy - c.y;
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
        scan_flags<3, 10, 20>(s, cnt, new_track, enqueue, three, total);
      if (active) {
        unsigned track_number = tn;
        if (found) {
          h.mark_used(best_h2);
          if (is_seed) {
            const unsigned t0 = static_cast<unsigned>(entry) & 0xFFFFu;
            h.mark_used(t0);
            h.mark_used(h0n);
            h.mark_used(h1n);
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
  __device__ __forceinline__ float means_square_fit_chi2(const Hit (&r)[3])
  {
    const float w = 6400.f;
    float s0, sx, sz, sxz, sz2, u0, uy, uz, uyz, uz2;
    s0 = sx = sz = sxz = sz2 = 0.0f;
    u0 = uy = uz = uyz = uz2 = 0.0f;
#pragma unroll
    for (unsigned i = 0; i < 3; ++i) {
      const float x = r[i].x, y = r[i].y, z = r[i].z;
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
      const float z = r[i].z;
      const float x = state_x + state_tx * z;
      const float y = state_y + state_ty * z;
      const float dx = x - r[i].x;
      const float dy = y - r[i].y;
      chi2 += dx * dx * w + dy * dy * w;
    }
    return chi2 * 0.5f;
  }

  // The three module pairs of a step (first, first - 1, first - 2), read by every thread.
  // The event's module pairs into shared memory, last first (threads 0-25; a barrier follows).
  __device__ __forceinline__ void module_pairs(
    ModulePair* mps, const Geometry* g, const unsigned* start, const unsigned* num, unsigned hit_offset)
  {
    const unsigned mp = threadIdx.x;
    if (mp < n_module_pairs) {
      ModulePair& m = mps[n_module_pairs - 1 - mp];
      m.hit_start = start[mp] - hit_offset;
      m.hit_num = num[mp];
      m.z[0] = __ldg(g->module_zs + 2 * mp);
      m.z[1] = __ldg(g->module_zs + 2 * mp + 1);
      m.table = mp % 3;
    }
  }

  // Seeding, forwarding and the tail of one event over staged hits (hit_used clear):
  // SearchByTriplet.cu:165-264.  Returns the event's counters; the track containers hold
  // its tracks and three-hit tracks.
  template<unsigned LPH, bool GATED, typename Shared>
  __device__ __forceinline__ Counters search_pass(
    const SearchParams& p,
    Shared& s,
    uint64_t* ring,
    const Constants& k,
    const Hits& h,
    const unsigned* start,
    const unsigned* num,
    unsigned hit_offset,
    TrackHits* tracks,
    unsigned track_limit,
    TrackletHits* three_hit,
    const uint8_t* gate,
    uint8_t* outcome)
  {
    if (threadIdx.x == 0) s.track_hits = s.candidates = s.searched = 0;
    if (threadIdx.x < 64) s.scan_sums[threadIdx.x >> 5][threadIdx.x & 31u] = 0;
    Counters cnt {0, 0, 0, 0};
    module_pairs(s.mps, p.geo, start, num, hit_offset);
    __syncthreads();
    unsigned first = n_module_pairs - 1;
    const ModulePair* md = s.mps;
    for (unsigned i = 0; i < 2; ++i)
      build_bucket_table_of(s.bucket[md[i].table], [h](unsigned j) { return h.phi(j); }, md[i].hit_start, md[i].hit_num);

    // One step per module pair first = 25 ... 2 (the first without forwarding), with a single
    // copy of the seeding code.
    unsigned last_ttf = 0;
    const unsigned window = GATED && gate != nullptr && p.seed_window ? p.seed_window : 4u;
    for (;;) {
      // the table of module pair first - 2 replaces that of first + 1, last read by the
      // previous step's seeding
      build_bucket_table_of(s.bucket[md[2].table], [h](unsigned j) { return h.phi(j); }, md[2].hit_start, md[2].hit_num);
      const bool forward = first < n_module_pairs - 1;
      const unsigned prev_ttf = last_ttf;
      if (forward) last_ttf = cnt.ttf;
      if (threadIdx.x == 0) s.local_hits = 0;
      __syncthreads(); // ring entries of the last seeding, the new bucket table
      if (forward) {
        forwarding(s, ring, cnt, k, h, md[2], prev_ttf, last_ttf - prev_ttf, tracks, track_limit, three_hit, p.status);
        // The ring holds 2048 entries; beyond that the reference overwrites entries it has
        // not read yet, an order-dependent outcome this kernel does not reproduce.
        if (threadIdx.x == 0 && cnt.ttf - prev_ttf > max_tracks_to_follow) set_error(p.status, err_ttf_overflow);
        __syncthreads(); // hit_used flags written by forwarding
      }
      if constexpr (LPH == 0) seeding_flat<GATED>(s, ring, cnt, k, h, md, forward ? window : 8u, gate, outcome);
      else seeding<LPH>(s, ring, cnt, k, h, md, forward ? 4u : 8u);
      if (forward && threadIdx.x == 0 && cnt.ttf - last_ttf > max_tracks_to_follow) set_error(p.status, err_ttf_overflow);
      if (--first <= 1) break;
      ++md;
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
        const unsigned excl = scan_flags<1>(s, cnt, seed, false, false, total);
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

  template<unsigned LPH, bool SMEM, bool GATED, typename Shared>
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

    // Stage the hits as 16-byte records: shared memory when they fit (SMEM), else the
    // event's global slice (16 bytes per estimated hit).
    const Hits h {SMEM ? reinterpret_cast<uint4*>(dsmem) : reinterpret_cast<uint4*>(p.hit_scratch) + hit_offset};
    {
      const ClusterView g {const_cast<char*>(p.sorted_container), T};
      // read once: streaming loads (evict first), which leave L2 to the staged hits
      for (unsigned i = threadIdx.x; i < n_hits; i += blockDim.x) {
        const unsigned gi = hit_offset + i;
        const unsigned module = ((__ldcs(&g.id(gi)) & 0x3FC0000u) >> 18) / 4;
        const unsigned flags = (module & 1u) ? flag_odd_module : 0u;
        h.r[i] = make_uint4(__float_as_uint(__ldcs(&g.x(gi))), __float_as_uint(__ldcs(&g.y(gi))),
                            __float_as_uint(__ldcs(&g.z(gi))), static_cast<uint16_t>(__ldcs(&g.phi(gi))) | (flags << 16));
      }
    }

    // Learned mode: the gate of the event's seed candidates, unless the fraction it lets
    // through falls outside the model's bounds, in which case the plain search runs
    unsigned mode = seed_mode_plain;
    const uint8_t* gate = nullptr;
    if (GATED && p.seed_gate != nullptr) {
      const unsigned cand = p.gate_stats[2 * e], kept = p.gate_stats[2 * e + 1];
      const float frac = cand > 0 ? __fdiv_rn(__uint2float_rn(kept), __uint2float_rn(cand)) : 1.0f;
      if (frac >= p.kept_lo && frac <= p.kept_hi) {
        gate = p.seed_gate + hit_offset;
        mode = seed_mode_learned;
      }
      else {
        mode = seed_mode_fallback;
      }
    }
    uint8_t* outcome = GATED && p.h1_outcome != nullptr ? p.h1_outcome + hit_offset : nullptr;
    Counters cnt =
      search_pass<LPH, GATED>(p, s, ring, k, h, start, num, hit_offset, tracks, track_limit, three_hit, gate, outcome);
    if (p.seed_stats != nullptr && threadIdx.x == 0) {
      p.seed_stats[3 * e] = s.candidates;
      p.seed_stats[3 * e + 1] = s.searched;
      p.seed_stats[3 * e + 2] = mode;
    }

    if (threadIdx.x == 0) {
      unsigned* atomics = p.atomics_velo + 3 * e;
      atomics[0] = cnt.n_three;
      atomics[1] = cnt.ttf;
      atomics[2] = s.local_hits;
      p.number_of_velo_tracks[e] = cnt.n_tracks;
      if (cnt.n_tracks > to_next - to) set_error(p.status, err_track_capacity);
    }
    {
      uint8_t* g_used = reinterpret_cast<uint8_t*>(p.hit_used) + hit_offset;
      for (unsigned i = threadIdx.x; i < n_hits; i += blockDim.x)
        g_used[i] = h.flags(i) & flag_used;
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
        const Hit r[3] = {h[t.hits[0]], h[t.hits[1]], h[t.hits[2]]};
        const bool any_used = ((r[0].flags | r[1].flags | r[2].flags) & flag_used) != 0;
        const float chi2 = means_square_fit_chi2(r);
        keep = !any_used && chi2 < k.max_chi2;
      }
      unsigned total;
      const unsigned excl = scan_flags<1>(s, cnt, keep, false, false, total);
      if (keep) out[filter_count + excl] = t;
      filter_count += total;
    }
    if (threadIdx.x == 0) {
      p.number_of_three_hit_tracks_output[e] = filter_count;
      p.event_track_hits[e] = s.track_hits + 3 * filter_count;
    }
    // the staged hits are dead (the filter's last scan is a barrier after the last read)
    if (!SMEM) discard_l2(h.r, size_t(16) * n_hits);
  }

  // One instantiation per (block size, lanes per seed, ring place); the chain launches the one
  // its launch configuration names (autotuned).  Events whose hits fit the shared-memory
  // capacity run the shared-memory body, the others the global-scratch body.  The ring of
  // tracks to follow (2048 entries, 16 KiB) sits in shared memory, or with RING = 1 in this
  // CTA's slice of a global scratch (persistent launches only: the slice is the CTA's index),
  // which leaves room for more resident CTAs per SM.
  // Flat-seeding kernels are register-capped for 2048 threads per SM (32 registers, some
  // spills): with the hits and the ring staged through L2 shared memory no longer limits the
  // CTAs per SM, and the extra resident events hide more latency than the spills cost
  // (measured per 16000-event launch: 4.01 ms at twelve 128-thread CTAs and 40 registers,
  // 3.83 ms at sixteen and 32 registers; the smaller the shared-memory footprint, the larger
  // the L1 that caches the hit records).
  template<unsigned THREADS, unsigned LPH, unsigned RING>
  __global__ void __launch_bounds__(THREADS, LPH == 0 ? 2048 / THREADS : 1) search_by_triplet_kernel(SearchParams p)
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

  // The learned search: flat seeding behind the seed gate (with seed_gate null, the plain
  // search, recording each seed candidate's outcome when h1_outcome is set).  The gate costs
  // one byte read per candidate, so this kernel keeps the plain kernel's register budget.
  template<unsigned THREADS, unsigned RING>
  __global__ void __launch_bounds__(THREADS, 2048 / THREADS) search_by_triplet_gated_kernel(SearchParams p)
  {
    extern __shared__ __align__(128) unsigned char dsmem[];
    __shared__ SearchSharedFlatPlain<THREADS, true> s;
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
#define VELO_GATED_CONFIG(T, R) template __global__ void search_by_triplet_gated_kernel<T, R>(SearchParams p);
  VELO_GATED_CONFIGS(VELO_GATED_CONFIG)
#undef VELO_GATED_CONFIG

} // namespace velo
