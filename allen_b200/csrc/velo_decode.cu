// VELO super-pixel decoding on sm_100a: candidate counting and input-size estimate
// (velo_calculate_number_of_candidates + velo_estimate_input_size), masked clustering,
// phi and the sort by phi (velo_masked_clustering + velo_sort_by_phi), one event per CTA.
//
// A CTA reads its event's raw blob (bank offsets + SP words) through L1/L2, or stages it
// into shared memory with one bulk copy through the TMA engine (cp.async.bulk, 16-byte
// aligned span, the ragged tail by plain loads) when the launch configuration gives it room.
// The O(n_sp^2) neighbour scans of the reference (EstimateInputSize.cu:111-141,
// MaskedVeloClustering.cu:361-402) become binary-searched key ranges of key-sorted bank
// copies, which the estimate kernel writes once per event and the clustering kernel reuses.
// Work is spread one thread per super pixel over the flattened bank list.
//
// The sorted container is independent of the order in which clusters are produced
// (rank by (phi, id), SortByPhi.cu:104-122), so clusters are appended to their module
// pair with shared-memory atomics and ranked in place; no unsorted container is written.
#include "velo_kernels.cuh"

namespace velo {

  constexpr unsigned max_banks = 512;
  constexpr unsigned bank_hints = 512; // bank_of() hints, one per 32 SPs
  constexpr unsigned estimate_sort_keys = 3584; // SPs of an event whose sort keys fit the estimate kernel's shared memory

  // ------------------------------------------------------------------------------------
  // Bulk copy (TMA engine) into shared memory, completion tracked by an mbarrier.
  // ------------------------------------------------------------------------------------
  __device__ __forceinline__ uint32_t smem_u32(const void* p)
  {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
  }

  __device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }

  __device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
  {
    uint64_t state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                 : "=l"(state)
                 : "r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    (void) state;
  }

  __device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
  {
    asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src),
      "r"(bytes),
      "r"(smem_u32(bar))
      : "memory");
  }

  __device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase)
  {
    uint32_t done;
    asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
    return done != 0;
  }

  constexpr unsigned bulk_wait_limit = 1u << 22; // try_wait rounds before giving up

  // Stages the event blob into `smem_blob` (16-byte aligned) when it fits; returns the
  // address of the event's first word (shared or global) and its length in words.
  // Ends with a __syncthreads().  `bar` must have been initialised with count 1; bar_phase
  // (the same in every thread) is the parity of its current phase.
  __device__ const uint32_t* stage_event(
    const RawInput& in,
    unsigned ev,
    unsigned char* smem_blob,
    unsigned smem_blob_bytes,
    uint64_t* bar,
    unsigned& bar_phase,
    unsigned* status,
    unsigned& n_words,
    unsigned& staged_bytes)
  {
    staged_bytes = 0;
    if (in.mep_layout) {
      // the event's banks are scattered over the MEP: read in place
      n_words = 0xFFFFFFFFu;
      __syncthreads();
      return reinterpret_cast<const uint32_t*>(in.raw);
    }
    const unsigned begin = in.offsets[ev];
    const unsigned end = in.offsets[ev + 1];
    n_words = (end - begin) / 4;
    const char* src = in.raw + begin;
    const uintptr_t s = reinterpret_cast<uintptr_t>(src);
    const uintptr_t e = s + (end - begin);
    const uintptr_t s_al = s & ~uintptr_t(15);
    const uintptr_t e_al = e & ~uintptr_t(15);
    const unsigned need = static_cast<unsigned>(((e + 15) & ~uintptr_t(15)) - s_al);
    const bool base_aligned = (reinterpret_cast<uintptr_t>(in.raw) & 15u) == 0;
    if (!base_aligned || need > smem_blob_bytes) {
      __syncthreads();
      return reinterpret_cast<const uint32_t*>(src);
    }
    const unsigned bulk = e_al > s_al ? static_cast<unsigned>(e_al - s_al) : 0u;
    if (threadIdx.x == 0 && bulk > 0) {
      mbar_expect_tx(bar, bulk);
      bulk_copy_g2s(smem_blob, reinterpret_cast<const void*>(s_al), bulk, bar);
    }
    // ragged tail (whole 32-bit words) by plain loads
    const uintptr_t tail = e_al > s ? e_al : s;
    for (uintptr_t a = tail + 4 * threadIdx.x; a < e; a += 4 * blockDim.x) {
      *reinterpret_cast<uint32_t*>(smem_blob + (a - s_al)) = *reinterpret_cast<const uint32_t*>(a);
    }
    bool ok = true;
    if (bulk > 0) {
      unsigned rounds = 0;
      while (!mbar_try_wait(bar, bar_phase)) {
        if (++rounds > bulk_wait_limit) {
          ok = false;
          break;
        }
      }
      bar_phase ^= 1u; // each completed copy advances the barrier by one phase
    }
    __syncthreads();
    if (!ok) {
      if (threadIdx.x == 0) set_error(status, err_bulk_copy_timeout);
      return reinterpret_cast<const uint32_t*>(src);
    }
    staged_bytes = need;
    return reinterpret_cast<const uint32_t*>(smem_blob + (s - s_al));
  }

  // ------------------------------------------------------------------------------------
  // Bank table of one event (ClusteringDefinitions.cuh:61-144)
  // ------------------------------------------------------------------------------------
  struct BankTable {
    unsigned n_banks;
    unsigned total_sp;
    unsigned count_total;
    unsigned words_off[max_banks]; // first SP word of the bank, in words from the event start
    unsigned n_sp[max_banks];      // SP words of the bank (any bank type)
    unsigned flat[max_banks + 1];  // exclusive scan of n_sp over VP/Velo banks
    unsigned source_id[max_banks];
    uint8_t velo[max_banks];
    // hint[k]: the bank holding flat SP k * 32 (entries up to total_sp / 32), where bank_of()
    // starts a short forward scan
    uint16_t hint[bank_hints];
  };

  __device__ __forceinline__ unsigned bank_module_pair(unsigned source_id, int version)
  {
    return (version == 2 || version == 3) ? (source_id & 0x1FFu) / 8 : ((source_id & 0x1FFu) << 1) / 8;
  }

  // MEP layout: the same table, with word offsets relative to the start of `raw` (the words
  // pointer stage_event returns).  A fragment must start on a 4-byte boundary; its word count
  // is clamped to the bank size.  Ends with a __syncthreads().
  __device__ void parse_banks_mep(const RawInput& in, unsigned ev, BankTable& bt, unsigned* warp_sums, unsigned* status)
  {
    const bool v23 = in.bank_version == 2 || in.bank_version == 3;
    const unsigned n_banks_raw = mep_n_banks(in);
    const unsigned n_banks = n_banks_raw < max_banks ? n_banks_raw : max_banks;
    if (n_banks_raw > max_banks && threadIdx.x == 0) set_error(status, err_input_capacity);
    const uint32_t* raw32 = reinterpret_cast<const uint32_t*>(in.raw);
    unsigned carry = 0, count = 0;
    for (unsigned base = 0; base < n_banks; base += blockDim.x) {
      const unsigned b = base + threadIdx.x;
      unsigned nsp_flat = 0;
      if (b < n_banks) {
        const unsigned frag = mep_fragment_offset(in, ev, b);
        const unsigned size = mep_bank_size(in, ev, b);
        const unsigned type = mep_bank_type(in, ev, b);
        const bool velo_bank = type == bank_type_vp || type == bank_type_velo;
        unsigned nsp = 0, first = 0;
        if (frag & 3u) {
          set_error(status, err_input_capacity);
        }
        else if (v23) {
          nsp = size >= 4 ? raw32[frag / 4] : 0u;
          first = frag / 4 + 1;
          if (velo_bank) count += nsp;
          if (nsp > (size >= 4 ? size / 4 - 1 : 0u)) {
            set_error(status, err_input_capacity);
            nsp = size >= 4 ? size / 4 - 1 : 0u;
          }
        }
        else {
          nsp = size / 4u;
          first = frag / 4;
          if (velo_bank) count += nsp;
        }
        bt.words_off[b] = first;
        bt.n_sp[b] = nsp;
        bt.source_id[b] = mep_source_id(in, b);
        bt.velo[b] = velo_bank;
        nsp_flat = velo_bank ? nsp : 0u;
      }
      unsigned total;
      const unsigned excl = block_exclusive_scan(nsp_flat, warp_sums, &total);
      if (b < n_banks) bt.flat[b] = carry + excl;
      carry += total;
    }
    unsigned total_count;
    block_exclusive_scan(count, warp_sums, &total_count);
    if (threadIdx.x == 0) {
      bt.n_banks = n_banks;
      bt.total_sp = carry;
      bt.flat[n_banks] = carry;
      bt.count_total = total_count;
    }
    __syncthreads();
  }

  // Fills the table; ends with a __syncthreads().
  __device__ void parse_banks(
    const RawInput& in,
    unsigned ev,
    const uint32_t* words,
    unsigned n_words,
    BankTable& bt,
    unsigned* warp_sums,
    unsigned* status)
  {
    const bool v23 = in.bank_version == 2 || in.bank_version == 3;
    if (in.mep_layout) {
      parse_banks_mep(in, ev, bt, warp_sums, status);
      return;
    }
    const unsigned n_banks_raw = n_words > 0 ? words[0] : 0u;
    const unsigned n_banks = n_banks_raw < max_banks ? n_banks_raw : max_banks;
    if (n_banks_raw > max_banks && threadIdx.x == 0) set_error(status, err_input_capacity);
    const uint16_t* sizes = bank_sizes(in, ev);
    const uint8_t* types = bank_types(in, ev);
    unsigned carry = 0, count = 0;
    for (unsigned base = 0; base < n_banks; base += blockDim.x) {
      const unsigned b = base + threadIdx.x;
      unsigned nsp_flat = 0;
      if (b < n_banks) {
        const unsigned off = (1 + b < n_words) ? words[1 + b] : 0u;
        const unsigned w = 2 + n_banks_raw + off / 4;
        const unsigned type = types[b];
        const bool velo_bank = type == bank_type_vp || type == bank_type_velo;
        const unsigned src = w < n_words ? words[w] : 0u;
        unsigned nsp, first;
        if (v23) {
          nsp = (w + 1 < n_words) ? words[w + 1] : 0u;
          first = w + 2;
        }
        else {
          nsp = sizes[b] / 4u;
          first = w + 1;
        }
        if (velo_bank) count += nsp;
        if (first > n_words) first = n_words;
        if (first + nsp > n_words || first + nsp < first) {
          set_error(status, err_input_capacity);
          nsp = n_words - first;
        }
        bt.words_off[b] = first;
        bt.n_sp[b] = nsp;
        bt.source_id[b] = src;
        bt.velo[b] = velo_bank;
        nsp_flat = velo_bank ? nsp : 0u;
      }
      unsigned total;
      const unsigned excl = block_exclusive_scan(nsp_flat, warp_sums, &total);
      if (b < n_banks) bt.flat[b] = carry + excl;
      carry += total;
    }
    // count of SP words of VP/Velo banks, unclamped (reference: raw_bank.count or size / 4)
    unsigned total_count;
    block_exclusive_scan(count, warp_sums, &total_count);
    if (threadIdx.x == 0) {
      bt.n_banks = n_banks;
      bt.total_sp = carry;
      bt.flat[n_banks] = carry;
      bt.count_total = total_count;
    }
    __syncthreads();
  }

  // atomicAdd(counter, 1) from the converged lanes of the warp, one atomic per counter (the
  // lanes that add to the same counter pass the same key): returns this lane's old value, the
  // lanes of a key taking consecutive values in lane order.
  __device__ __forceinline__ unsigned warp_aggregated_inc(unsigned* counter, unsigned key)
  {
    const unsigned peers = __match_any_sync(__activemask(), key);
    const unsigned lane = threadIdx.x & 31u;
    const unsigned leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<unsigned>(__popc(peers)));
    return __shfl_sync(peers, base, leader) + __popc(peers & ((1u << lane) - 1u));
  }

  // atomicAdd(counter, v) from the converged lanes of the warp, one atomic per counter.
  __device__ __forceinline__ void warp_aggregated_add(unsigned* counter, unsigned key, unsigned v)
  {
    const unsigned peers = __match_any_sync(__activemask(), key);
    const unsigned sum = __reduce_add_sync(peers, v);
    if ((threadIdx.x & 31u) == static_cast<unsigned>(__ffs(peers) - 1) && sum) atomicAdd(counter, sum);
  }

  // The hint table of a parsed bank table; ends with a __syncthreads().
  __device__ __forceinline__ void index_banks(BankTable& bt)
  {
    for (unsigned b = threadIdx.x; b < bt.n_banks; b += blockDim.x) {
      const unsigned hi = bt.flat[b + 1];
      for (unsigned k = (bt.flat[b] + 31) / 32; k < bank_hints && k * 32 < hi; ++k)
        bt.hint[k] = static_cast<uint16_t>(b);
    }
    __syncthreads();
  }

  __device__ __forceinline__ unsigned bank_of(const BankTable& bt, unsigned f)
  {
    // last bank b with flat[b] <= f < total_sp (banks with no SP share their start with the next)
    if (f / 32 < bank_hints) {
      unsigned b = bt.hint[f / 32];
      while (b + 1 < bt.n_banks && bt.flat[b + 1] <= f)
        ++b;
      return b;
    }
    unsigned lo = 0, hi = bt.n_banks;
    while (hi - lo > 1) {
      const unsigned mid = (lo + hi) / 2;
      if (bt.flat[mid] <= f) lo = mid;
      else hi = mid;
    }
    return lo;
  }

  // ------------------------------------------------------------------------------------
  // Sorted bank copies.  The neighbour scans of the reference visit every SP of the bank
  // for every SP (EstimateInputSize.cu:111-141) and every candidate
  // (MaskedVeloClustering.cu:361-402).  Each match ORs pattern bits into an accumulator, so
  // the result depends neither on which non-matching SPs are visited nor on how often a
  // matching one is.  With a copy of the bank sorted by key (address bits 22:8, plus the
  // sensor bit 23 for bank version 4), all SPs that can match lie in one key range, found
  // by binary search.  The readout does not write SPs in column order, so the copy is made
  // here: by the estimate kernel into the event's allocation of a global sort scratch, which
  // the clustering kernel then reads; without that scratch, by the clustering kernel itself
  // (in shared memory behind the staged event, or in its slice of the scratch); events that
  // leave no room for it keep the full scans.
  // ------------------------------------------------------------------------------------
  __device__ __forceinline__ uint32_t sp_key_mask(int version) { return version > 3 ? 0xFFFFu : 0x7FFFu; }

  // sorted[bt.flat[b] + r] = the SP word of VP/Velo bank b with rank r by (key, position).
  // Banks hold fewer than 2^16 SPs (the event fits the staging buffer).  Ends with a
  // __syncthreads().
  // With `keys` (shared memory of key_capacity words, the event's SPs fitting it), the
  // (key, position) pairs are formed once per SP and the rank loop reads them from there.
  __device__ void sort_bank_words(const BankTable& bt, const uint32_t* words, uint32_t* sorted, uint32_t key_mask,
                                  uint32_t* keys = nullptr, unsigned key_capacity = 0)
  {
    if (keys != nullptr && bt.total_sp <= key_capacity) {
      for (unsigned f = threadIdx.x; f < bt.total_sp; f += blockDim.x) {
        const unsigned b = bank_of(bt, f);
        const unsigned i = f - bt.flat[b];
        keys[f] = (((words[bt.words_off[b] + i] >> 8) & key_mask) << 16) | i;
      }
      __syncthreads();
      for (unsigned f = threadIdx.x; f < bt.total_sp; f += blockDim.x) {
        const unsigned b = bank_of(bt, f);
        const uint32_t* k = keys + bt.flat[b];
        const unsigned n = bt.flat[b + 1] - bt.flat[b];
        const uint32_t mine = keys[f];
        unsigned rank = 0;
        for (unsigned j = 0; j < n; ++j)
          rank += k[j] < mine;
        sorted[f - (mine & 0xFFFFu) + rank] = words[bt.words_off[b] + (mine & 0xFFFFu)];
      }
      __syncthreads();
      return;
    }
    for (unsigned f = threadIdx.x; f < bt.total_sp; f += blockDim.x) {
      const unsigned b = bank_of(bt, f);
      const unsigned i = f - bt.flat[b];
      const uint32_t* w = words + bt.words_off[b];
      const unsigned n = bt.flat[b + 1] - bt.flat[b];
      const uint32_t mine = (((w[i] >> 8) & key_mask) << 16) | i;
      unsigned rank = 0;
      for (unsigned j = 0; j < n; ++j)
        rank += ((((w[j] >> 8) & key_mask) << 16) | j) < mine;
      sorted[bt.flat[b] + rank] = w[i];
    }
    __syncthreads();
  }

  // First index in [0, n) whose key is >= k (keys non-decreasing).
  __device__ __forceinline__ unsigned first_key_at_least(const uint32_t* w, unsigned n, uint32_t k, uint32_t key_mask)
  {
    unsigned lo = 0, len = n;
    while (len > 0) {
      const unsigned half = len >> 1;
      if (((w[lo + half] >> 8) & key_mask) < k) {
        lo += half + 1;
        len -= half + 1;
      }
      else {
        len = half;
      }
    }
    return lo;
  }

  // ------------------------------------------------------------------------------------
  // Candidate search of a non-isolated SP (EstimateInputSize.cu:72-204).  Every SP of
  // the bank is a potential neighbour: the reference reads the current SP's own
  // no-neighbour bit instead of the other's (line 113), which is always 0 here.
  // Returns up to two candidate pixel codes: bit 8 set = present, bits 0..2 = pixel.
  // ------------------------------------------------------------------------------------
  __device__ __forceinline__ void
  add_neighbour_pixels(uint32_t& pixels, uint32_t ow, uint32_t sp_row, uint32_t sp_col)
  {
    const uint32_t oaddr = (ow & 0x007FFF00u) >> 8;
    const uint32_t orow = oaddr & 0x3Fu;
    const uint32_t ocol = oaddr >> 6;
    const uint32_t osp = ow & 0xFFu;
    const bool col_same = ocol == sp_col;
    const bool col_right = ocol == sp_col + 1;
    if (!(col_same || col_right)) return;
    if (orow == sp_row + 1) {
      if (col_same) pixels |= (((osp & 0x01u) | ((osp & 0x10u) << 2)) << 4);
      else pixels |= ((osp & 0x01u) << 16);
    }
    else if (orow == sp_row) {
      if (col_right) pixels |= ((osp & 0x0Fu) << 12);
    }
    else if (orow == sp_row - 1) {
      if (col_right) pixels |= ((osp & 0x08u) << 8);
      else pixels |= ((osp & 0x80u) >> 2);
    }
  }

  // key_mask != 0: the bank is sorted by (w >> 8) & key_mask.  Neighbours of either
  // sensor count (the reference compares bits 22:8 only), so version 4 banks, sorted by
  // (sensor bit, address), are searched in two ranges.
  __device__ __forceinline__ uint32_t
  sp_candidates(uint32_t sp_word, const uint32_t* bank_words, unsigned n_sp, uint32_t key_mask = 0)
  {
    const uint32_t sp_addr = (sp_word & 0x007FFF00u) >> 8;
    const uint32_t sp = sp_word & 0xFFu;
    uint32_t pixels = (sp & 0x0Fu) | ((sp & 0xF0u) << 2);
    const uint32_t sp_row = sp_addr & 0x3Fu;
    const uint32_t sp_col = sp_addr >> 6;
    if (key_mask == 0) {
      for (unsigned k = 0; k < n_sp; ++k)
        add_neighbour_pixels(pixels, bank_words[k], sp_row, sp_col);
    }
    else {
      // matches have column sp_col or sp_col + 1 and row sp_row - 1 .. sp_row + 1
      const uint32_t lo_off = (sp_col << 6) + (sp_row > 0 ? sp_row - 1 : 0u);
      const uint32_t hi_off = ((sp_col + 1) << 6) + (sp_row < 63 ? sp_row + 1 : 63u);
      for (uint32_t half = 0; half <= (key_mask >> 15); ++half) {
        const uint32_t k_hi = (half << 15) + hi_off;
        for (unsigned k = first_key_at_least(bank_words, n_sp, (half << 15) + lo_off, key_mask); k < n_sp; ++k) {
          const uint32_t ow = bank_words[k];
          if (((ow >> 8) & key_mask) > k_hi) break;
          add_neighbour_pixels(pixels, ow, sp_row, sp_col);
        }
      }
    }
    const uint32_t inside = pixels & 0x3CFu;
    const uint32_t mask = (inside << 1) | (inside << 5) | (inside << 6) | (inside << 7);
    const uint32_t working = mask & (~pixels);
    const uint32_t cand_tmp = (working >> 1) & (working >> 5) & (working >> 6) & (working >> 7);
    const uint32_t cands = cand_tmp & pixels;
    const uint32_t consolidated = (cands & 0x0Fu) | ((cands >> 2) & 0xF0u);
    const uint32_t first = consolidated & 0x33u;
    const uint32_t second = consolidated & 0xCCu;
    uint32_t r = 0;
    if (first) r |= 0x100u | (__clz(first) - 24);
    if (second) r |= (0x100u | (__clz(second) - 24)) << 16;
    return r;
  }

  __device__ __forceinline__ bool isolated_two_clusters(uint32_t sp)
  {
    const bool pattern_0 = (sp & 0x88u) && !(sp & 0x44u) && (sp & 0x33u);
    const bool pattern_1 = (sp & 0xCCu) && !(sp & 0x22u) && (sp & 0x11u);
    return pattern_0 || pattern_1;
  }

  constexpr unsigned estimate_queue = 1024; // SPs per chunk of the estimate (and queue entries)
  static_assert(estimate_queue % decode_threads == 0, "every lane takes the same number of SPs per chunk");

  // ------------------------------------------------------------------------------------
  // estimate_kernel: dev_number_of_candidates, dev_velo_bank_index (as a max-reduced
  // key), dev_estimated_input_size and dev_module_candidate_num.
  // ------------------------------------------------------------------------------------
  __device__ __forceinline__ void estimate_event(const EstimateParams& p, unsigned e, uint64_t* bar, unsigned& bar_phase)
  {
    extern __shared__ __align__(128) unsigned char dsmem[];
    __shared__ BankTable bt;
    __shared__ unsigned est_mp[n_module_pairs];
    __shared__ unsigned cand_count;
    __shared__ unsigned warp_sums[33];
    __shared__ uint16_t queue[estimate_queue];
    __shared__ unsigned queue_count[2];
    __shared__ unsigned sorted_at;
    __shared__ uint32_t sort_keys[estimate_sort_keys];

    const unsigned ev = e + p.in.event_start;
    const bool v23 = p.in.bank_version == 2 || p.in.bank_version == 3;
    if (threadIdx.x < n_module_pairs) est_mp[threadIdx.x] = 0;
    if (threadIdx.x == 0) cand_count = 0;
    if (threadIdx.x < 2) queue_count[threadIdx.x] = 0;
    __syncthreads();

    unsigned n_words, staged;
    const uint32_t* words = stage_event(p.in, ev, dsmem, p.smem_blob_bytes, bar, bar_phase, p.status, n_words, staged);
    parse_banks(p.in, ev, words, n_words, bt, warp_sums, p.status);
    index_banks(bt);
    (void) staged;
    // The event's banks sorted by key into its allocation of the sort scratch: this kernel's
    // neighbour search then scans key ranges, and the clustering kernel reuses the copies.
    // Without scratch (or room in it) the search scans every SP of the bank.
    const uint32_t key_mask = sp_key_mask(p.in.bank_version);
    const uint32_t* sorted = nullptr;
    if (p.sp_scratch != nullptr) {
      if (threadIdx.x == 0) {
        const unsigned at = atomicAdd(p.sp_alloc, bt.total_sp);
        sorted_at = (at <= p.sp_capacity && bt.total_sp <= p.sp_capacity - at) ? at : no_sorted_copy;
        p.sp_base[e] = sorted_at;
      }
      __syncthreads();
      if (sorted_at != no_sorted_copy) {
        sort_bank_words(bt, words, p.sp_scratch + sorted_at, key_mask, sort_keys, estimate_sort_keys);
        sorted = p.sp_scratch + sorted_at;
      }
    }

    // velo_calculate_number_of_candidates: block 0 of the reference's launch (grid of
    // ceil(N / 256) blocks, one thread per event) handles events 0, stride, 2 stride, ...
    // and the last of them to write an entry wins.
    if (p.designated_stride > 0 && e % p.designated_stride == 0) {
      const unsigned long long key_hi = static_cast<unsigned long long>(e) << 32;
      for (unsigned b = threadIdx.x; b < bt.n_banks; b += blockDim.x) {
        const unsigned src = bt.source_id[b] & 0x1FFu;
        if (p.in.bank_version > 3) {
          if ((src << 1) < n_sensors) atomicMax(p.bank_index_key + (src << 1), key_hi | b);
          if (((src << 1) | 1u) < n_sensors) atomicMax(p.bank_index_key + ((src << 1) | 1u), key_hi | b);
        }
        else if (src < n_sensors) {
          atomicMax(p.bank_index_key + src, key_hi | b);
        }
      }
    }

    // Two passes per chunk of SPs, so that the warps do not diverge between the isolated SPs
    // (about two thirds: one pattern test each) and the neighbour scans of the others: pass 1
    // counts the isolated SPs and queues the others (warp-aggregated), pass 2 scans the
    // queued SPs with every lane busy.  The counts are sums, so the order does not matter.
    const unsigned chunk = estimate_queue;
    for (unsigned chunk_base = 0, parity = 0; chunk_base < bt.total_sp; chunk_base += chunk, parity ^= 1u) {
      for (unsigned f = chunk_base + threadIdx.x; f < chunk_base + chunk; f += blockDim.x) {
        bool queued = false;
        if (f < bt.total_sp) {
          const unsigned b = bank_of(bt, f);
          const uint32_t word = words[bt.words_off[b] + f - bt.flat[b]];
          if (word & 0x80000000u) {
            const unsigned mp = bank_module_pair(bt.source_id[b], p.in.bank_version);
            if (mp < n_module_pairs) warp_aggregated_add(&est_mp[mp], mp, isolated_two_clusters(word & 0xFFu) ? 2u : 1u);
            else set_error(p.status, err_input_capacity);
          }
          else {
            queued = true;
          }
        }
        const unsigned lane = threadIdx.x & 31u;
        const unsigned mask = __ballot_sync(0xFFFFFFFFu, queued);
        if (mask) {
          const unsigned leader = __ffs(mask) - 1;
          unsigned at = 0;
          if (lane == leader) at = atomicAdd(&queue_count[parity], __popc(mask));
          at = __shfl_sync(0xFFFFFFFFu, at, leader);
          if (queued) queue[at + __popc(mask & ((1u << lane) - 1u))] = static_cast<uint16_t>(f - chunk_base);
        }
      }
      __syncthreads();
      const unsigned n_queued = min(queue_count[parity], chunk);
      if (threadIdx.x == 0) queue_count[parity ^ 1u] = 0;
      for (unsigned q = threadIdx.x; q < n_queued; q += blockDim.x) {
        const unsigned f = chunk_base + queue[q];
        const unsigned b = bank_of(bt, f);
        const uint32_t* bank_words = words + bt.words_off[b];
        const uint32_t word = bank_words[f - bt.flat[b]];
        const uint32_t c = sorted ? sp_candidates(word, sorted + bt.flat[b], bt.n_sp[b], key_mask)
                                  : sp_candidates(word, bank_words, bt.n_sp[b]);
        const unsigned add = ((c >> 8) & 1u) + ((c >> 24) & 1u);
        warp_aggregated_add(&cand_count, 0u, add);
        const unsigned mp = bank_module_pair(bt.source_id[b], p.in.bank_version);
        if (mp < n_module_pairs) warp_aggregated_add(&est_mp[mp], mp, add);
        else set_error(p.status, err_input_capacity);
      }
      __syncthreads();
    }
    if (threadIdx.x < n_module_pairs) {
      p.estimated_input_size[e * n_module_pairs + threadIdx.x] = est_mp[threadIdx.x];
    }
    if (threadIdx.x == 0) {
      unsigned s = 0;
      for (unsigned mp = 0; mp < n_module_pairs; ++mp)
        s += est_mp[mp];
      p.event_estimate[e] = s;
      p.number_of_candidates[e] = 2 * bt.count_total;
      p.module_candidate_num[e] = cand_count;
    }
    (void) v23;
  }

  __global__ void __launch_bounds__(decode_threads, 2048 / decode_threads) estimate_kernel(EstimateParams p)
  {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    unsigned bar_phase = 0;
    for_each_event(p.queue, p.in.n_events, [&](unsigned e, unsigned) { estimate_event(p, e, &bar, bar_phase); });
  }

  // ------------------------------------------------------------------------------------
  // Mask clustering of one candidate (MaskedVeloClustering.cu:21-84, 290-496)
  // ------------------------------------------------------------------------------------
  __device__ __forceinline__ uint64_t make_8con_mask(uint64_t c)
  {
    return c | ((c & 0x7FFF7FFF7FFF7FFFull) << 1) | ((c & 0xFFFEFFFEFFFEFFFEull) << 15) | (c << 16) |
           ((c & 0xFFFCFFFCFFFCFFFCull) << 17) | ((c & 0xFFFEFFFEFFFEFFFEull) >> 1) |
           ((c & 0x7FFF7FFF7FFF7FFFull) >> 15) | (c >> 16) | ((c & 0x3FFF3FFF3FFF3FFFull) >> 17);
  }

  __device__ __forceinline__ uint64_t mask_east(uint64_t c)
  {
    const uint64_t m = c >> 48;
    return m | ((m & 0x7FFF7FFF7FFF7FFFull) << 1) | (m >> 1);
  }

  __device__ __forceinline__ uint64_t mask_west(uint64_t c)
  {
    const uint64_t m = c << 48;
    return m | (m << 1) | ((m & 0xFFFEFFFEFFFEFFFEull) >> 1);
  }

  struct PixelCluster {
    uint64_t pixels;
    uint32_t x, y, n;
  };

  __device__ __forceinline__ PixelCluster
  make_cluster(uint64_t map, uint64_t start, uint32_t col_lower, uint32_t row_lower)
  {
    uint64_t cur = 0, next = start;
    while (cur != next) {
      cur = next;
      next = map & make_8con_mask(cur);
    }
    PixelCluster c;
    c.pixels = cur;
    c.n = __popcll(cur);
    c.x = col_lower * c.n + __popcll(cur & 0x00000000FFFF0000ull) + __popcll(cur & 0x0000FFFF00000000ull) * 2 +
          __popcll(cur & 0xFFFF000000000000ull) * 3;
    uint32_t y = row_lower * c.n;
#pragma unroll
    for (unsigned r = 1; r <= 14; ++r)
      y += __popcll(cur & (0x0001000100010001ull << r)) * r;
    c.y = y;
    return c;
  }

  struct ClusterOut {
    uint32_t id;
    float x, y, z;
    int16_t phi;
  };

  __device__ __forceinline__ void
  local_to_global(const Geometry* g, const float* ltg, float local_x, float local_y, ClusterOut& o)
  {
    o.x = __ldg(ltg + 0) * local_x + __ldg(ltg + 1) * local_y + __ldg(ltg + 9);
    o.y = __ldg(ltg + 3) * local_x + __ldg(ltg + 4) * local_y + __ldg(ltg + 10);
    o.z = __ldg(ltg + 6) * local_x + __ldg(ltg + 7) * local_y + __ldg(ltg + 11);
  }

  __device__ bool rest_of_clusters(
    const Geometry* g,
    const Constants& k,
    uint32_t candidate,
    const uint32_t* bank_words,
    const uint32_t* sorted_words,
    unsigned n_sp,
    int version,
    ClusterOut& o,
    bool& bad)
  {
    const uint32_t sp_index = candidate >> 11;
    const uint32_t sensor_number = (candidate >> 3) & 0xFFu;
    const uint32_t start_loc = candidate & 0x7u;
    const float* ltg = g->ltg + 12 * sensor_number;
    const uint32_t sp_word = bank_words[sp_index];
    const uint32_t sp_addr = (sp_word & 0x007FFF00u) >> 8;
    const int32_t sp_row = static_cast<int32_t>(sp_addr & 0x3Fu);
    const int32_t sp_col = static_cast<int32_t>(sp_addr >> 6);

    uint32_t pa[5] = {0, 0, 0, 0, 0};
    const int32_t r_lo = sp_row - 2, r_hi = sp_row + 1;
    const int32_t c_lo = sp_col - 3, c_hi = sp_col + 1;
    const int32_t row_lower = r_lo * 4;
    const int32_t col_lower = c_lo * 2;
    // window SPs lie in one key range of a sorted bank (version 4: of this sensor)
    const uint32_t key_mask = sp_key_mask(version);
    const uint32_t* scan = sorted_words ? sorted_words : bank_words;
    unsigned j = 0;
    uint32_t k_hi = 0xFFFFFFFFu;
    if (sorted_words) {
      const uint32_t half = version > 3 ? (sensor_number & 0x1u) << 15 : 0u;
      const uint32_t k_lo = half + (static_cast<uint32_t>(max(c_lo, 0)) << 6) + static_cast<uint32_t>(max(r_lo, 0));
      k_hi = half + (static_cast<uint32_t>(c_hi) << 6) + static_cast<uint32_t>(min(r_hi, 63));
      j = first_key_at_least(sorted_words, n_sp, k_lo, key_mask);
    }
    for (; j < n_sp; ++j) {
      const uint32_t ow = scan[j];
      if (((ow >> 8) & key_mask) > k_hi) break;
      if (version > 3) {
        const uint32_t other_bit = (ow & 0x800000u) ? 1u : 0u;
        if (other_bit != (sensor_number & 0x1u)) continue;
      }
      if (ow & 0x80000000u) continue;
      const uint32_t oaddr = (ow & 0x007FFF00u) >> 8;
      const int32_t orow = static_cast<int32_t>(oaddr & 0x3Fu);
      const int32_t ocol = static_cast<int32_t>(oaddr >> 6);
      if (orow >= r_lo && orow <= r_hi && ocol >= c_lo && ocol <= c_hi) {
        const uint32_t osp = ow & 0xFFu;
        const int rel_row = orow - r_lo;
        const int rel_col = ocol - c_lo;
        const uint32_t bits = ((osp & 0x0Fu) << (4 * rel_row)) | ((osp & 0xF0u) << (12 + 4 * rel_row));
#pragma unroll
        for (int c = 0; c < 5; ++c)
          if (c == rel_col) pa[c] |= bits;
      }
    }

    const uint32_t rel_row0 = start_loc & 0x3u;
    const uint32_t rel_col0 = start_loc < 4 ? 1u : 0u;
    const uint32_t col = static_cast<uint32_t>(sp_col) * 2 + rel_col0;
    const uint64_t start = (static_cast<uint64_t>(0x01u << (11 - rel_row0)) << (16 * (col & 0x01u))) << 32;
    const uint64_t map = (static_cast<uint64_t>(pa[3]) << 32) | pa[2];
    const PixelCluster cl = make_cluster(map, start, static_cast<uint32_t>(col_lower + 4), static_cast<uint32_t>(row_lower));
    const uint64_t precedence = (mask_east(cl.pixels) & pa[4]) | (cl.pixels & (start ^ (0ull - start)));
    bool keep = precedence == 0 && !(cl.pixels & 0x8000800080008000ull) && !(cl.pixels & 0x0001000100010001ull);
    if (!keep) return false;
    uint32_t x = cl.x, y = cl.y, n = cl.n;
    if (cl.pixels & 0xFFFFull) {
      const uint64_t west_map = (static_cast<uint64_t>(pa[1]) << 32) | pa[0];
      const uint64_t west_start = mask_west(cl.pixels) & west_map;
      const PixelCluster ext =
        make_cluster(west_map, west_start, static_cast<uint32_t>(col_lower), static_cast<uint32_t>(row_lower));
      x += ext.x;
      y += ext.y;
      n += ext.n;
      keep = !(ext.pixels & 0x8000800080008000ull) && !(ext.pixels & 0xFFFFull) &&
             !(cl.pixels & 0x0001000100010001ull);
    }
    if (!keep) return false;
    // A candidate whose bank index names another bank (the reference's lookup of the bank by
    // sensor, when a slice holds more than one bank per sensor) can leave the start pixel
    // outside the map: no pixel, and the reference divides by zero.
    if (n == 0) {
      bad = true;
      return false;
    }
    // The integer centroids x / n and y / n are the truncated correctly rounded quotients: a
    // quotient below 1024 (columns < 768, rows < 256) with n < 32768 pixels is at least 1 / n
    // below the next integer, more than half an ulp, so rounding never reaches it.  The
    // fractions are the reference's fl(x / n) - cx (MaskedVeloClustering.cu:461-466).
    const float qx = __fdiv_rn(__uint2float_rn(x), __uint2float_rn(n));
    const float qy = __fdiv_rn(__uint2float_rn(y), __uint2float_rn(n));
    const uint32_t cx = __float2uint_rz(qx);
    const uint32_t cy = __float2uint_rz(qy);
    const float fx = qx - __uint2float_rn(cx);
    const float fy = qy - __uint2float_rn(cy);
    const uint32_t chip = cx >> 8;
    o.id = lhcb_id(channel_id(sensor_number, chip, cx & 0xFFu, cy));
    const float local_x = column_local_x(g, cx) + fx * column_x_pitch(g, cx);
    const float local_y = (__uint2float_rn(cy) + 0.5f + fy) * 0.055f;
    local_to_global(g, ltg, local_x, local_y, o);
    o.phi = hit_phi_16(k, o.x, o.y);
    return true;
  }

  // Isolated SP through the lookup tables (MaskedVeloClustering.cu:131-288); which = 0/1.
  __device__ __forceinline__ void isolated_cluster(
    const Geometry* g,
    const Constants& k,
    uint32_t sp_word,
    unsigned source_id,
    int version,
    unsigned which,
    ClusterOut& o)
  {
    const bool v23 = version == 2 || version == 3;
    const bool bit23 = (sp_word & 0x800000u) != 0;
    const uint32_t pair = source_id & 0x1FFu;
    const uint32_t sensor_index = v23 ? source_id : (bit23 ? ((pair << 1) | 1u) : (pair << 1));
    const float* ltg = g->ltg + 12 * (v23 ? pair : (bit23 ? ((pair << 1) | 1u) : (pair << 1)));
    const uint32_t sp_addr = (sp_word & 0x007FFF00u) >> 8;
    const int32_t sp_row = static_cast<int32_t>(sp_addr & 0x3Fu);
    const int32_t sp_col = static_cast<int32_t>(sp_addr >> 6);
    const uint32_t sp = sp_word & 0xFFu;
    const uint32_t idx = __ldg(g->sp_patterns + sp);
    const uint32_t chip = static_cast<uint32_t>(sp_col) >> 7;
    const uint32_t row = which ? (idx >> 4) & 3u : idx & 3u;
    const uint32_t col = which ? (idx >> 6) & 1u : (idx >> 2) & 1u;
    const uint32_t cx = static_cast<uint32_t>(sp_col) * 2 + col;
    const uint32_t cy = static_cast<uint32_t>(sp_row) * 4 + row;
    o.id = lhcb_id(channel_id(sensor_index, chip, cx & 0xFFu, cy));
    const float fx = __ldg(g->sp_fx + sp * 2 + which);
    const float fy = __ldg(g->sp_fy + sp * 2 + which);
    const float local_x = column_local_x(g, cx) + fx * column_x_pitch(g, cx);
    const float local_y = (__uint2float_rn(cy) + 0.5f + fy) * 0.055f;
    local_to_global(g, ltg, local_x, local_y, o);
    o.phi = hit_phi_16(k, o.x, o.y);
  }

  // ------------------------------------------------------------------------------------
  // cluster_sort_kernel
  // ------------------------------------------------------------------------------------
  // queued candidates per chunk of 2 THREADS SPs (two candidates at most per SP)
  template<unsigned THREADS>
  constexpr unsigned candidate_queue = 4 * THREADS;

  __device__ __forceinline__ unsigned sort_bucket(int16_t phi) { return static_cast<unsigned>(phi + 32768) >> 9; }

  // u16 counters packed two per 32-bit word; returns the previous count of counter b.
  __device__ __forceinline__ uint16_t count_in_bucket(uint16_t* counters, unsigned b)
  {
    const unsigned shift = 16 * (b & 1u);
    const uint32_t old = atomicAdd(reinterpret_cast<uint32_t*>(counters) + (b >> 1), 1u << shift);
    return static_cast<uint16_t>(old >> shift);
  }
  template<unsigned THREADS>
  __device__ __forceinline__ void
  cluster_sort_event(const ClusterSortParams& p, unsigned e, uint64_t* bar, unsigned& bar_phase)
  {
    constexpr unsigned queue_size = candidate_queue<THREADS>;
    extern __shared__ __align__(128) unsigned char dsmem[];
    __shared__ BankTable bt;
    __shared__ unsigned region[n_module_pairs + 1]; // estimated start of each module pair, event-relative
    __shared__ unsigned mp_count[n_module_pairs];
    __shared__ unsigned staged_first[n_module_pairs + 1]; // staged clusters before each module pair
    __shared__ unsigned warp_sums[33];
    __shared__ unsigned sorted_total;
    __shared__ uint32_t queue[queue_size];
    __shared__ unsigned queue_count[2];

    const unsigned ev = e + p.in.event_start;
    const unsigned n = p.in.n_events;
    const int version = p.in.bank_version;
    const unsigned base = p.event_base[e];
    const unsigned T = p.event_base[n];
    if (T > p.cluster_capacity) {
      // the slice needs more clusters than reserved: nothing is written
      if (threadIdx.x == 0) set_error(p.status, err_input_capacity);
      return;
    }

    if (threadIdx.x == 0) {
      unsigned s = 0;
      for (unsigned mp = 0; mp < n_module_pairs; ++mp) {
        region[mp] = s;
        s += p.estimated_input_size[e * n_module_pairs + mp];
      }
      region[n_module_pairs] = s;
    }
    if (threadIdx.x < n_module_pairs) mp_count[threadIdx.x] = 0;
    if (threadIdx.x < 2) queue_count[threadIdx.x] = 0;
    __syncthreads();
    if (threadIdx.x < n_module_pairs) {
      p.offsets_estimated_input_size[e * n_module_pairs + threadIdx.x] = base + region[threadIdx.x];
    }
    if (e == n - 1 && threadIdx.x == 0) p.offsets_estimated_input_size[n * n_module_pairs] = T;

    const unsigned est_total = region[n_module_pairs];
    // Staging of the unsorted clusters (18 bytes each) plus two u16 per cluster for the
    // sort: shared memory when they fit, else the event's slice of the global staging
    // buffer (24 bytes per estimated cluster).  Bucket counters and the blob follow.
    const bool staged_in_smem = est_total <= p.smem_cluster_capacity;
    const unsigned cap = staged_in_smem ? p.smem_cluster_capacity : est_total;
    char* stage_base = staged_in_smem ? reinterpret_cast<char*>(dsmem) : p.staging + size_t(24) * base;
    ClusterView st {stage_base, est_total};
    uint16_t* slot_in_bucket = reinterpret_cast<uint16_t*>(stage_base + size_t(element_size) * cap);
    uint16_t* members = slot_in_bucket + cap;
    uint16_t* bucket_start = reinterpret_cast<uint16_t*>(dsmem + cluster_sort_counter_offset(p.smem_cluster_capacity));
    unsigned char* blob = dsmem + cluster_sort_blob_offset(p.smem_cluster_capacity);
    for (unsigned i = threadIdx.x; i < sort_counters / 2; i += blockDim.x)
      reinterpret_cast<uint32_t*>(bucket_start)[i] = 0;

    unsigned n_words, staged;
    const uint32_t* words = stage_event(p.in, ev, blob, p.smem_blob_bytes, bar, bar_phase, p.status, n_words, staged);
    parse_banks(p.in, ev, words, n_words, bt, warp_sums, p.status);
    index_banks(bt);
    const uint32_t key_mask = sp_key_mask(version);
    // sorted bank copies: behind the staged event (or at the start of the blob), else in the
    // event's slice of the global scratch (L2-resident), else none (full neighbour scans)
    uint32_t* sorted = nullptr;
    bool sorted_in_scratch = false;
    if (p.sp_base != nullptr) {
      // sorted by the estimate kernel (no copy when its scratch had no room: full scans)
      const unsigned at = p.sp_base[e];
      if (at != no_sorted_copy) {
        sorted = p.sp_scratch + at;
        sorted_in_scratch = true;
      }
    }
    else if (staged + 4 * bt.total_sp <= p.smem_blob_bytes) {
      sorted = reinterpret_cast<uint32_t*>(blob + staged);
    }
    else if (p.sp_scratch != nullptr) {
      const unsigned sp_base = p.candidates_offsets[e] / 2;
      if (sp_base + bt.total_sp <= p.sp_capacity) {
        sorted = p.sp_scratch + sp_base;
        sorted_in_scratch = true;
      }
    }
    if (sorted && p.sp_base == nullptr) sort_bank_words(bt, words, sorted, key_mask);

    const Geometry* g = p.geo;
    auto stage_cluster = [&](const ClusterOut& o, unsigned mp) {
      const unsigned slot = warp_aggregated_inc(&mp_count[mp], mp);
      if (region[mp] + slot < region[mp + 1]) {
        const unsigned i = region[mp] + slot;
        st.id(i) = o.id;
        st.x(i) = o.x;
        st.y(i) = o.y;
        st.z(i) = o.z;
        st.phi(i) = o.phi;
        slot_in_bucket[i] = count_in_bucket(bucket_start, mp * sort_buckets + sort_bucket(o.phi));
      }
      else {
        set_error(p.status, err_cluster_capacity);
      }
    };

    // Two passes per chunk of SPs, so that the warps do not diverge between the isolated
    // SPs (about two thirds, one table lookup each) and the flood fills of candidates:
    // pass 1 makes the clusters of isolated SPs and queues the candidates of the others
    // (EstimateInputSize.cu:72-204 order of codes), pass 2 runs rest_of_clusters on the
    // queue.  A chunk has queue_size / 2 SPs, so the queue cannot overflow; every lane takes
    // the same number of SPs per chunk.
    const unsigned chunk = queue_size / 2;
    for (unsigned chunk_base = 0, parity = 0; chunk_base < bt.total_sp; chunk_base += chunk, parity ^= 1u) {
      for (unsigned f = chunk_base + threadIdx.x; f < chunk_base + chunk; f += blockDim.x) {
        uint32_t cand[2] = {0, 0};
        bool valid[2] = {false, false};
        if (f < bt.total_sp) {
          const unsigned b = bank_of(bt, f);
          const unsigned mp = bank_module_pair(bt.source_id[b], version);
          const uint32_t* bank_words = words + bt.words_off[b];
          const unsigned sp_index = f - bt.flat[b];
          const uint32_t word = bank_words[sp_index];
          if (mp >= n_module_pairs) {
            // a source id beyond the 26 module pairs: malformed input, flagged by estimate_kernel
          }
          else if (word & 0x80000000u) {
            const unsigned n_clusters = (__ldg(g->sp_patterns + (word & 0xFFu)) & 8u) ? 2u : 1u;
            for (unsigned which = 0; which < n_clusters; ++which) {
              ClusterOut o;
              isolated_cluster(g, p.k, word, bt.source_id[b], version, which, o);
              stage_cluster(o, mp);
            }
          }
          else {
            const uint32_t c = sorted ? sp_candidates(word, sorted + bt.flat[b], bt.n_sp[b], key_mask)
                                      : sp_candidates(word, bank_words, bt.n_sp[b]);
            const bool v23 = version == 2 || version == 3;
            const uint32_t sensor_number =
              v23 ? (bt.source_id[b] & 0x1FFu) : (((bt.source_id[b] & 0x1FFu) << 1) | ((word >> 23) & 0x1u));
            for (unsigned which = 0; which < 2; ++which) {
              const uint32_t code = which ? (c >> 16) : c;
              if (!(code & 0x100u)) continue;
              cand[which] = (sp_index << 11) | (sensor_number << 3) | (code & 0x7u);
              // MaskedVeloClustering.cu:567-572: the candidate's bank is looked up by sensor
              if (((cand[which] >> 3) & 0xFFu) >= n_sensors) set_error(p.status, err_bad_sensor);
              else valid[which] = true;
            }
          }
        }
        // warp-aggregated append to the queue (every lane of the warp gets here)
        const unsigned lane = threadIdx.x & 31u;
        for (unsigned which = 0; which < 2; ++which) {
          const unsigned mask = __ballot_sync(0xFFFFFFFFu, valid[which]);
          if (mask == 0) continue;
          const unsigned leader = __ffs(mask) - 1;
          unsigned at = 0;
          if (lane == leader) at = atomicAdd(&queue_count[parity], __popc(mask));
          at = __shfl_sync(0xFFFFFFFFu, at, leader);
          if (valid[which]) queue[at + __popc(mask & ((1u << lane) - 1u))] = cand[which];
        }
      }
      __syncthreads();
      const unsigned queued = min(queue_count[parity], queue_size);
      if (threadIdx.x == 0) queue_count[parity ^ 1u] = 0;
      for (unsigned q = threadIdx.x; q < queued; q += blockDim.x) {
        const uint32_t candidate = queue[q];
        const uint32_t cand_sensor = (candidate >> 3) & 0xFFu;
        const unsigned b2 = static_cast<unsigned>(p.bank_index_key[cand_sensor] & 0xFFFFFFFFull);
        if (b2 >= bt.n_banks || (candidate >> 11) >= bt.n_sp[b2]) {
          set_error(p.status, err_input_capacity);
          continue;
        }
        ClusterOut o;
        bool bad = false;
        const uint32_t* sorted_b2 = sorted && bt.velo[b2] ? sorted + bt.flat[b2] : nullptr;
        if (rest_of_clusters(g, p.k, candidate, words + bt.words_off[b2], sorted_b2, bt.n_sp[b2], version, o, bad))
          stage_cluster(o, cand_sensor / 8);
        else if (bad)
          set_error(p.status, err_bad_super_pixel);
      }
      __syncthreads();
    }

    // Sort by (phi, id) inside each module pair (SortByPhi.cu:104-122).  The reference
    // ranks every pair of clusters; here clusters were counted into 128 phi buckets per
    // module pair while staged, so a scan of the counters places every bucket and a
    // cluster's rank is its bucket's start plus the number of smaller (phi, id) keys in the
    // same bucket - the same position as the reference's full count.
    {
      // each thread owns `per` consecutive counters: it sums them, and after the scan turns
      // them into starts in place (no other thread reads them in between)
      constexpr unsigned per = (sort_counters + THREADS - 1) / THREADS;
      unsigned sum = 0;
      for (unsigned q = 0; q < per; ++q) {
        const unsigned b = threadIdx.x * per + q;
        if (b < sort_counters) sum += bucket_start[b];
      }
      unsigned total;
      unsigned excl = block_exclusive_scan(sum, warp_sums, &total);
      if (threadIdx.x == 0) {
        sorted_total = total;
        unsigned staged = 0;
        for (unsigned mp = 0; mp < n_module_pairs; ++mp) {
          staged_first[mp] = staged;
          staged += min(mp_count[mp], region[mp + 1] - region[mp]);
        }
        staged_first[n_module_pairs] = staged;
      }
      for (unsigned q = 0; q < per; ++q) {
        const unsigned b = threadIdx.x * per + q;
        if (b < sort_counters) {
          const unsigned count = bucket_start[b];
          bucket_start[b] = static_cast<uint16_t>(excl);
          excl += count;
        }
      }
    }
    __syncthreads();
    // the k-th staged cluster of the event: its module pair (the last one whose first staged
    // cluster is at most k, empty ones skipped) and its staging index
    const unsigned n_staged = staged_first[n_module_pairs];
    auto module_pair_of = [&](unsigned k) {
      unsigned lo = 0, hi = n_module_pairs;
      while (hi - lo > 1) {
        const unsigned mid = (lo + hi) / 2;
        if (staged_first[mid] <= k) lo = mid;
        else hi = mid;
      }
      return lo;
    };
    for (unsigned k = threadIdx.x; k < n_staged; k += blockDim.x) {
      const unsigned mp = module_pair_of(k);
      const unsigned i = region[mp] + (k - staged_first[mp]);
      const unsigned b = mp * sort_buckets + sort_bucket(st.phi(i));
      const unsigned q = bucket_start[b] + slot_in_bucket[i];
      if (q < cap) members[q] = static_cast<uint16_t>(i);
    }
    __syncthreads();
    ClusterView out {p.sorted_container, T};
    for (unsigned k = threadIdx.x; k < n_staged; k += blockDim.x) {
      const unsigned mp = module_pair_of(k);
      const unsigned i = region[mp] + (k - staged_first[mp]);
      const unsigned count = staged_first[mp + 1] - staged_first[mp];
      const int16_t phi = st.phi(i);
      const uint32_t id = st.id(i);
      const unsigned b = mp * sort_buckets + sort_bucket(phi);
      const unsigned b_end = min(b + 1 < sort_counters ? unsigned(bucket_start[b + 1]) : sorted_total, cap);
      unsigned position = bucket_start[b] - bucket_start[mp * sort_buckets];
      for (unsigned q = bucket_start[b]; q < b_end; ++q) {
        const unsigned j = members[q];
        if (j == i || j >= est_total) continue;
        const int16_t other = st.phi(j);
        position += phi > other || (phi == other && id > st.id(j));
      }
      if (position >= count) {
        set_error(p.status, err_cluster_capacity);
        continue;
      }
      // written once here, read by the next kernel: streaming stores (evict first), which
      // leave L2 to the staging of the events in flight
      const unsigned dst = base + region[mp] + position;
      __stcs(&out.id(dst), id);
      __stcs(&out.phi(dst), phi);
      __stcs(&out.x(dst), st.x(i));
      __stcs(&out.y(dst), st.y(i));
      __stcs(&out.z(dst), st.z(i));
    }
    if (threadIdx.x < n_module_pairs) {
      const unsigned mp = threadIdx.x;
      p.module_cluster_num[e * n_module_pairs + mp] = staged_first[mp + 1] - staged_first[mp];
    }
    // the event's slices of the global staging and of the sorted bank copies are dead
    __syncthreads();
    if (!staged_in_smem) discard_l2(stage_base, size_t(24) * est_total);
    if (sorted && sorted_in_scratch) discard_l2(sorted, size_t(4) * bt.total_sp);
  }

  // Capped for 2048 threads per SM (32 registers, no spills: eight 256-thread CTAs, or
  // twelve 128-thread ones where shared memory ends them): with the clusters staged through L2
  // (cluster_stage_capacity 0) and no event staging (cluster_blob_bytes 0) shared memory allows
  // that many; measured 2.59 -> 2.21 -> 2.13 ms per launch from six CTAs with staging.
  template<unsigned THREADS>
  __global__ void __launch_bounds__(THREADS, 2048 / THREADS) cluster_sort_kernel(ClusterSortParams p)
  {
    static_assert(THREADS == 128 || THREADS == 256, "block size");
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    unsigned bar_phase = 0;
    for_each_event(p.queue, p.in.n_events, [&](unsigned e, unsigned) { cluster_sort_event<THREADS>(p, e, &bar, bar_phase); });
  }
  template __global__ void cluster_sort_kernel<128>(ClusterSortParams p);
  template __global__ void cluster_sort_kernel<256>(ClusterSortParams p);

  // Events of the slice by raw size, largest first: a counting sort over 1024 size classes
  // of 64 bytes (order within a class is arbitrary).  One CTA of scan_threads threads.
  __global__ void __launch_bounds__(scan_threads) event_order_kernel(RawInput in, unsigned* order)
  {
    constexpr unsigned classes = 1024;
    __shared__ unsigned count[classes];
    __shared__ unsigned warp_sums[33];
    for (unsigned c = threadIdx.x; c < classes; c += blockDim.x)
      count[c] = 0;
    __syncthreads();
    auto size_class = [&](unsigned e) {
      const unsigned bytes = in.offsets[e + in.event_start + 1] - in.offsets[e + in.event_start];
      return classes - 1 - min(bytes / 64u, classes - 1); // descending size
    };
    if (in.mep_layout) {
      // no per-event blob sizes in a MEP: keep the events in order
      for (unsigned e = threadIdx.x; e < in.n_events; e += blockDim.x)
        order[e] = e;
      return;
    }
    for (unsigned e = threadIdx.x; e < in.n_events; e += blockDim.x)
      atomicAdd(&count[size_class(e)], 1u);
    __syncthreads();
    unsigned total;
    const unsigned mine = threadIdx.x < classes ? count[threadIdx.x] : 0u;
    const unsigned excl = block_exclusive_scan(mine, warp_sums, &total);
    __syncthreads();
    if (threadIdx.x < classes) count[threadIdx.x] = excl;
    __syncthreads();
    for (unsigned e = threadIdx.x; e < in.n_events; e += blockDim.x)
      order[atomicAdd(&count[size_class(e)], 1u)] = e;
  }

  // ------------------------------------------------------------------------------------
  // exclusive_scan_kernel: one CTA per job; out[0] = 0, out[i + 1] = sum(in[0..i])
  // (host_prefix_sum_t, HostPrefixSum.cpp:76-108, without the host round trip).
  // ------------------------------------------------------------------------------------
  __global__ void __launch_bounds__(scan_threads) exclusive_scan_kernel(ScanParams p)
  {
    __shared__ unsigned warp_sums[33];
    const ScanJob job = p.jobs[blockIdx.x];
    if (job.in == nullptr) return;
    unsigned carry = 0;
    constexpr unsigned per_thread = 4;
    const unsigned tile = blockDim.x * per_thread;
    for (unsigned t0 = 0; t0 < job.n; t0 += tile) {
      unsigned v[per_thread];
      unsigned s = 0;
#pragma unroll
      for (unsigned q = 0; q < per_thread; ++q) {
        const unsigned i = t0 + threadIdx.x * per_thread + q;
        v[q] = i < job.n ? job.in[i] : 0u;
        s += v[q];
      }
      unsigned total;
      unsigned excl = block_exclusive_scan(s, warp_sums, &total);
#pragma unroll
      for (unsigned q = 0; q < per_thread; ++q) {
        const unsigned i = t0 + threadIdx.x * per_thread + q;
        if (i < job.n) job.out[i] = carry + excl;
        excl += v[q];
      }
      carry += total;
    }
    if (threadIdx.x == 0) job.out[job.n] = carry;
  }

} // namespace velo
