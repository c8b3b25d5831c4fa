// Retina-cluster decoding on sm_100a: the VELO front end for VPRetinaCluster banks (type 73),
// whose words already hold a cluster's column, row and fraction.  Replaces
// calculate_number_of_retinaclusters_each_sensor_pair, its prefix sum and decode_retinaclusters
// (device/velo/retinacluster_decoding/src/CalculateNumberOfRetinaClustersPerSensor.cu:12-48,
// DecodeRetinaClusters.cu:11-383) with two kernels and one scan of per-event totals:
//
//   retina_count_kernel   [N CTAs]  clusters per sensor (pair) of each event and the event's
//                                   total; the slice's first event writes the bank index
//   exclusive_scan_kernel           event bases from the totals
//   retina_decode_kernel  [N CTAs]  per event: the sensor offsets (prefix sum inside the CTA
//                                   plus the event base), the module-pair offsets, the clusters
//                                   decoded, keyed by (phi, id), ranked inside their module
//                                   pair and written to their sorted slot
//
// Outputs are the reference's: dev_each_sensor_pair_size, dev_offsets_each_sensor_pair_size,
// dev_retina_bank_index, dev_module_cluster_num, dev_offsets_module_pair_cluster (the search's
// dev_offsets_estimated_input_size) and the sorted cluster container.  The permutation and the
// key array are intermediate and stay in shared memory (or, for events above the shared-memory
// capacity, in a global scratch slice).  Arithmetic in the reference's order and rounding, so
// every cluster is bit-identical.
#include "velo_kernels.cuh"

namespace velo {

  __device__ __forceinline__ unsigned retina_sensors(int version) { return (version == 2 || version == 3) ? n_sensors : n_sensors / 2; }

  struct RetinaBank {
    unsigned source_id, count, size, type;
    const uint32_t* word;
  };

  __device__ __forceinline__ unsigned retina_n_banks(const RawInput& in, unsigned ev)
  {
    return in.mep_layout ? mep_n_banks(in) : reinterpret_cast<const uint32_t*>(in.raw + in.offsets[ev])[0];
  }

  __device__ __forceinline__ RetinaBank retina_bank(const RawInput& in, unsigned ev, unsigned b)
  {
    const bool v23 = in.bank_version == 2 || in.bank_version == 3;
    if (in.mep_layout) {
      // MEPTools.h:55-205: the fragment starts with the bank data (no sourceID word)
      RetinaBank r;
      const uint32_t* frag = reinterpret_cast<const uint32_t*>(in.raw + mep_fragment_offset(in, ev, b));
      r.source_id = mep_source_id(in, b);
      r.count = v23 ? frag[0] : 0u;
      r.word = frag + (v23 ? 1 : 0);
      r.size = mep_bank_size(in, ev, b);
      r.type = mep_bank_type(in, ev, b);
      return r;
    }
    const char* blob = in.raw + in.offsets[ev];
    const uint32_t* w = reinterpret_cast<const uint32_t*>(blob);
    const unsigned n_banks = w[0];
    const char* payload = blob + 4 * (n_banks + 2);
    const uint32_t* bank = reinterpret_cast<const uint32_t*>(payload + w[1 + b]);
    RetinaBank r;
    r.source_id = bank[0];
    r.count = v23 ? bank[1] : 0u;
    r.word = bank + (v23 ? 2 : 1);
    r.size = bank_sizes(in, ev)[b];
    r.type = bank_types(in, ev)[b];
    return r;
  }

  // CalculateNumberOfRetinaClustersPerSensor.cu:12-48, plus the event total
  __global__ void __launch_bounds__(decode_threads) retina_count_kernel(RetinaParams p)
  {
    __shared__ unsigned warp_sums[33];
    const unsigned e = blockIdx.x, ev = e + p.in.event_start;
    const unsigned per_event = retina_sensors(p.in.bank_version);
    unsigned* size = p.each_sensor_pair_size + size_t(e) * per_event;
    for (unsigned s = threadIdx.x; s < per_event; s += blockDim.x)
      size[s] = 0;
    __syncthreads();
    const unsigned n_banks = retina_n_banks(p.in, ev);
    for (unsigned b = threadIdx.x; b < n_banks; b += blockDim.x) {
      const RetinaBank bank = retina_bank(p.in, ev, b);
      if (bank.type == bank_type_vp_retina) {
        const bool v23 = p.in.bank_version == 2 || p.in.bank_version == 3;
        const unsigned s = v23 ? bank.source_id : (bank.source_id & 0x1FFu);
        if (s < per_event) size[s] = v23 ? bank.count : bank.size / 4u;
        else set_error(p.status, err_input_capacity);
      }
      // the reference's block 0 writes every bank's number in bank order: the last wins
      if (e == 0 && (bank.source_id & 0x1FFu) < per_event) atomicMax(p.bank_index + (bank.source_id & 0x1FFu), b);
    }
    __syncthreads();
    unsigned part = 0;
    for (unsigned s = threadIdx.x; s < per_event; s += blockDim.x)
      part += size[s];
    unsigned total;
    block_exclusive_scan(part, warp_sums, &total);
    if (threadIdx.x == 0) p.event_total[e] = total;
  }

  struct RetinaCluster {
    uint32_t id;
    float x, y, z;
    int16_t phi;
    unsigned sensor;
  };

  // populate_retinacluster / populate_sorting_key (DecodeRetinaClusters.cu:80-160, 246-303)
  __device__ __forceinline__ RetinaCluster
  decode_word(const Geometry* g, const Constants& k, int version, unsigned source_id, uint32_t w)
  {
    RetinaCluster c;
    if (version == 2 || version == 3) c.sensor = source_id;
    else c.sensor = ((source_id & 0x1FFu) << 1) | ((w >> 22) & 0x1u);
    uint32_t cx, cy, or_fx, or_fy;
    float fx, fy;
    if (version == 2) {
      cx = (w >> 14) & 0x3FFu;
      fx = __fdiv_rn(__uint2float_rn((w >> 11) & 0x7u), 8.f);
      cy = (w >> 3) & 0xFFu;
      fy = __fdiv_rn(__uint2float_rn(w & 0x7FFu), 8.f);
      or_fx = 0;
      or_fy = 0;
    }
    else {
      cx = (w >> 12) & 0x3FFu;
      fx = __fdiv_rn(__uint2float_rn((w >> 10) & 0x3u), 4.f);
      cy = (w >> 2) & 0xFFu;
      fy = __fdiv_rn(__uint2float_rn(w & 0x3FFu), 4.f);
      or_fx = ((w >> 11) & 0x1u) | ((w >> 10) & 0x1u);
      or_fy = ((w >> 1) & 0x1u) | (w & 0x1u);
    }
    const unsigned sensor = c.sensor < n_sensors ? c.sensor : 0u;
    const float* ltg = g->ltg + 12 * sensor;
    const float local_x = column_local_x(g, cx) + fx * column_x_pitch(g, cx);
    const float local_y = (0.5f + fy) * 0.055f;
    c.x = __ldg(ltg + 0) * local_x + __ldg(ltg + 1) * local_y + __ldg(ltg + 9);
    c.y = __ldg(ltg + 3) * local_x + __ldg(ltg + 4) * local_y + __ldg(ltg + 10);
    c.z = __ldg(ltg + 6) * local_x + __ldg(ltg + 7) * local_y + __ldg(ltg + 11);
    c.id = lhcb_id((or_fx << 27) | (or_fy << 26) | channel_id(c.sensor, cx >> 8, cx & 0xFFu, cy));
    c.phi = hit_phi_16(k, c.x, c.y);
    return c;
  }

  // The word of cluster c (event-relative) of sensor s: the bank comes from the bank index the
  // slice's first event wrote (as in the reference); returns false, with an error flag, when
  // that bank does not exist in this event or holds fewer words than the event's counts.
  __device__ __forceinline__ bool
  cluster_word(const RetinaParams& p, unsigned ev, unsigned s, unsigned index, RetinaBank& bank, uint32_t& w)
  {
    const unsigned n_banks = retina_n_banks(p.in, ev);
    const unsigned b = p.bank_index[s];
    if (b >= n_banks) {
      set_error(p.status, err_input_capacity);
      return false;
    }
    bank = retina_bank(p.in, ev, b);
    if (bank.type != bank_type_vp_retina) return false;
    const bool v23 = p.in.bank_version == 2 || p.in.bank_version == 3;
    if (index >= (v23 ? bank.count : bank.size / 4u)) {
      set_error(p.status, err_input_capacity);
      return false;
    }
    w = bank.word[index];
    return true;
  }

  // binary_search_rightmost (BinarySearch.cuh:33-47)
  __device__ __forceinline__ unsigned rightmost(const unsigned* a, unsigned n, unsigned value)
  {
    int l = 0, r = int(n);
    while (l < r) {
      const int m = (l + r) / 2;
      if (a[m] > value) r = m;
      else l = m + 1;
    }
    return unsigned(r - 1);
  }

  // Rank buckets per module pair: the top 6 bits of the (signed) sort key, so that bucket order
  // is key order; about 1.3 clusters per bucket at nu = 7.6.
  constexpr unsigned rank_buckets = 64;
  constexpr unsigned rank_counters = n_module_pairs * rank_buckets;

  __device__ __forceinline__ unsigned key_bucket(int64_t key)
  {
    return static_cast<unsigned>(static_cast<int>(key >> 58) + 32);
  }

  // u16 counters packed two per 32-bit word; returns the previous value of counter b.
  __device__ __forceinline__ unsigned bump_u16(uint16_t* counters, unsigned b)
  {
    const unsigned shift = 16 * (b & 1u);
    const uint32_t old = atomicAdd(reinterpret_cast<uint32_t*>(counters) + (b >> 1), 1u << shift);
    return (old >> shift) & 0xFFFFu;
  }

  // Capped for eight CTAs per SM (32 registers): with the keys in L2-resident scratch the
  // shared memory (16 KB of bucket order plus about 4.5 KB of counters and offsets, 21 KB)
  // allows that many.
  __global__ void __launch_bounds__(decode_threads, 8) retina_decode_kernel(RetinaParams p)
  {
    extern __shared__ __align__(16) unsigned char dsmem[];
    __shared__ unsigned so[n_sensors + 1]; // event-relative sensor offsets
    __shared__ unsigned mp_num[n_module_pairs], mp_zero[n_module_pairs];
    __shared__ unsigned warp_sums[33];
    __shared__ __align__(4) uint16_t bucket_end[rank_counters];
    __shared__ unsigned irregular;
    const unsigned e = blockIdx.x, ev = e + p.in.event_start, n = p.in.n_events;
    const int version = p.in.bank_version;
    const unsigned per_event = retina_sensors(version);
    const unsigned step = per_event / n_module_pairs;
    const unsigned base = p.event_base[e];
    const unsigned T = p.event_base[n];
    if (T > p.cluster_capacity) {
      if (threadIdx.x == 0) set_error(p.status, err_input_capacity);
      return;
    }
    // sensor offsets: prefix sum of this event's sizes (per_event <= 208 < blockDim)
    const unsigned* size = p.each_sensor_pair_size + size_t(e) * per_event;
    const unsigned mine = threadIdx.x < per_event ? size[threadIdx.x] : 0u;
    unsigned total;
    const unsigned excl = block_exclusive_scan(mine, warp_sums, &total);
    if (threadIdx.x < per_event) {
      so[threadIdx.x] = excl;
      p.offsets_each_sensor_pair_size[size_t(e) * per_event + threadIdx.x] = base + excl;
    }
    if (threadIdx.x == 0) {
      so[per_event] = total;
      if (e == n - 1) p.offsets_each_sensor_pair_size[size_t(n) * per_event] = base + total;
      if (e == 0) p.offsets_module_pair_cluster[0] = 0;
      irregular = 0;
    }
    if (threadIdx.x < n_module_pairs) {
      mp_num[threadIdx.x] = 0;
      mp_zero[threadIdx.x] = 0;
    }
    for (unsigned i = threadIdx.x; i < rank_counters / 2; i += blockDim.x)
      reinterpret_cast<uint32_t*>(bucket_end)[i] = 0;
    __syncthreads();
    // populate_module_pair_offsets_and_sizes (DecodeRetinaClusters.cu:11-35)
    if (threadIdx.x < n_module_pairs) p.offsets_module_pair_cluster[e * n_module_pairs + threadIdx.x + 1] = base + so[(threadIdx.x + 1) * step];

    // keys in shared memory when the event fits the key capacity, else in its slice of the global
    // (L2-resident) scratch; the bucket order in shared memory behind them when the event fits the
    // order capacity, else no buckets (the full comparison)
    const bool keys_in_smem = total <= p.smem_key_capacity;
    const bool in_smem = total <= p.smem_order_capacity; // the bucketed rank
    int64_t* keys = keys_in_smem ? reinterpret_cast<int64_t*>(dsmem) : reinterpret_cast<int64_t*>(p.key_scratch) + base;
    uint16_t* order = reinterpret_cast<uint16_t*>(dsmem + size_t(p.smem_key_capacity) * sizeof(int64_t));
    const Geometry* g = p.geo;
    const Constants k = p.k;
    // velo_calculate_sorting_key (DecodeRetinaClusters.cu:162-244)
    for (unsigned c = threadIdx.x; c < total; c += blockDim.x) {
      const unsigned s = rightmost(so, per_event, c);
      RetinaBank bank;
      uint32_t w;
      int64_t key = 0x7FFFFFFFFFFFFFFFll;
      bool counted = false;
      if (cluster_word(p, ev, s, c - so[s], bank, w)) {
        const RetinaCluster cl = decode_word(g, k, version, bank.source_id, w);
        const unsigned mp = cl.sensor / 8;
        if (mp < n_module_pairs) {
          atomicAdd(w != 0 ? &mp_num[mp] : &mp_zero[mp], 1u);
          counted = mp == s / step;
        }
        if (w != 0) key = static_cast<int64_t>((static_cast<uint64_t>(static_cast<uint16_t>(cl.phi)) << 48) | cl.id);
      }
      keys[c] = key;
      if (in_smem) {
        if (counted) bump_u16(bucket_end, (s / step) * rank_buckets + key_bucket(key));
        else irregular = 1; // a cluster the module-pair counts miss: rank by the full comparison
      }
    }
    __syncthreads();
    if (threadIdx.x < n_module_pairs) p.module_cluster_num[e * n_module_pairs + threadIdx.x] = mp_num[threadIdx.x];

    // velo_calculate_permutations + decode_retinaclusters_sorted (DecodeRetinaClusters.cu:37-78,
    // 305-383): a cluster's slot is its module pair's start plus the number of smaller keys of
    // the module pair.  When every cluster was counted in its module pair's (key) buckets, the
    // buckets are laid out in order by a scan of their counts, each cluster is placed in its
    // bucket, and its rank is the bucket's start plus the smaller keys of the same bucket.
    const bool bucketed = in_smem && !irregular;
    if (bucketed) {
      constexpr unsigned per = (rank_counters + decode_threads - 1) / decode_threads;
      unsigned v[per];
      unsigned sum = 0;
#pragma unroll
      for (unsigned q = 0; q < per; ++q) {
        const unsigned b = threadIdx.x * per + q;
        v[q] = b < rank_counters ? bucket_end[b] : 0u;
        sum += v[q];
      }
      unsigned all;
      unsigned run = block_exclusive_scan(sum, warp_sums, &all);
      __syncthreads(); // every count read before the starts overwrite them
#pragma unroll
      for (unsigned q = 0; q < per; ++q) {
        const unsigned b = threadIdx.x * per + q;
        if (b < rank_counters) bucket_end[b] = static_cast<uint16_t>(run); // start; the fill below ends it
        run += v[q];
      }
      __syncthreads();
      for (unsigned c = threadIdx.x; c < total; c += blockDim.x) {
        const unsigned s = rightmost(so, per_event, c);
        order[bump_u16(bucket_end, (s / step) * rank_buckets + key_bucket(keys[c]))] = static_cast<uint16_t>(c);
      }
      __syncthreads();
    }
    ClusterView out {p.container, T};
    for (unsigned c = threadIdx.x; c < total; c += blockDim.x) {
      const unsigned s = rightmost(so, per_event, c);
      RetinaBank bank;
      uint32_t w;
      if (!cluster_word(p, ev, s, c - so[s], bank, w)) continue;
      const unsigned mp = s / step;
      const unsigned start = so[mp * step];
      const int64_t key = keys[c];
      unsigned position = 0;
      if (bucketed) {
        const unsigned b = mp * rank_buckets + key_bucket(key);
        const unsigned first = b ? bucket_end[b - 1] : 0u, last = bucket_end[b];
        position = first - start;
        for (unsigned i = first; i < last; ++i)
          position += key > keys[order[i]];
      }
      else {
        const unsigned num = min(mp_num[mp] + mp_zero[mp], total - start);
        for (unsigned j = 0; j < num; ++j)
          position += (start + j != c) && key > keys[start + j];
      }
      const RetinaCluster cl = decode_word(g, k, version, bank.source_id, w);
      const unsigned dst = base + start + position;
      if (dst >= T) {
        set_error(p.status, err_cluster_capacity);
        continue;
      }
      out.id(dst) = cl.id;
      out.x(dst) = cl.x;
      out.y(dst) = cl.y;
      out.z(dst) = cl.z;
      out.phi(dst) = cl.phi;
    }
  }

} // namespace velo
