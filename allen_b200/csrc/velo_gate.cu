// Learned seed gate: decides, before the triplet search, which hits the seeding searches as the
// middle hit h1 of a seed.  One CTA of 128 threads per event; every hit of module pairs 1..24
// (the pairs the seeding takes h1 from, SearchByTriplet.cu:165-245) gets 12 geometric features
// from its neighbours in the module pairs on either side, one hit per thread.  The 12-32-32-1
// network scores 128 hits at a time on the fifth-generation tensor cores (velo_umma.cuh): the
// inputs as a 128 x 16 bf16 tile in shared memory, tcgen05.mma by one thread into a 128 x 32
// fp32 accumulator in tensor memory, read back (tcgen05.ld) by each thread for its own row,
// ReLU and bf16 into the next tile, the second layer the same way (two K steps), the output
// unit on the CUDA cores; the hit's gate byte says whether its logit is above the model's
// threshold.  In recording mode the same features go,
// with the plain search's outcome for the hit as label, into training records.
//
// Why a gate on h1 and not a score per (h0, h1) doublet: the plain seeding searches every
// unused h1 (phase A: the h0 candidates, phase B: one h2 window per doublet) and about three in
// four of them make no seed (noise hits, the first hit of a track whose h0 partner is missing).
// Gating h1 skips both phases for those, where scoring doublets could only skip phase B and
// paid the network inside the branchy search kernel.  A track whose first h1 is gated off is
// seeded one module pair later with that hit as its h0, so efficiency barely moves.
//
// No counterpart in the reference; the features are geometric and independent of which hits are
// used, so the gate of an event is known before its search.
#include <type_traits>

#include "velo_kernels.cuh"
#include "velo_umma.cuh"

namespace velo {

  namespace {
    struct PairRange {
      unsigned start; // first hit, event-relative
      unsigned num;
    };

    struct EventHits {
      ClusterView v;      // the slice's sorted container
      unsigned offset;    // the event's first hit
      const int16_t* phi; // event-relative phi column
      __device__ __forceinline__ float x(unsigned i) const { return v.x(offset + i); }
      __device__ __forceinline__ float y(unsigned i) const { return v.y(offset + i); }
      __device__ __forceinline__ float z(unsigned i) const { return v.z(offset + i); }
    };

    __device__ __forceinline__ int16_t clamp_i16(int v) { return static_cast<int16_t>(max(-32768, min(32767, v))); }

    // hits of a module pair with phi in [phi - w, phi + w] (no wrap at +-pi), at most 16
    __device__ __forceinline__ float window_count(
      const uint16_t* table, const int16_t* phis, const PairRange& r, int16_t phi, int w)
    {
      const int lo = leftmost(table, phis + r.start, r.num, clamp_i16(int(phi) - w));
      const int hi_value = int(phi) + w + 1;
      const int hi = hi_value > 32767 ? int(r.num) : leftmost(table, phis + r.start, r.num, static_cast<int16_t>(hi_value));
      return static_cast<float>(min(hi - lo, 16));
    }

    // Features of seed candidate h1 (event-relative, on module pair m = 1..24).  fp32 with
    // correctly rounded division and square root and no contraction, so the host restatement
    // (oracle/velo_seed_oracle.py) reproduces them bit for bit:
    //  0 r(h1), 1 z(h1),
    //  2 sqrt of the smallest xy distance to the beam axis of the lines through h1 and each of
    //    its 4 h0 candidates nearest in phi on module pair m + 1 (the seeding's pendulum order,
    //    used hits included), 3 z of closest approach of that best line, 4 its slope |t|,
    //  5 sqrt of the second smallest distance,
    //  6, 7 sqrt of the smallest scatter of the first 3 hits of the h2 window (module pair m - 1)
    //    that the best and the second line open, as the seeding extrapolates (31.6: none),
    //  8, 9 hits of module pairs m + 1 and m - 1 within twice the phi tolerance (at most 16),
    //  10 smallest |phi(h1) - phi(h0)| of the 4 candidates (rad / pi), 11 phi(h1) (rad / pi).
    __device__ __forceinline__ void seed_features(
      const EventHits& h,
      const uint16_t (*bucket)[n_buckets + 1],
      const Constants& k,
      unsigned m,
      const PairRange& prev,
      const PairRange& next,
      float dz_next,
      unsigned h1,
      float (&f)[mlp_features])
    {
      const int tol = k.phi_tolerance_i16;
      const float x1 = h.x(h1), y1 = h.y(h1), z1 = h.z(h1);
      const int16_t phi1 = h.phi[h1];
      float best_d = 1000.0f, second_d = 1000.0f, best_z = 0.0f, best_t = 0.0f, min_dphi = 1.0f;
      float best_tx = 0.0f, best_ty = 0.0f, second_tx = 0.0f, second_ty = 0.0f;
      int best_h0 = -1, second_h0 = -1;
      const int n_prev = static_cast<int>(prev.num);
      int pos = leftmost(bucket[m + 1], h.phi + prev.start, prev.num, phi1);
      for (int i = 0; i < n_prev && i < 4; ++i) {
        pos += (i & 1) ? i : -i;
        const int in_bounds = pos < 0 ? pos + n_prev : (pos >= n_prev ? pos - n_prev : pos);
        const unsigned h0 = prev.start + static_cast<unsigned>(in_bounds);
        const float x0 = h.x(h0), y0 = h.y(h0), z0 = h.z(h0);
        const float inv = __fdiv_rn(1.0f, z1 - z0);
        const float tx = (x1 - x0) * inv;
        const float ty = (y1 - y0) * inv;
        const float t2 = tx * tx + ty * ty;
        const float t = __fsqrt_rn(t2);
        const float d = __fdiv_rn(fabsf(x1 * ty - y1 * tx), fmaxf(t, 1e-6f));
        const float dphi =
          static_cast<float>(abs(static_cast<int>(static_cast<int16_t>(phi1 - h.phi[h0])))) * 3.0517578125e-05f;
        min_dphi = fminf(min_dphi, dphi);
        if (d < best_d) {
          second_d = best_d;
          second_h0 = best_h0;
          second_tx = best_tx;
          second_ty = best_ty;
          best_d = d;
          best_h0 = static_cast<int>(h0);
          best_tx = tx;
          best_ty = ty;
          best_z = z1 - __fdiv_rn(x1 * tx + y1 * ty, fmaxf(t2, 1e-12f));
          best_t = t;
        }
        else if (d < second_d) {
          second_d = d;
          second_h0 = static_cast<int>(h0);
          second_tx = tx;
          second_ty = ty;
        }
      }
      float scatter[2] = {1000.0f, 1000.0f};
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int h0i = c == 0 ? best_h0 : second_h0;
        if (h0i < 0 || next.num == 0) continue;
        const unsigned h0 = static_cast<unsigned>(h0i);
        const float tx = c == 0 ? best_tx : second_tx, ty = c == 0 ? best_ty : second_ty;
        const float x0 = h.x(h0), y0 = h.y(h0), z0 = h.z(h0);
        // find_forward_candidate (SearchByTriplet.cu:272-292), as the seeding extrapolates
        const float xp = x0 + tx * dz_next;
        const float yp = y0 + ty * dz_next;
        const int16_t phi_p = hit_phi_16(k, xp, yp);
        const int16_t lo = static_cast<int16_t>(phi_p - static_cast<int16_t>(tol));
        const int start = static_cast<int16_t>(leftmost(bucket[m - 1], h.phi + next.start, next.num, lo));
        unsigned idx = static_cast<unsigned>(start) % next.num;
        for (unsigned j = 0; j < next.num && j < 3; ++j, idx = (idx + 1 == next.num) ? 0u : idx + 1) {
          const unsigned h2 = next.start + idx;
          const int16_t diff = static_cast<int16_t>(h.phi[h2] - phi_p);
          if (abs(static_cast<int>(diff)) > tol) break;
          const float dz = h.z(h2) - z0;
          const float dx = (x0 + tx * dz) - h.x(h2);
          const float dy = (y0 + ty * dz) - h.y(h2);
          scatter[c] = fminf(scatter[c], dx * dx + dy * dy);
        }
      }
      f[0] = __fsqrt_rn(x1 * x1 + y1 * y1);
      f[1] = z1;
      f[2] = __fsqrt_rn(best_d);
      f[3] = best_z;
      f[4] = best_t;
      f[5] = __fsqrt_rn(second_d);
      f[6] = __fsqrt_rn(scatter[0]);
      f[7] = __fsqrt_rn(scatter[1]);
      f[8] = window_count(bucket[m + 1], h.phi, prev, phi1, 2 * tol);
      f[9] = window_count(bucket[m - 1], h.phi, next, phi1, 2 * tol);
      f[10] = min_dphi;
      f[11] = static_cast<float>(phi1) * 3.0517578125e-05f;
    }
  } // namespace

  // Shared state of the gate kernel's network (inference): the 128-row input and hidden tiles,
  // the weight tiles (B operands, N = 32 rows), the MMA completion barrier and the TMEM base.
  struct GateMlpShared {
    alignas(128) unsigned char a1[gate_threads * mlp_k1 * 2];    // inputs, 128 x 16 bf16
    alignas(128) unsigned char a2[gate_threads * mlp_hidden * 2]; // layer-1 outputs, 128 x 32 bf16
    alignas(128) unsigned char w1[mlp_hidden * mlp_k1 * 2];       // W1, 32 x 16 bf16
    alignas(128) unsigned char w2[mlp_hidden * mlp_hidden * 2];   // W2, 32 x 32 bf16
    uint64_t bar;
    uint32_t tmem;
  };
  constexpr unsigned gate_tmem_columns = 32; // one 128 x 32 fp32 accumulator, reused by both layers
  constexpr unsigned gate_wait_limit = 1u << 22;

  __device__ __forceinline__ void put_u32(unsigned char* tile, unsigned r, unsigned k, unsigned K, uint32_t v)
  {
    *reinterpret_cast<uint32_t*>(tile + umma::tile_offset(r, k, K)) = v;
  }

  template<bool RECORD>
  __global__ void __launch_bounds__(gate_threads) seed_gate_kernel(GateParams p)
  {
    __shared__ uint16_t bucket[n_module_pairs][n_buckets + 1];
    __shared__ unsigned start[n_module_pairs + 1]; // event-relative first hit of each module pair
    __shared__ unsigned num[n_module_pairs];
    __shared__ unsigned first_item[n_module_pairs]; // candidates before module pair m (m = 1..24)
    __shared__ unsigned kept_count;
    __shared__ std::conditional_t<RECORD, int, GateMlpShared> mlp;
    const unsigned e = blockIdx.x;
    const unsigned T = p.offsets_estimated_input_size[p.n_events * n_module_pairs];
    if (T > p.cluster_capacity) return; // flagged by the clustering kernel (before any TMEM is held)
    const unsigned* g_start = p.offsets_estimated_input_size + e * n_module_pairs;
    const unsigned* g_num = p.module_cluster_num + e * n_module_pairs;
    const unsigned hit_offset = g_start[0];
    const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (tid < n_module_pairs) {
      start[tid] = g_start[tid] - hit_offset;
      num[tid] = g_num[tid];
    }
    if (tid == 0) kept_count = 0;
    __syncthreads();
    if (tid == 0) {
      unsigned s = 0;
      for (unsigned m = 0; m < n_module_pairs; ++m) {
        first_item[m] = s;
        if (m >= 1 && m <= n_module_pairs - 2) s += num[m];
      }
      start[n_module_pairs] = s; // the event's seed candidates
    }
    const EventHits h {ClusterView {const_cast<char*>(p.sorted_container), T}, hit_offset,
                       ClusterView {const_cast<char*>(p.sorted_container), T}.phi_begin() + hit_offset};
    build_bucket_tables(bucket, h.phi, g_start, g_num, hit_offset);
    uint32_t tmem = 0;
    unsigned phase = 0;
    if constexpr (!RECORD) {
      // TMEM for the accumulator, the barrier, the weights in their canonical tiles
      if (warp == 0) umma::alloc(&mlp.tmem, gate_tmem_columns);
      if (tid == 0) umma::mbar_init(&mlp.bar, 1);
      for (unsigned i = tid; i < mlp_hidden * (mlp_k1 / 2); i += blockDim.x)
        put_u32(mlp.w1, i / (mlp_k1 / 2), 2 * (i % (mlp_k1 / 2)), mlp_k1, __ldg(&p.model->w1[0][0] + i));
      for (unsigned i = tid; i < mlp_hidden * (mlp_hidden / 2); i += blockDim.x)
        put_u32(mlp.w2, i / (mlp_hidden / 2), 2 * (i % (mlp_hidden / 2)), mlp_hidden, __ldg(&p.model->w2[0][0] + i));
      umma::fence_async_shared();
      umma::fence_before_sync();
    }
    __syncthreads();
    if constexpr (!RECORD) {
      umma::fence_after_sync();
      tmem = mlp.tmem;
    }
    const unsigned n_items = start[n_module_pairs];
    const Constants k = p.k;
    constexpr uint32_t idesc = umma::idesc_bf16(gate_threads, mlp_hidden);
    bool failed = false;
    // one candidate per thread, 128 per tile
    for (unsigned base = 0; base < n_items; base += blockDim.x) {
      const unsigned item = base + tid;
      unsigned h1 = 0xFFFFFFFFu;
      float f[mlp_features];
      bool active = item < n_items;
      unsigned m = 1;
      if (active) {
        // the candidate's module pair: the last m with first_item[m] <= item (binary search)
        unsigned lo = 1, hi = n_module_pairs - 2;
        while (lo < hi) {
          const unsigned mid = (lo + hi + 1) / 2;
          if (first_item[mid] <= item) lo = mid;
          else hi = mid - 1;
        }
        m = lo;
        h1 = start[m] + (item - first_item[m]);
      }
      if constexpr (RECORD) {
        if (active) {
          const uint8_t outcome = p.h1_outcome[hit_offset + h1];
          active = outcome != 0 && ((e * 0x9E3779B1u) ^ ((hit_offset + h1) * 0x85EBCA77u)) % p.record_every == 0;
          if (active) {
            const float dz_next = __ldg(p.geo->module_zs + 2 * (m - 1)) - __ldg(p.geo->module_zs + 2 * (m + 1));
            seed_features(h, bucket, k, m, PairRange {start[m + 1], num[m + 1]}, PairRange {start[m - 1], num[m - 1]},
                          dz_next, h1, f);
            const unsigned slot = atomicAdd(p.record_count, 1u);
            if (slot < p.record_capacity) {
              SeedRecord r;
#pragma unroll
              for (unsigned i = 0; i < mlp_features; ++i)
                r.f[i] = f[i];
              r.label = outcome == 2 ? 1.0f : 0.0f;
              r.event = e;
              r.h0 = 0xFFFFFFFFu;
              r.h1 = hit_offset + h1;
              p.records[slot] = r;
            }
          }
        }
      }
      else {
        // layer 1: the standardised bf16 inputs as row tid of the input tile
        uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (active) {
          const float dz_next = __ldg(p.geo->module_zs + 2 * (m - 1)) - __ldg(p.geo->module_zs + 2 * (m + 1));
          seed_features(h, bucket, k, m, PairRange {start[m + 1], num[m + 1]}, PairRange {start[m - 1], num[m - 1]},
                        dz_next, h1, f);
          standardise_pairs(*p.model, f, w);
        }
#pragma unroll
        for (unsigned i = 0; i < 8; ++i)
          put_u32(mlp.a1, tid, 2 * i, mlp_k1, w[i]);
        umma::fence_async_shared();
        __syncthreads();
        if (tid == 0) {
          umma::fence_after_sync();
          umma::mma(tmem, umma::desc(mlp.a1, mlp_k1, 0), umma::desc(mlp.w1, mlp_k1, 0), idesc, false);
          umma::commit(&mlp.bar);
        }
        failed = __syncthreads_or(!umma::mbar_wait(&mlp.bar, phase, gate_wait_limit));
        phase ^= 1u;
        if (failed) break;
        umma::fence_after_sync();
        float acc[32];
        umma::load32(tmem + ((warp * 32u) << 16), acc);
        // layer 2: bias, ReLU, bf16 as row tid of the hidden tile
#pragma unroll
        for (unsigned i = 0; i < mlp_hidden / 2; ++i)
          put_u32(mlp.a2, tid, 2 * i, mlp_hidden,
                  pack_bf16(relu(acc[2 * i] + __ldg(&p.model->b1[2 * i])), relu(acc[2 * i + 1] + __ldg(&p.model->b1[2 * i + 1]))));
        umma::fence_before_sync();
        umma::fence_async_shared();
        __syncthreads();
        if (tid == 0) {
          umma::fence_after_sync();
          umma::mma(tmem, umma::desc(mlp.a2, mlp_hidden, 0), umma::desc(mlp.w2, mlp_hidden, 0), idesc, false);
          umma::mma(tmem, umma::desc(mlp.a2, mlp_hidden, 1), umma::desc(mlp.w2, mlp_hidden, 1), idesc, true);
          umma::commit(&mlp.bar);
        }
        failed = __syncthreads_or(!umma::mbar_wait(&mlp.bar, phase, gate_wait_limit));
        phase ^= 1u;
        if (failed) break;
        umma::fence_after_sync();
        umma::load32(tmem + ((warp * 32u) << 16), acc);
        // layer 3 on the CUDA cores: the bf16 hidden units against W3 (fp32 values of bf16 weights)
        float logit = __ldg(&p.model->b3);
#pragma unroll
        for (unsigned i = 0; i < mlp_hidden; ++i) {
          const float a = __uint_as_float(pack_bf16(relu(acc[i] + __ldg(&p.model->b2[i])), 0.0f) << 16);
          logit += a * __ldg(&p.model->w3f[i]);
        }
        if (active) {
          const bool keep = logit > __ldg(&p.model->threshold_logit);
          p.gate[hit_offset + h1] = keep ? 1 : 0;
          if (keep) atomicAdd(&kept_count, 1u);
        }
        umma::fence_before_sync();
        __syncthreads(); // the tiles and the accumulator are free for the next candidates
      }
    }
    if constexpr (!RECORD) {
      if (failed) {
        // an MMA that did not complete in time: flag it, let it drain (bounded), keep no gate
        if (tid == 0) set_error(p.status, err_mma_timeout);
        __syncthreads_or(!umma::mbar_wait(&mlp.bar, phase ^ 1u, gate_wait_limit)); // the phase that timed out
      }
      __syncthreads();
      if (warp == 0) umma::dealloc(tmem, gate_tmem_columns);
      if (tid == 0) {
        p.gate_stats[2 * e] = n_items;
        p.gate_stats[2 * e + 1] = failed ? 0u : kept_count;
      }
    }
  }

  template __global__ void seed_gate_kernel<false>(GateParams p);
  template __global__ void seed_gate_kernel<true>(GateParams p);

} // namespace velo
