// Training of the learned seed pruner on sm_100a, and the host conversion of a model to
// its device form.  No counterpart in the reference (see velo_mlp.cuh).
//
// mlp_train_kernel: 128-record tiles on the fifth-generation tensor cores (tcgen05.mma from
// shared-memory tiles into tensor memory, velo_umma.cuh), one record per thread for the
// element-wise work; the weight gradients of both layers accumulate in tensor memory over the
// CTA's tiles and go to the global fp32 gradient once per CTA.  adam_kernel updates the fp32
// master weights and publish_kernel writes the bf16 copies the kernels read.
// mlp_score_kernel (logits of records, for the threshold calibration) stays on warp-level
// mma.sync tiles of 16 records.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "velo_b200.h"
#include "velo_mlp.cuh"
#include "velo_umma.cuh"

namespace velo_host {
  void set_last_error(const std::string& what); // velo_chain.cu
}

namespace velo {

  constexpr unsigned n_params = VELO_SEED_PARAMS;
  constexpr unsigned off_w1 = 0, off_b1 = 384, off_w2 = 416, off_b2 = 1440, off_w3 = 1472, off_b3 = 1504;
  static_assert(off_b3 + 1 == n_params, "parameter layout");

  uint16_t host_bf16(float v)
  {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return static_cast<uint16_t>((u >> 16) | ((u & 0xFFFFu) ? 0x40u : 0u));
    u += 0x7FFFu + ((u >> 16) & 1u); // round to nearest, ties to even
    return static_cast<uint16_t>(u >> 16);
  }

  float host_bf16_value(float v)
  {
    const uint32_t u = uint32_t(host_bf16(v)) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  }

  // Flat parameters (w1, b1, w2, b2, w3, b3) plus the model's standardisation and bounds.
  void make_model_device(const float* params, const VeloSeedModel& meta, MlpModelDevice& d)
  {
    std::memset(&d, 0, sizeof(d));
    auto pair = [](float lo, float hi) { return uint32_t(host_bf16(lo)) | (uint32_t(host_bf16(hi)) << 16); };
    const float* w1 = params + off_w1;
    const float* w2 = params + off_w2;
    const float* w3 = params + off_w3;
    for (unsigned o = 0; o < mlp_hidden; ++o) {
      for (unsigned i = 0; i < mlp_k1 / 2; ++i) {
        const float lo = 2 * i < mlp_features ? w1[o * mlp_features + 2 * i] : 0.0f;
        const float hi = 2 * i + 1 < mlp_features ? w1[o * mlp_features + 2 * i + 1] : 0.0f;
        d.w1[o][i] = pair(lo, hi);
      }
      for (unsigned i = 0; i < mlp_hidden / 2; ++i) {
        d.w2[o][i] = pair(w2[o * mlp_hidden + 2 * i], w2[o * mlp_hidden + 2 * i + 1]);
        d.w2t[o][i] = pair(w2[(2 * i) * mlp_hidden + o], w2[(2 * i + 1) * mlp_hidden + o]);
      }
      d.b1[o] = params[off_b1 + o];
      d.b2[o] = params[off_b2 + o];
      d.w3f[o] = host_bf16_value(w3[o]);
    }
    for (unsigned i = 0; i < mlp_hidden / 2; ++i)
      d.w3[0][i] = pair(w3[2 * i], w3[2 * i + 1]);
    d.b3 = params[off_b3];
    for (unsigned i = 0; i < mlp_features; ++i) {
      d.mean[i] = meta.mean[i];
      d.inv_std[i] = meta.inv_std[i];
    }
    d.threshold_logit = meta.threshold_logit;
    d.kept_lo = meta.kept_lo;
    d.kept_hi = meta.kept_hi;
  }

  void model_params(const VeloSeedModel& m, float* params)
  {
    std::memcpy(params + off_w1, m.w1, sizeof(m.w1));
    std::memcpy(params + off_b1, m.b1, sizeof(m.b1));
    std::memcpy(params + off_w2, m.w2, sizeof(m.w2));
    std::memcpy(params + off_b2, m.b2, sizeof(m.b2));
    std::memcpy(params + off_w3, m.w3, sizeof(m.w3));
    params[off_b3] = m.b3;
  }

} // namespace velo

namespace velo {

  struct TrainParams {
    const SeedRecord* records;
    unsigned long long first;
    unsigned batch;
    float inv_batch;
    float pos_weight;
    const MlpModelDevice* model;
    float* grads; // [n_params], accumulated
    float* loss;  // [1], accumulated (sum of weighted losses / batch)
  };

  // Standardised input of one record, feature i (0 beyond the 12 features or the batch).
  __device__ __forceinline__ float train_input(const MlpModelDevice& m, const SeedRecord* r, bool valid, unsigned i)
  {
    if (!valid || i >= mlp_features) return 0.0f;
    return fminf(fmaxf((__ldg(&r->f[i]) - __ldg(&m.mean[i])) * __ldg(&m.inv_std[i]), -8.0f), 8.0f);
  }

  // Shared tiles of the tcgen05 training kernel (canonical no-swizzle K-major bf16 tiles,
  // velo_umma.cuh).  The weight gradients of both layers come from one MMA chain: A holds
  // dZ2^T in rows 0..31 and dZ1^T in rows 32..63 (rows 64..127 zero), B holds a2^T in rows
  // 0..31 and x^T in rows 32..47, K runs over the tile's 128 records; D[0..31][0..31] is dW2 and
  // D[32..63][32..47] dW1 (the cross terms are not read), accumulated in TMEM over the tiles.
  struct TrainShared {
    alignas(128) unsigned char x[train_rows * mlp_k1 * 2];        // 128 x 16: layer-1 inputs
    alignas(128) unsigned char a2[train_rows * mlp_hidden * 2];   // 128 x 32: layer-2 inputs
    alignas(128) unsigned char e2[train_rows * mlp_hidden * 2];   // 128 x 32: dZ2 (A of dH1 = dZ2 W2)
    alignas(128) unsigned char ga[train_rows * train_rows * 2];   // 128 x 128: [dZ2^T; dZ1^T; 0]
    alignas(128) unsigned char gb[48 * train_rows * 2];           // 48 x 128: [a2^T; x^T]
    alignas(128) unsigned char w1[mlp_hidden * mlp_k1 * 2];       // W1 (B of layer 1)
    alignas(128) unsigned char w2[mlp_hidden * mlp_hidden * 2];   // W2 (B of layer 2)
    alignas(128) unsigned char w2t[mlp_hidden * mlp_hidden * 2];  // W2^T (B of dH1)
    uint64_t bar;
    uint32_t tmem;
    float sums[3 * mlp_hidden + 2]; // gb1, gb2, gw3, gb3, loss of the CTA
  };
  constexpr unsigned train_tmem_columns = 128; // 32 for the layer outputs, 48 for the gradients
  constexpr unsigned train_wait_limit = 1u << 22;

  __device__ __forceinline__ void put_bf16(unsigned char* tile, unsigned r, unsigned k, unsigned K, float v)
  {
    *reinterpret_cast<__nv_bfloat16*>(tile + umma::tile_offset(r, k, K)) = __float2bfloat16_rn(v);
  }
  __device__ __forceinline__ void put_pair(unsigned char* tile, unsigned r, unsigned k, unsigned K, uint32_t v)
  {
    *reinterpret_cast<uint32_t*>(tile + umma::tile_offset(r, k, K)) = v;
  }
  __device__ __forceinline__ void put_half(unsigned char* tile, unsigned r, unsigned k, unsigned K, uint32_t v)
  {
    *reinterpret_cast<uint16_t*>(tile + umma::tile_offset(r, k, K)) = static_cast<uint16_t>(v);
  }

  // One MMA chain of this CTA: issue (thread 0), commit, wait in every thread (bounded).  False
  // in every thread if the MMAs did not complete in time.
  template<typename Issue>
  __device__ __forceinline__ bool run_mma(TrainShared& s, unsigned& phase, Issue issue)
  {
    umma::fence_before_sync();
    umma::fence_async_shared();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
      issue();
      umma::commit(&s.bar);
    }
    const bool failed = __syncthreads_or(!umma::mbar_wait(&s.bar, phase, train_wait_limit));
    phase ^= 1u;
    umma::fence_after_sync();
    return !failed;
  }

  // Forward and backward passes over 128-record tiles on the fifth-generation tensor cores, one
  // record per thread: tcgen05.mma issued by thread 0 from shared-memory tiles into TMEM (the
  // 128 x 32 layer outputs, then dH1 = dZ2 W2, then the weight gradients accumulated over the
  // CTA's tiles), tcgen05.ld back per row; bias, ReLU, the output unit and the loss on the CUDA
  // cores with the same bf16 rounding points as the inference.
  __global__ void __launch_bounds__(train_rows) mlp_train_kernel(TrainParams p)
  {
    extern __shared__ __align__(128) unsigned char train_smem[];
    TrainShared& s = *reinterpret_cast<TrainShared*>(train_smem);
    const unsigned tid = threadIdx.x, warp = tid >> 5;
    const MlpModelDevice& m = *p.model;
    if (warp == 0) umma::alloc(&s.tmem, train_tmem_columns);
    if (tid == 0) umma::mbar_init(&s.bar, 1);
    for (unsigned i = tid; i < sizeof(s.ga) / 4; i += blockDim.x)
      reinterpret_cast<uint32_t*>(s.ga)[i] = 0u;
    for (unsigned i = tid; i < 3 * mlp_hidden + 2; i += blockDim.x)
      s.sums[i] = 0.0f;
    for (unsigned i = tid; i < mlp_hidden * (mlp_k1 / 2); i += blockDim.x)
      put_pair(s.w1, i / (mlp_k1 / 2), 2 * (i % (mlp_k1 / 2)), mlp_k1, __ldg(&m.w1[0][0] + i));
    for (unsigned i = tid; i < mlp_hidden * (mlp_hidden / 2); i += blockDim.x) {
      put_pair(s.w2, i / (mlp_hidden / 2), 2 * (i % (mlp_hidden / 2)), mlp_hidden, __ldg(&m.w2[0][0] + i));
      put_pair(s.w2t, i / (mlp_hidden / 2), 2 * (i % (mlp_hidden / 2)), mlp_hidden, __ldg(&m.w2t[0][0] + i));
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = s.tmem, lane_base = (warp * 32u) << 16;
    const uint32_t t_out = tmem, t_grad = tmem + 32u;
    constexpr uint32_t id32 = umma::idesc_bf16(train_rows, mlp_hidden);
    constexpr uint32_t id48 = umma::idesc_bf16(train_rows, 48);
    unsigned phase = 0;
    bool ok = true, grads_started = false;
    float gb1[mlp_hidden] = {}, gb2[mlp_hidden] = {}, gw3[mlp_hidden] = {};
    float gb3 = 0.0f, loss = 0.0f;
    const unsigned n_tiles = (p.batch + train_rows - 1) / train_rows;
    for (unsigned t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
      const unsigned r = t * train_rows + tid;
      const bool valid = r < p.batch;
      const SeedRecord* rec = p.records + p.first + (valid ? r : 0);
      // inputs: row tid of x, column tid of x^T (rows 32..47 of B)
#pragma unroll
      for (unsigned i = 0; i < mlp_k1; i += 2) {
        const uint32_t pr = pack_bf16(train_input(m, rec, valid, i), train_input(m, rec, valid, i + 1));
        put_pair(s.x, tid, i, mlp_k1, pr);
        put_half(s.gb, 32 + i, tid, train_rows, pr);
        put_half(s.gb, 33 + i, tid, train_rows, pr >> 16);
      }
      // layer 1
      ok = run_mma(s, phase, [&] { umma::mma(t_out, umma::desc(s.x, mlp_k1, 0), umma::desc(s.w1, mlp_k1, 0), id32, false); });
      if (!ok) break;
      float h1[mlp_hidden];
      umma::load32(t_out + lane_base, h1);
#pragma unroll
      for (unsigned i = 0; i < mlp_hidden; i += 2) {
        h1[i] += __ldg(&m.b1[i]);
        h1[i + 1] += __ldg(&m.b1[i + 1]);
        const uint32_t pr = pack_bf16(relu(h1[i]), relu(h1[i + 1]));
        put_pair(s.a2, tid, i, mlp_hidden, pr);
        put_half(s.gb, i, tid, train_rows, pr);
        put_half(s.gb, i + 1, tid, train_rows, pr >> 16);
      }
      // layer 2
      ok = run_mma(s, phase, [&] {
        umma::mma(t_out, umma::desc(s.a2, mlp_hidden, 0), umma::desc(s.w2, mlp_hidden, 0), id32, false);
        umma::mma(t_out, umma::desc(s.a2, mlp_hidden, 1), umma::desc(s.w2, mlp_hidden, 1), id32, true);
      });
      if (!ok) break;
      float h2[mlp_hidden];
      umma::load32(t_out + lane_base, h2);
      // output unit, loss, dZ2
      float z = __ldg(&m.b3);
#pragma unroll
      for (unsigned i = 0; i < mlp_hidden; ++i) {
        h2[i] += __ldg(&m.b2[i]);
        z += bf16_lo(pack_bf16(relu(h2[i]), 0.0f)) * __ldg(&m.w3f[i]);
      }
      float dz = 0.0f;
      if (valid) {
        const float y = __ldg(&rec->label);
        const float w = y > 0.5f ? p.pos_weight : 1.0f;
        const float prob = 1.0f / (1.0f + expf(-z));
        dz = w * (prob - y) * p.inv_batch;
        loss += w * (fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z))));
      }
      gb3 += dz;
#pragma unroll
      for (unsigned i = 0; i < mlp_hidden; i += 2) {
        const float a0 = bf16_lo(pack_bf16(relu(h2[i]), 0.0f)), a1 = bf16_lo(pack_bf16(relu(h2[i + 1]), 0.0f));
        gw3[i] += dz * a0;
        gw3[i + 1] += dz * a1;
        const float d0 = h2[i] > 0.0f ? dz * __ldg(&m.w3f[i]) : 0.0f;
        const float d1 = h2[i + 1] > 0.0f ? dz * __ldg(&m.w3f[i + 1]) : 0.0f;
        gb2[i] += d0;
        gb2[i + 1] += d1;
        const uint32_t pr = pack_bf16(d0, d1);
        put_pair(s.e2, tid, i, mlp_hidden, pr);
        put_half(s.ga, i, tid, train_rows, pr);
        put_half(s.ga, i + 1, tid, train_rows, pr >> 16);
      }
      // dH1 = dZ2 W2 (B: W2^T, K-major over the layer-2 units)
      ok = run_mma(s, phase, [&] {
        umma::mma(t_out, umma::desc(s.e2, mlp_hidden, 0), umma::desc(s.w2t, mlp_hidden, 0), id32, false);
        umma::mma(t_out, umma::desc(s.e2, mlp_hidden, 1), umma::desc(s.w2t, mlp_hidden, 1), id32, true);
      });
      if (!ok) break;
      float d1[mlp_hidden];
      umma::load32(t_out + lane_base, d1);
#pragma unroll
      for (unsigned i = 0; i < mlp_hidden; ++i) {
        const float v = h1[i] > 0.0f ? d1[i] : 0.0f;
        gb1[i] += v;
        put_bf16(s.ga, 32 + i, tid, train_rows, v);
      }
      // weight gradients of both layers, accumulated in TMEM over the tiles
      const bool acc = grads_started;
      ok = run_mma(s, phase, [&] {
#pragma unroll
        for (unsigned k = 0; k < train_rows / 16; ++k)
          umma::mma(t_grad, umma::desc(s.ga, train_rows, k), umma::desc(s.gb, train_rows, k), id48, acc || k > 0);
      });
      grads_started = true;
    }
    // per-thread sums into the CTA's sums, then the global gradient
#pragma unroll
    for (unsigned i = 0; i < mlp_hidden; ++i) {
      atomicAdd(&s.sums[i], gb1[i]);
      atomicAdd(&s.sums[mlp_hidden + i], gb2[i]);
      atomicAdd(&s.sums[2 * mlp_hidden + i], gw3[i]);
    }
    atomicAdd(&s.sums[3 * mlp_hidden], gb3);
    atomicAdd(&s.sums[3 * mlp_hidden + 1], loss);
    __syncthreads();
    if (ok && grads_started) {
      float g[32];
      if (warp == 0) { // rows 0..31: dW2[j][i], TMEM columns 32..63
        umma::load32(t_grad + lane_base, g);
        for (unsigned i = 0; i < mlp_hidden; ++i)
          atomicAdd(&p.grads[off_w2 + (tid & 31u) * mlp_hidden + i], g[i]);
      }
      else if (warp == 1) { // rows 32..63: dW1[j][f], TMEM columns 64..75
        umma::load32(t_grad + lane_base + 32u, g);
        for (unsigned f = 0; f < mlp_features; ++f)
          atomicAdd(&p.grads[off_w1 + (tid & 31u) * mlp_features + f], g[f]);
      }
    }
    else if (!ok) {
      // an MMA chain that did not complete in time: let it drain (bounded), then mark the step
      // failed with a NaN in b3's gradient, which the optimiser carries into the weights
      umma::mbar_wait(&s.bar, phase ^ 1u, train_wait_limit);
      if (tid == 0) p.grads[off_b3] = __int_as_float(0x7FC00000);
    }
    for (unsigned i = tid; i < mlp_hidden; i += blockDim.x) {
      atomicAdd(&p.grads[off_b1 + i], s.sums[i]);
      atomicAdd(&p.grads[off_b2 + i], s.sums[mlp_hidden + i]);
      atomicAdd(&p.grads[off_w3 + i], s.sums[2 * mlp_hidden + i]);
    }
    if (tid == 0) {
      atomicAdd(&p.grads[off_b3], s.sums[3 * mlp_hidden]);
      atomicAdd(p.loss, s.sums[3 * mlp_hidden + 1] * p.inv_batch);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::dealloc(tmem, train_tmem_columns);
  }

} // namespace velo

namespace velo {

  struct AdamParams {
    float* params; // fp32 master weights [n_params]
    float* m;
    float* v;
    float* grads;  // zeroed after the update
    float lr, beta1, beta2, eps, correction1, correction2;
  };

  __global__ void adam_kernel(AdamParams a)
  {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_params) return;
    const float g = a.grads[i];
    const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * g;
    const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    a.params[i] -= a.lr * (m / a.correction1) / (sqrtf(v / a.correction2) + a.eps);
    a.grads[i] = 0.0f;
  }

  // The bf16 device form of the master weights (layout of make_model_device).
  __global__ void publish_kernel(const float* params, MlpModelDevice* d)
  {
    const unsigned t = threadIdx.x;
    for (unsigned idx = t; idx < mlp_hidden * (mlp_k1 / 2); idx += blockDim.x) {
      const unsigned o = idx / (mlp_k1 / 2), i = idx % (mlp_k1 / 2);
      const float lo = 2 * i < mlp_features ? params[off_w1 + o * mlp_features + 2 * i] : 0.0f;
      const float hi = 2 * i + 1 < mlp_features ? params[off_w1 + o * mlp_features + 2 * i + 1] : 0.0f;
      d->w1[o][i] = pack_bf16(lo, hi);
    }
    for (unsigned idx = t; idx < mlp_hidden * (mlp_hidden / 2); idx += blockDim.x) {
      const unsigned o = idx / (mlp_hidden / 2), i = idx % (mlp_hidden / 2);
      d->w2[o][i] = pack_bf16(params[off_w2 + o * mlp_hidden + 2 * i], params[off_w2 + o * mlp_hidden + 2 * i + 1]);
      d->w2t[o][i] =
        pack_bf16(params[off_w2 + (2 * i) * mlp_hidden + o], params[off_w2 + (2 * i + 1) * mlp_hidden + o]);
    }
    if (t < mlp_hidden / 2) d->w3[0][t] = pack_bf16(params[off_w3 + 2 * t], params[off_w3 + 2 * t + 1]);
    if (t < mlp_hidden) {
      d->b1[t] = params[off_b1 + t];
      d->b2[t] = params[off_b2 + t];
      d->w3f[t] = __bfloat162float(__float2bfloat16_rn(params[off_w3 + t]));
    }
    if (t == 0) d->b3 = params[off_b3];
  }

  __global__ void __launch_bounds__(256) mlp_score_kernel(
    const SeedRecord* records, unsigned long long n, const MlpModelDevice* model, float* logits)
  {
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, c = lane & 3u;
    const unsigned long long n_tiles = (n + 15) / 16;
    const MlpModelDevice& m = *model;
    for (unsigned long long t = blockIdx.x * 8ull + (threadIdx.x >> 5); t < n_tiles; t += gridDim.x * 8ull) {
      const unsigned long long r0 = 16 * t + g, r1 = r0 + 8;
      const bool v0 = r0 < n, v1 = r1 < n;
      const SeedRecord* rec0 = records + (v0 ? r0 : 0);
      const SeedRecord* rec1 = records + (v1 ? r1 : 0);
      uint32_t x[4];
      x[0] = pack_bf16(train_input(m, rec0, v0, 2 * c), train_input(m, rec0, v0, 2 * c + 1));
      x[1] = pack_bf16(train_input(m, rec1, v1, 2 * c), train_input(m, rec1, v1, 2 * c + 1));
      x[2] = pack_bf16(train_input(m, rec0, v0, 2 * c + 8), train_input(m, rec0, v0, 2 * c + 9));
      x[3] = pack_bf16(train_input(m, rec1, v1, 2 * c + 8), train_input(m, rec1, v1, 2 * c + 9));
      float lg, lg8;
      mlp_forward_tile(model, x, lg, lg8);
      if (c == 0) {
        if (v0) logits[r0] = lg;
        if (v1) logits[r1] = lg8;
      }
    }
  }

} // namespace velo

// ---------------------------------------------------------------------------------------
// C ABI: the trainer
// ---------------------------------------------------------------------------------------
struct VeloSeedTrainer {
  VeloSeedModel meta {};
  float lr = 1e-3f, pos_weight = 1.0f, beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  unsigned long long steps = 0;
  float* params = nullptr; // master weights, Adam moments, gradients, loss: one allocation
  float* m = nullptr;
  float* v = nullptr;
  float* grads = nullptr;
  float* loss = nullptr;
  velo::MlpModelDevice* model = nullptr;
  int sm_count = 148;
};

namespace {
  VeloStatus fail(VeloStatus s, const std::string& what)
  {
    velo_host::set_last_error(what);
    return s;
  }
#define VELO_TRY(call)                                                                                  \
  do {                                                                                                  \
    const cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return fail(VELO_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

  VeloStatus accumulate(
    VeloSeedTrainer* t, const VeloSeedRecord* records, unsigned long long first, unsigned batch, cudaStream_t s)
  {
    velo::TrainParams p;
    p.records = reinterpret_cast<const velo::SeedRecord*>(records);
    p.first = first;
    p.batch = batch;
    p.inv_batch = 1.0f / float(batch);
    p.pos_weight = t->pos_weight;
    p.model = t->model;
    p.grads = t->grads;
    p.loss = t->loss;
    const unsigned tiles = (batch + velo::train_rows - 1) / velo::train_rows;
    // two CTAs per SM (256 registers a thread, 71 KB of tiles each) overlap each other's MMA waits
    const unsigned grid = std::min<unsigned>(tiles, 2u * unsigned(t->sm_count));
    VELO_TRY(cudaMemsetAsync(t->loss, 0, sizeof(float), s));
    velo::mlp_train_kernel<<<grid, velo::train_rows, sizeof(velo::TrainShared), s>>>(p);
    VELO_TRY(cudaGetLastError());
    return VELO_OK;
  }
} // namespace

static_assert(sizeof(VeloSeedRecord) == sizeof(velo::SeedRecord), "record layout");

VeloStatus velo_seed_trainer_create(const VeloSeedModel* init, float learning_rate, float pos_weight, VeloSeedTrainer** out)
{
  if (!init || !out || !(learning_rate > 0.0f) || !(pos_weight > 0.0f)) return fail(VELO_ERR_ARGUMENT, "bad argument");
  VeloSeedTrainer* t = new VeloSeedTrainer;
  t->meta = *init;
  t->lr = learning_rate;
  t->pos_weight = pos_weight;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&t->sm_count, cudaDevAttrMultiProcessorCount, dev);
  const cudaError_t attr = cudaFuncSetAttribute(
    velo::mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(velo::TrainShared)));
  if (attr != cudaSuccess) {
    delete t;
    return fail(VELO_ERR_CUDA, std::string("training kernel shared memory: ") + cudaGetErrorString(attr));
  }
  float* block = nullptr;
  cudaError_t e = cudaMalloc(&block, sizeof(float) * (4 * velo::n_params + 1));
  if (e != cudaSuccess) {
    delete t;
    return fail(VELO_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  t->params = block;
  t->m = block + velo::n_params;
  t->v = block + 2 * velo::n_params;
  t->grads = block + 3 * velo::n_params;
  t->loss = block + 4 * velo::n_params;
  e = cudaMalloc(&t->model, sizeof(velo::MlpModelDevice));
  std::vector<float> host(velo::n_params);
  velo::model_params(*init, host.data());
  velo::MlpModelDevice d;
  velo::make_model_device(host.data(), *init, d);
  if (e == cudaSuccess) e = cudaMemcpy(t->params, host.data(), sizeof(float) * velo::n_params, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(t->m, 0, sizeof(float) * (3 * velo::n_params + 1));
  if (e == cudaSuccess) e = cudaMemcpy(t->model, &d, sizeof(d), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    velo_seed_trainer_destroy(t);
    return fail(VELO_ERR_CUDA, std::string("trainer set-up: ") + cudaGetErrorString(e));
  }
  *out = t;
  return VELO_OK;
}

VeloStatus velo_seed_trainer_step(
  VeloSeedTrainer* t, const VeloSeedRecord* records, unsigned long long first, unsigned batch, VeloStream stream, float* loss)
{
  if (!t || !records || batch == 0) return fail(VELO_ERR_ARGUMENT, "bad argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const VeloStatus st = accumulate(t, records, first, batch, s);
  if (st != VELO_OK) return st;
  ++t->steps;
  velo::AdamParams a {t->params, t->m, t->v, t->grads, t->lr, t->beta1, t->beta2, t->eps,
                      float(1.0 - std::pow(double(t->beta1), double(t->steps))),
                      float(1.0 - std::pow(double(t->beta2), double(t->steps)))};
  velo::adam_kernel<<<(velo::n_params + 255) / 256, 256, 0, s>>>(a);
  velo::publish_kernel<<<1, 512, 0, s>>>(t->params, t->model);
  VELO_TRY(cudaGetLastError());
  if (loss) {
    VELO_TRY(cudaMemcpyAsync(loss, t->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    VELO_TRY(cudaStreamSynchronize(s));
  }
  return VELO_OK;
}

VeloStatus velo_seed_trainer_gradients(
  VeloSeedTrainer* t,
  const VeloSeedRecord* records,
  unsigned long long first,
  unsigned batch,
  VeloStream stream,
  float* grads,
  float* loss)
{
  if (!t || !records || batch == 0 || !grads) return fail(VELO_ERR_ARGUMENT, "bad argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  VELO_TRY(cudaMemsetAsync(t->grads, 0, sizeof(float) * velo::n_params, s));
  const VeloStatus st = accumulate(t, records, first, batch, s);
  if (st != VELO_OK) return st;
  VELO_TRY(cudaMemcpyAsync(grads, t->grads, sizeof(float) * velo::n_params, cudaMemcpyDeviceToHost, s));
  if (loss) VELO_TRY(cudaMemcpyAsync(loss, t->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  VELO_TRY(cudaMemsetAsync(t->grads, 0, sizeof(float) * velo::n_params, s));
  VELO_TRY(cudaStreamSynchronize(s));
  return VELO_OK;
}

VeloStatus velo_seed_trainer_score(
  VeloSeedTrainer* t, const VeloSeedRecord* records, unsigned long long n, float* logits, VeloStream stream)
{
  if (!t || !records || !logits) return fail(VELO_ERR_ARGUMENT, "bad argument");
  if (n == 0) return VELO_OK;
  const unsigned long long tiles = (n + 15) / 16;
  const unsigned grid = unsigned(std::min<unsigned long long>((tiles + 7) / 8, unsigned(t->sm_count) * 8ull));
  velo::mlp_score_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
    reinterpret_cast<const velo::SeedRecord*>(records), n, t->model, logits);
  VELO_TRY(cudaGetLastError());
  return VELO_OK;
}

VeloStatus velo_seed_trainer_model(VeloSeedTrainer* t, VeloSeedModel* out)
{
  if (!t || !out) return fail(VELO_ERR_ARGUMENT, "bad argument");
  std::vector<float> host(velo::n_params);
  VELO_TRY(cudaDeviceSynchronize());
  VELO_TRY(cudaMemcpy(host.data(), t->params, sizeof(float) * velo::n_params, cudaMemcpyDeviceToHost));
  *out = t->meta;
  std::memcpy(out->w1, host.data() + velo::off_w1, sizeof(out->w1));
  std::memcpy(out->b1, host.data() + velo::off_b1, sizeof(out->b1));
  std::memcpy(out->w2, host.data() + velo::off_w2, sizeof(out->w2));
  std::memcpy(out->b2, host.data() + velo::off_b2, sizeof(out->b2));
  std::memcpy(out->w3, host.data() + velo::off_w3, sizeof(out->w3));
  out->b3 = host[velo::off_b3];
  return VELO_OK;
}

void velo_seed_trainer_destroy(VeloSeedTrainer* t)
{
  if (!t) return;
  if (t->params) cudaFree(t->params);
  if (t->model) cudaFree(t->model);
  delete t;
}
