// Training of the learned seed pruner on sm_100a, and the host conversion of a model to
// its device form.  No counterpart in the reference (see velo_mlp.cuh).
//
// mlp_train_kernel: each warp takes 16-record tiles; the forward pass keeps every layer in
// mma.sync fragments (C layout of one layer = A layout of the next); the backward pass gets
// the transposed operands of the weight gradients (dZ^T as A, the layer input as B) with
// movmatrix, so no tile goes through shared memory.  Per-warp gradient sums are reduced in
// shared memory and added to the global fp32 gradient once per CTA.  adam_kernel updates
// the fp32 master weights and writes the bf16 copies the kernels read.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "velo_b200.h"
#include "velo_mlp.cuh"

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

  __global__ void __launch_bounds__(256) mlp_train_kernel(TrainParams p)
  {
    __shared__ float block_grads[n_params + 1];
    for (unsigned i = threadIdx.x; i <= n_params; i += blockDim.x)
      block_grads[i] = 0.0f;
    __syncthreads();

    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, c = lane & 3u;
    const unsigned warps = blockDim.x >> 5;
    const MlpModelDevice& m = *p.model;
    const unsigned n_tiles = (p.batch + 15) / 16;

    float gw1[2][2][4] = {}, gw2[2][4][4] = {}, gb1[4][2] = {}, gb2[4][2] = {}, gw3[4][2] = {};
    float gb3 = 0.0f, loss = 0.0f;
    for (unsigned t = blockIdx.x * warps + (threadIdx.x >> 5); t < n_tiles; t += gridDim.x * warps) {
      const unsigned r0 = 16 * t + g, r1 = r0 + 8;
      const bool v0 = r0 < p.batch, v1 = r1 < p.batch;
      const SeedRecord* rec0 = p.records + p.first + (v0 ? r0 : 0);
      const SeedRecord* rec1 = p.records + p.first + (v1 ? r1 : 0);
      uint32_t x[4];
      x[0] = pack_bf16(train_input(m, rec0, v0, 2 * c), train_input(m, rec0, v0, 2 * c + 1));
      x[1] = pack_bf16(train_input(m, rec1, v1, 2 * c), train_input(m, rec1, v1, 2 * c + 1));
      x[2] = pack_bf16(train_input(m, rec0, v0, 2 * c + 8), train_input(m, rec0, v0, 2 * c + 9));
      x[3] = pack_bf16(train_input(m, rec1, v1, 2 * c + 8), train_input(m, rec1, v1, 2 * c + 9));

      float h1[4][4], h2[4][4], lg, lg8;
      uint32_t a2[2][4], a3[2][4];
      mlp_forward_tile(p.model, x, h1, a2, h2, a3, lg, lg8);
      const float z0 = __shfl_sync(0xFFFFFFFFu, lg, lane & ~3u);
      const float z1 = __shfl_sync(0xFFFFFFFFu, lg8, lane & ~3u);

      // d loss / d logit, per row (weighted binary cross-entropy, mean over the batch)
      float dz[2] = {0.0f, 0.0f};
      const float zs[2] = {z0, z1};
      const bool vs[2] = {v0, v1};
      const SeedRecord* rs[2] = {rec0, rec1};
#pragma unroll
      for (unsigned q = 0; q < 2; ++q) {
        if (!vs[q]) continue;
        const float y = __ldg(&rs[q]->label);
        const float w = y > 0.5f ? p.pos_weight : 1.0f;
        const float z = zs[q];
        const float prob = 1.0f / (1.0f + expf(-z));
        dz[q] = w * (prob - y) * p.inv_batch;
        if (c == 0) loss += w * (fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z))));
      }
      if (c == 0) gb3 += dz[0] + dz[1];

      // layer 3: dW3 = sum dz * a3, dH2 = dz * W3, dZ2 = dH2 where h2 > 0
      float d2[4][4];
#pragma unroll
      for (unsigned j = 0; j < 4; ++j) {
        const uint32_t top = a3[j >> 1][(j & 1u) ? 2 : 0], bottom = a3[j >> 1][(j & 1u) ? 3 : 1];
        gw3[j][0] += dz[0] * bf16_lo(top) + dz[1] * bf16_lo(bottom);
        gw3[j][1] += dz[0] * bf16_hi(top) + dz[1] * bf16_hi(bottom);
        const float wl = __ldg(&m.w3f[8 * j + 2 * c]), wh = __ldg(&m.w3f[8 * j + 2 * c + 1]);
        d2[j][0] = h2[j][0] > 0.0f ? dz[0] * wl : 0.0f;
        d2[j][1] = h2[j][1] > 0.0f ? dz[0] * wh : 0.0f;
        d2[j][2] = h2[j][2] > 0.0f ? dz[1] * wl : 0.0f;
        d2[j][3] = h2[j][3] > 0.0f ? dz[1] * wh : 0.0f;
        gb2[j][0] += d2[j][0] + d2[j][2];
        gb2[j][1] += d2[j][1] + d2[j][3];
      }
      uint32_t e2[4][2];
#pragma unroll
      for (unsigned j = 0; j < 4; ++j) {
        e2[j][0] = pack_bf16(d2[j][0], d2[j][1]);
        e2[j][1] = pack_bf16(d2[j][2], d2[j][3]);
      }
      // dW2 += dZ2^T a2 (A: dZ2 transposed, B: a2 transposed into k-major pairs)
#pragma unroll
      for (unsigned mt = 0; mt < 2; ++mt) {
        const uint32_t A[4] = {movmatrix_trans(e2[2 * mt][0]), movmatrix_trans(e2[2 * mt + 1][0]),
                               movmatrix_trans(e2[2 * mt][1]), movmatrix_trans(e2[2 * mt + 1][1])};
#pragma unroll
        for (unsigned nt = 0; nt < 4; ++nt) {
          const uint32_t b0 = movmatrix_trans(a2[nt >> 1][(nt & 1u) ? 2 : 0]);
          const uint32_t b1 = movmatrix_trans(a2[nt >> 1][(nt & 1u) ? 3 : 1]);
          mma_bf16(gw2[mt][nt], A, b0, b1);
        }
      }
      // dH1 = dZ2 W2 (A: dZ2 in C-to-A layout, B: W2 transposed), dZ1 = dH1 where h1 > 0
      float d1[4][4] = {};
#pragma unroll
      for (unsigned s = 0; s < 2; ++s) {
        const uint32_t A[4] = {e2[2 * s][0], e2[2 * s][1], e2[2 * s + 1][0], e2[2 * s + 1][1]};
#pragma unroll
        for (unsigned nt = 0; nt < 4; ++nt)
          mma_bf16(d1[nt], A, __ldg(&m.w2t[8 * nt + g][8 * s + c]), __ldg(&m.w2t[8 * nt + g][8 * s + 4 + c]));
      }
      uint32_t e1[4][2];
#pragma unroll
      for (unsigned j = 0; j < 4; ++j) {
#pragma unroll
        for (unsigned q = 0; q < 4; ++q)
          d1[j][q] = h1[j][q] > 0.0f ? d1[j][q] : 0.0f;
        gb1[j][0] += d1[j][0] + d1[j][2];
        gb1[j][1] += d1[j][1] + d1[j][3];
        e1[j][0] = pack_bf16(d1[j][0], d1[j][1]);
        e1[j][1] = pack_bf16(d1[j][2], d1[j][3]);
      }
      // dW1 += dZ1^T x
#pragma unroll
      for (unsigned mt = 0; mt < 2; ++mt) {
        const uint32_t A[4] = {movmatrix_trans(e1[2 * mt][0]), movmatrix_trans(e1[2 * mt + 1][0]),
                               movmatrix_trans(e1[2 * mt][1]), movmatrix_trans(e1[2 * mt + 1][1])};
#pragma unroll
        for (unsigned nf = 0; nf < 2; ++nf)
          mma_bf16(gw1[mt][nf], A, movmatrix_trans(x[nf ? 2 : 0]), movmatrix_trans(x[nf ? 3 : 1]));
      }
    }

    // reduce: per-lane partial sums into the CTA's shared copy
    float* bg = block_grads;
#pragma unroll
    for (unsigned mt = 0; mt < 2; ++mt)
#pragma unroll
      for (unsigned nf = 0; nf < 2; ++nf)
#pragma unroll
        for (unsigned q = 0; q < 4; ++q) {
          const unsigned o = 16 * mt + g + ((q & 2u) ? 8 : 0), f = 8 * nf + 2 * c + (q & 1u);
          if (f < mlp_features) atomicAdd(&bg[off_w1 + o * mlp_features + f], gw1[mt][nf][q]);
        }
#pragma unroll
    for (unsigned mt = 0; mt < 2; ++mt)
#pragma unroll
      for (unsigned nt = 0; nt < 4; ++nt)
#pragma unroll
        for (unsigned q = 0; q < 4; ++q) {
          const unsigned o = 16 * mt + g + ((q & 2u) ? 8 : 0), i = 8 * nt + 2 * c + (q & 1u);
          atomicAdd(&bg[off_w2 + o * mlp_hidden + i], gw2[mt][nt][q]);
        }
#pragma unroll
    for (unsigned j = 0; j < 4; ++j)
#pragma unroll
      for (unsigned q = 0; q < 2; ++q) {
        atomicAdd(&bg[off_b1 + 8 * j + 2 * c + q], gb1[j][q]);
        atomicAdd(&bg[off_b2 + 8 * j + 2 * c + q], gb2[j][q]);
        atomicAdd(&bg[off_w3 + 8 * j + 2 * c + q], gw3[j][q]);
      }
    if (c == 0) {
      atomicAdd(&bg[off_b3], gb3);
      atomicAdd(&bg[n_params], loss);
    }
    __syncthreads();
    for (unsigned i = threadIdx.x; i < n_params; i += blockDim.x)
      atomicAdd(&p.grads[i], block_grads[i]);
    if (threadIdx.x == 0) atomicAdd(p.loss, block_grads[n_params] * p.inv_batch);
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
    const unsigned tiles = (batch + 15) / 16;
    const unsigned grid = std::min<unsigned>((tiles + 7) / 8, unsigned(t->sm_count) * 4u);
    VELO_TRY(cudaMemsetAsync(t->loss, 0, sizeof(float), s));
    velo::mlp_train_kernel<<<grid, 256, 0, s>>>(p);
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
