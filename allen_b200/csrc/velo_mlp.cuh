// Learned seed gate of the triplet search: the device copy of the 12-32-32-1 network and the
// warp-level tensor-core building blocks (mma.sync m16n8k16, bf16 operands, fp32
// accumulators; ldmatrix and movmatrix for fragment layouts).  The features are in
// velo_gate.cu.
//
// No counterpart in the reference: the reference's seeding (SearchByTriplet.cu:298-446)
// searches every unused hit of the module pair as the middle hit h1 of a seed.  The network
// scores each seed candidate h1 from its neighbours before the search; candidates below the
// threshold are not searched.  It is trained on the plain search's own outcomes (label 1 =
// the plain seeding made a seed with this h1).
//
// Fragment layouts (PTX ISA, mma.m16n8k16 with .bf16): lane = 4 g + c.
//   A (16 x 16, row-major): a0 = A[g][2c..2c+1], a1 = A[g+8][2c..], a2 = A[g][2c+8..],
//                           a3 = A[g+8][2c+8..]
//   B (16 x 8, "col"):      b0 = B[2c..2c+1][g], b1 = B[2c+8..2c+9][g]
//   C/D (16 x 8, fp32):     d0 = D[g][2c], d1 = D[g][2c+1], d2 = D[g+8][2c], d3 = D[g+8][2c+1]
// The low 16 bits of a packed pair hold the element with the lower column (or k) index.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "velo_b200.h"

namespace velo {

  constexpr unsigned mlp_features = 12; // inputs of the network
  constexpr unsigned mlp_k1 = 16;       // inputs padded to one k-step
  constexpr unsigned mlp_hidden = 32;   // units of each hidden layer
  constexpr unsigned train_rows = 128;  // records per tensor-core tile of the training kernel

  // The network as the kernels read it: bf16 weights in [out][in] order (PyTorch's Linear
  // layout, so a B fragment pair is one aligned 32-bit word), fp32 biases and the feature
  // standardisation.  w2t is W2 transposed (for the backward pass).
  struct MlpModelDevice {
    uint32_t w1[mlp_hidden][mlp_k1 / 2];      // W1[out][in], in 12..15 zero
    uint32_t w2[mlp_hidden][mlp_hidden / 2];  // W2[out][in]
    uint32_t w2t[mlp_hidden][mlp_hidden / 2]; // W2[in][out]
    uint32_t w3[8][mlp_hidden / 2];           // row 0 = W3, rows 1..7 zero
    float b1[mlp_hidden];
    float b2[mlp_hidden];
    float w3f[mlp_hidden];                    // W3 as fp32 values of the bf16 weights
    float b3;
    float mean[mlp_features];
    float inv_std[mlp_features];
    float threshold_logit;                    // search a seed candidate when its logit > threshold
    float kept_lo, kept_hi;                   // per-event bounds of kept / all seed candidates
  };

  // Host: a model (flat parameters w1, b1, w2, b2, w3, b3 and meta's standardisation,
  // threshold and bounds) in its device form, with bf16 weights rounded to nearest even.
  void make_model_device(const float* params, const VeloSeedModel& meta, MlpModelDevice& d);
  void model_params(const VeloSeedModel& m, float* params);

  // One training example, written by the seed gate in recording mode (64 bytes).
  struct SeedRecord {
    float f[mlp_features]; // raw features (before standardisation)
    float label;           // 1 if the plain seeding made a seed with this middle hit
    uint32_t event;        // event index in the slice
    uint32_t h0, h1;       // h0: 0xFFFFFFFF (the candidate is h1 alone); h1: index in the sorted container
  };

  __device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
  {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
  }

  __device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
  __device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xFFFF0000u); }

  __device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
  {
    asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  }

  // Transpose of an 8 x 8 b16 matrix held one row pair per lane (row g, columns 2c, 2c+1).
  __device__ __forceinline__ uint32_t movmatrix_trans(uint32_t v)
  {
    uint32_t r;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;" : "=r"(r) : "r"(v));
    return r;
  }

  __device__ __forceinline__ void ldmatrix_x4(uint32_t (&a)[4], const void* row_address)
  {
    const uint32_t addr = static_cast<uint32_t>(__cvta_generic_to_shared(row_address));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                 : "r"(addr));
  }

  // Standardised, clamped to [-8, 8] and rounded to bf16 pairs: word w holds inputs 2w, 2w+1.
  __device__ __forceinline__ void
  standardise_pairs(const MlpModelDevice& m, const float (&f)[mlp_features], uint32_t (&w)[8])
  {
    float v[mlp_k1];
#pragma unroll
    for (unsigned i = 0; i < mlp_features; ++i)
      v[i] = fminf(fmaxf((f[i] - __ldg(&m.mean[i])) * __ldg(&m.inv_std[i]), -8.0f), 8.0f);
#pragma unroll
    for (unsigned i = mlp_features; i < mlp_k1; ++i)
      v[i] = 0.0f;
#pragma unroll
    for (unsigned i = 0; i < 8; ++i)
      w[i] = pack_bf16(v[2 * i], v[2 * i + 1]);
  }

  __device__ __forceinline__ float relu(float v) { return fmaxf(v, 0.0f); }

  // Layer output (4 n-tiles of a 16-row tile, C layout) to the A fragments of the next
  // layer's two k-steps, after ReLU and rounding to bf16.
  __device__ __forceinline__ void relu_to_a(const float (&h)[4][4], uint32_t (&a)[2][4])
  {
#pragma unroll
    for (unsigned s = 0; s < 2; ++s) {
      a[s][0] = pack_bf16(relu(h[2 * s][0]), relu(h[2 * s][1]));
      a[s][1] = pack_bf16(relu(h[2 * s][2]), relu(h[2 * s][3]));
      a[s][2] = pack_bf16(relu(h[2 * s + 1][0]), relu(h[2 * s + 1][1]));
      a[s][3] = pack_bf16(relu(h[2 * s + 1][2]), relu(h[2 * s + 1][3]));
    }
  }

  // Forward pass of one 16-row tile whose A fragment is x.  h1, h2: pre-activations of the
  // hidden layers (C layout); a2, a3: the bf16 inputs of layers 2 and 3; returns the logits
  // of rows g and g + 8 (valid in lanes with c == 0).  Weights are read through L1.
  __device__ __forceinline__ void mlp_forward_tile(
    const MlpModelDevice* m,
    const uint32_t (&x)[4],
    float (&h1)[4][4],
    uint32_t (&a2)[2][4],
    float (&h2)[4][4],
    uint32_t (&a3)[2][4],
    float& logit_g,
    float& logit_g8)
  {
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, c = lane & 3u;
#pragma unroll
    for (unsigned j = 0; j < 4; ++j) {
      const float bl = __ldg(&m->b1[8 * j + 2 * c]), bh = __ldg(&m->b1[8 * j + 2 * c + 1]);
      h1[j][0] = bl;
      h1[j][1] = bh;
      h1[j][2] = bl;
      h1[j][3] = bh;
      mma_bf16(h1[j], x, __ldg(&m->w1[8 * j + g][c]), __ldg(&m->w1[8 * j + g][4 + c]));
    }
    relu_to_a(h1, a2);
#pragma unroll
    for (unsigned j = 0; j < 4; ++j) {
      const float bl = __ldg(&m->b2[8 * j + 2 * c]), bh = __ldg(&m->b2[8 * j + 2 * c + 1]);
      h2[j][0] = bl;
      h2[j][1] = bh;
      h2[j][2] = bl;
      h2[j][3] = bh;
#pragma unroll
      for (unsigned s = 0; s < 2; ++s)
        mma_bf16(h2[j], a2[s], __ldg(&m->w2[8 * j + g][8 * s + c]), __ldg(&m->w2[8 * j + g][8 * s + 4 + c]));
    }
    relu_to_a(h2, a3);
    const float b3 = __ldg(&m->b3);
    float o[4] = {b3, b3, b3, b3};
#pragma unroll
    for (unsigned s = 0; s < 2; ++s)
      mma_bf16(o, a3[s], __ldg(&m->w3[g][8 * s + c]), __ldg(&m->w3[g][8 * s + 4 + c]));
    logit_g = o[0];
    logit_g8 = o[2];
  }

  __device__ __forceinline__ void mlp_forward_tile(const MlpModelDevice* m, const uint32_t (&x)[4], float& logit_g, float& logit_g8)
  {
    float h1[4][4], h2[4][4];
    uint32_t a2[2][4], a3[2][4];
    mlp_forward_tile(m, x, h1, a2, h2, a3, logit_g, logit_g8);
  }

} // namespace velo
