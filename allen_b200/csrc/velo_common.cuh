// Device-side definitions shared by the VELO kernels (sm_100a).
//
// Layout contract (identical to the reference so that the buffers drop into an
// Allen sequence): the cluster container of VeloEventModel.cuh:92-189 with FP32
// coordinates (the reference CPU build's half_t == float), 18 bytes per hit:
//   u32 id[T] | f32 xyz[3T] interleaved | i16 phi[T],   T = total estimated clusters.
// Track hits (Velo::TrackHits, VeloEventModel.cuh:67-86): u16 hits[26], u8 hitsNum,
// one padding byte = 54 bytes.  Three-hit tracklets: u16 hits[3] = 6 bytes.
//
// All floating point in this library is compiled with -fmad=false: every multiply
// and add rounds separately, in the reference's expression order, so positions,
// phi values and fits are bit-identical to the reference CPU build.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace velo {

  constexpr unsigned n_modules = 52;
  constexpr unsigned n_module_pairs = 26;
  constexpr unsigned n_sensors = 208;
  constexpr unsigned n_cols = 768;
  constexpr unsigned max_track_size = 26;
  constexpr unsigned max_tracks_to_follow = 2048;
  constexpr unsigned minimum_container_size = 10;
  constexpr unsigned element_size = 18;
  constexpr unsigned element_size_half = 12; // the same container with half-precision x, y, z (CUDA builds)
  constexpr unsigned bank_type_velo = 8;
  constexpr unsigned bank_type_vp = 63;
  constexpr unsigned bank_type_vp_retina = 73; // LHCb::RawBank::VPRetinaCluster

  // Error flags (bit set in the chain's device status word; read by the host after a run).
  enum ErrorBits : unsigned {
    err_cluster_capacity = 1u << 0,  // more clusters than the estimate reserved for a module pair
    err_track_capacity = 1u << 1,    // an event produced more tracks than its container slice
    err_ttf_overflow = 1u << 2,      // more than 2048 tracks in flight in one event
    err_bad_sensor = 1u << 3,        // a candidate names a sensor outside the geometry
    err_bulk_copy_timeout = 1u << 4, // a bulk copy into shared memory did not complete in time
    err_output_capacity = 1u << 5,   // consolidated output larger than the reserved buffer
    err_input_capacity = 1u << 6,    // slice larger than the reserved workspace
    err_hits_per_event = 1u << 7,    // more than 65535 estimated hits in one event (u16 indices)
    err_bad_super_pixel = 1u << 8,   // a candidate's flood fill found no pixel (bank index names another bank)
    err_mma_timeout = 1u << 9,       // a tensor-core MMA of the seed gate did not complete in time (gate off)
  };

  // Detector description and super-pixel lookup tables, one copy in global memory
  // (read through the read-only cache: sensors and patterns differ across a warp).
  struct Geometry {
    float module_zs[n_modules];
    float local_x[n_cols];
    float x_pitch[n_cols];
    float ltg[n_sensors * 12];
    uint8_t sp_patterns[256];
    float sp_fx[512];
    float sp_fy[512];
  };

  // Pixel-column lookups.  The tables sit in the same order as in the reference's geometry
  // struct (VeloGeometry, ClusteringDefinitions.cuh:154-161: module z, local x, x pitch,
  // ltg), so a column beyond the sensor's 768 - from a malformed bank, or retina words
  // decoded with another bank version - reads on into the next table exactly as the
  // reference does.  Super-pixel and retina columns stay below 1026; the clamps keep even a
  // larger one inside the struct.
  __device__ __forceinline__ float column_local_x(const Geometry* g, uint32_t cx)
  {
    const float* flat = reinterpret_cast<const float*>(g) + offsetof(Geometry, local_x) / sizeof(float);
    return __ldg(flat + min(cx, 2 * n_cols - 1));
  }
  __device__ __forceinline__ float column_x_pitch(const Geometry* g, uint32_t cx)
  {
    const float* flat = reinterpret_cast<const float*>(g) + offsetof(Geometry, x_pitch) / sizeof(float);
    return __ldg(flat + min(cx, n_cols + 12 * n_sensors - 1));
  }

  // Scalars computed once on the host (IEEE single precision, as the reference's
  // constexpr values and properties), passed by value to the kernels.
  struct Constants {
    float convert_factor_i16; // 2^15 / pi
    float c1;                 // pi / 4
    float c2;                 // 3 pi / 4
    float max_scatter;
    float max_chi2;
    int phi_tolerance_i16;
    unsigned max_skipped_modules;
  };

  struct TrackHits {
    uint16_t hits[max_track_size];
    uint8_t hits_num;
    uint8_t pad;
  };
  static_assert(sizeof(TrackHits) == 54, "TrackHits layout");

  struct TrackletHits {
    uint16_t hits[3];
  };
  static_assert(sizeof(TrackletHits) == 6, "TrackletHits layout");

  // ---------------------------------------------------------------------------------
  // phi (VeloTools.cuh:18-63): approximate atan2 scaled to int16.
  // ---------------------------------------------------------------------------------
  __device__ __forceinline__ float fast_atan2f(const Constants& k, float y, float x)
  {
    const float abs_y = fabsf(y);
    const float x_plus_y = x + abs_y;
    const float x_sub_y = x - abs_y;
    const float y_sub_x = abs_y - x;
    const float nom = (x > 0) ? x_sub_y : x_plus_y;
    const float den = (x > 0) ? x_plus_y : y_sub_x;
    const float r = __fdiv_rn(nom, den);
    const float angle = ((x > 0) ? k.c1 : k.c2) - k.c1 * r;
    return copysignf(angle, y);
  }

  // float -> int16 through a 32-bit truncation (the reference's x86 conversion:
  // values in (-2^31, 2^31) truncate identically, NaN gives 0 on both).
  __device__ __forceinline__ int16_t float_to_i16(float v) { return static_cast<int16_t>(__float2int_rz(v)); }

  __device__ __forceinline__ int16_t hit_phi_16(const Constants& k, float x, float y)
  {
    return float_to_i16(fast_atan2f(k, y, x) * k.convert_factor_i16);
  }

  // BinarySearch.cuh:15-30
  __device__ __forceinline__ int binary_search_leftmost(const int16_t* a, unsigned n, int16_t value)
  {
    int l = 0, r = static_cast<int>(n);
    while (l < r) {
      const int m = (l + r) / 2;
      if (value > a[m]) l = m + 1;
      else r = m;
    }
    return l;
  }

  // VeloEventModel.cuh:192-196
  __device__ __forceinline__ unsigned track_offset(const unsigned* offsets_est, unsigned event)
  {
    return static_cast<unsigned>(__uint2float_rn(offsets_est[event * n_module_pairs]) * 0.34f);
  }

  __device__ __forceinline__ uint32_t lhcb_id(uint32_t cid) { return (2u << 28) | (cid & 0x0FFFFFFFu); }

  __device__ __forceinline__ uint32_t channel_id(uint32_t sensor, uint32_t chip, uint32_t col, uint32_t row)
  {
    return (sensor << 18) | (chip << 16) | (col << 8) | row;
  }

  // Cluster container view over a base pointer (global or shared memory alike).
  struct ClusterView {
    char* base;
    unsigned total;
    __device__ __forceinline__ uint32_t& id(unsigned i) const { return reinterpret_cast<uint32_t*>(base)[i]; }
    __device__ __forceinline__ float& x(unsigned i) const { return reinterpret_cast<float*>(base)[total + 3 * i]; }
    __device__ __forceinline__ float& y(unsigned i) const { return reinterpret_cast<float*>(base)[total + 3 * i + 1]; }
    __device__ __forceinline__ float& z(unsigned i) const { return reinterpret_cast<float*>(base)[total + 3 * i + 2]; }
    __device__ __forceinline__ int16_t& phi(unsigned i) const
    {
      return reinterpret_cast<int16_t*>(base)[8u * total + i];
    }
    __device__ __forceinline__ int16_t* phi_begin() const { return reinterpret_cast<int16_t*>(base) + 8u * total; }
  };

  // ---------------------------------------------------------------------------------
  // Raw event access (Allen layout; ClusteringDefinitions.cuh:61-144, MEPTools.h:26-53)
  // ---------------------------------------------------------------------------------
  struct RawInput {
    const char* raw;
    const unsigned* offsets;
    const unsigned* sizes;
    const unsigned* types;
    unsigned event_start;
    unsigned n_events;
    int bank_version;
    int mep_layout; // 1: MEP layout (MEPTools.h:55-205), banks of one source together
  };

  // MEP layout accessors (MEPTools.h:55-205): offsets = [n_banks, n_events, source ids,
  // per event the byte offset of every bank's fragment]; sizes and types: one u32 offset per
  // bank, then the bank's per-event values.  A fragment has no sourceID word.
  __device__ __forceinline__ unsigned mep_n_banks(const RawInput& in) { return in.offsets[0]; }
  __device__ __forceinline__ unsigned mep_source_id(const RawInput& in, unsigned b) { return in.offsets[2 + b]; }
  __device__ __forceinline__ unsigned mep_fragment_offset(const RawInput& in, unsigned ev, unsigned b)
  {
    return in.offsets[2 + in.offsets[0] * (1 + ev) + b];
  }
  __device__ __forceinline__ unsigned mep_bank_size(const RawInput& in, unsigned ev, unsigned b)
  {
    return (reinterpret_cast<const uint16_t*>(in.sizes) + in.sizes[b])[ev];
  }
  __device__ __forceinline__ unsigned mep_bank_type(const RawInput& in, unsigned ev, unsigned b)
  {
    return (reinterpret_cast<const uint8_t*>(in.types) + in.types[b])[ev];
  }

  __device__ __forceinline__ const uint16_t* bank_sizes(const RawInput& in, unsigned event)
  {
    return reinterpret_cast<const uint16_t*>(in.sizes) + in.sizes[event];
  }
  __device__ __forceinline__ const uint8_t* bank_types(const RawInput& in, unsigned event)
  {
    return reinterpret_cast<const uint8_t*>(in.types) + in.types[event];
  }

  // ---------------------------------------------------------------------------------
  // Block-wide helpers
  // ---------------------------------------------------------------------------------
  // Exclusive scan of one value per thread over the block (blockDim.x a multiple of 32,
  // at most 1024).  `warp_sums` needs 33 entries of shared memory.  Returns the exclusive
  // prefix; *total receives the block total.
  __device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* warp_sums, unsigned* total)
  {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    const unsigned n_warps = blockDim.x >> 5;
    unsigned incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= static_cast<unsigned>(o)) incl += t;
    }
    __syncthreads();
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      unsigned s = lane < n_warps ? warp_sums[lane] : 0u;
      unsigned si = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xFFFFFFFFu, si, o);
        if (lane >= static_cast<unsigned>(o)) si += t;
      }
      warp_sums[lane] = si - s;
      if (lane == 31) warp_sums[32] = si;
    }
    __syncthreads();
    const unsigned result = warp_sums[warp] + incl - v;
    *total = warp_sums[32];
    __syncthreads();
    return result;
  }

  __device__ __forceinline__ void set_error(unsigned* status, unsigned bit) { atomicOr(status, bit); }

  // Invalidates, without writing them back to HBM, the 128-byte L2 lines that lie wholly
  // inside [p, p + bytes): a CTA's scratch that no thread reads again (every thread of the
  // CTA calls it, after a barrier that follows the last read; discard.global.L2).
  __device__ __forceinline__ void discard_l2(const void* p, size_t bytes)
  {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uintptr_t lo = (a + 127) & ~uintptr_t(127);
    const uintptr_t hi = (a + bytes) & ~uintptr_t(127);
    for (uintptr_t line = lo + uintptr_t(threadIdx.x) * 128; line < hi; line += uintptr_t(blockDim.x) * 128)
      asm volatile("discard.global.L2 [%0], 128;" ::"l"(line) : "memory");
  }

} // namespace velo
