// velo_kalman_filter on sm_100a: the simplified Kalman fit of every consolidated VELO
// track, to the beamline (upstream) and to the end of the VELO (downstream).
//
// Reference: device/velo/simplified_kalman_filter/src/VeloKalmanFilter.cu:333-399 (linear_fit
// and the kernel) and include/VeloKalmanFilter.cuh:24-158 (velo_kalman_filter_step,
// simplified_fit).  Same arithmetic in the same order (the chain is built without FMA
// contraction, with IEEE division), so the states are bit-identical to the reference CPU build.
//
// Mapping: one thread per track over all tracks of the slice (the reference runs one CTA per
// event and loops over its tracks), grid-stride, six 256-thread CTAs per SM.  A track's hits
// are consecutive in the consolidated container, so the hits of a warp's 32 tracks form one
// contiguous span, which the warp stages in shared memory with coalesced loads (warp-level
// synchronisation only); both fits read the hits from there.  (Staging a whole CTA's hits behind
// block barriers measured slower: 0.48 ms against 0.29 ms per 16000-event slice, and staging in x,
// y and z rows slower than the container's interleaved order: 0.217 against 0.200 ms.)  States are
// written with 8-byte stores that cover every sector: the fields the reference leaves unwritten
// (qop, chi2, ndof of Velo::Consolidated::States) are written as 0.
#include "velo_kernels.cuh"

namespace velo {

  constexpr float kalman_param_w = 6400.f;                 // VeloDefinitions.cuh:35
  constexpr float kalman_param_w_inverted = 0.00015625f;   // VeloDefinitions.cuh:36
  constexpr float kalman_z_end_velo = 770.f;               // VeloDefinitions.cuh:20

  struct KalmanState {
    float x, y, z, tx, ty, c00, c20, c22, c11, c31, c33;
  };

  // velo_kalman_filter_step (VeloKalmanFilter.cuh:24-58) applied to x and to y.  The covariance
  // update reads only the z step, the hit weight and the covariance itself, never the hit or the
  // state position; the x and y covariances start equal (c00 = c11, c20 = c31 = 0, c22 = c33 = 1) and
  // receive the same noise, so they stay bitwise equal and one gain serves both projections.  The
  // arithmetic of each quantity is the reference's, in its order.
  __device__ __forceinline__ void kalman_step_xy(
    float z, float zhit, float xhit, float yhit, float whit, float& x, float& tx, float& y, float& ty, float& cxx,
    float& cxtx, float& ctxtx)
  {
    const float dz = zhit - z;
    const float predx = x + dz * tx;
    const float predy = y + dz * ty;
    const float dz_t_covTxTx = dz * ctxtx;
    const float predcovXTx = cxtx + dz_t_covTxTx;
    const float dx_t_covXTx = dz * cxtx;
    const float predcovXX = cxx + 2.f * dx_t_covXTx + dz * dz_t_covTxTx;
    const float predcovTxTx = ctxtx;
    const float R = 1.0f / ((1.0f / whit) + predcovXX);
    const float Kx = predcovXX * R;
    const float KTx = predcovXTx * R;
    const float rx = xhit - predx;
    const float ry = yhit - predy;
    x = predx + Kx * rx;
    tx = tx + KTx * rx;
    y = predy + Kx * ry;
    ty = ty + KTx * ry;
    cxx = (1.f - Kx) * predcovXX;
    cxtx = (1.f - Kx) * predcovXTx;
    ctxtx = predcovTxTx - KTx * predcovXTx;
  }

  // simplified_fit<upstream> (VeloKalmanFilter.cuh:63-158); hits: x y z per hit.
  template<bool UPSTREAM>
  __device__ __forceinline__ KalmanState
  simplified_fit(const float* hits, int n, float state_tx, float state_ty, float bx, float by, bool backward)
  {
    const int direction = (backward ? 1 : -1) * (UPSTREAM ? 1 : -1);
    const float noise2PerLayer = 1e-8f + 7e-6f * (state_tx * state_tx + state_ty * state_ty);
    int firsthit = 0, lasthit = n - 1, dhit = 1;
    if ((hits[3 * lasthit + 2] - hits[3 * firsthit + 2]) * static_cast<float>(direction) < 0) {
      firsthit = n - 1;
      lasthit = 0;
      dhit = -1;
    }
    KalmanState s;
    s.x = hits[3 * firsthit];
    s.y = hits[3 * firsthit + 1];
    s.z = hits[3 * firsthit + 2];
    s.tx = state_tx;
    s.ty = state_ty;
    // c00 c20 c22 stand for c11 c31 c33 as well (equal throughout: kalman_step_xy)
    s.c00 = kalman_param_w_inverted;
    s.c20 = 0.f;
    s.c22 = 1.f;
    for (int i = firsthit + dhit; i != lasthit + dhit; i += dhit) {
      const float hx = hits[3 * i], hy = hits[3 * i + 1], hz = hits[3 * i + 2];
      s.c22 += noise2PerLayer;
      kalman_step_xy(s.z, hz, hx, hy, kalman_param_w, s.x, s.tx, s.y, s.ty, s.c00, s.c20, s.c22);
      s.z = hz;
    }
    s.c22 += noise2PerLayer;
    const float delta_z = UPSTREAM ? (s.tx * (bx - s.x) + s.ty * (by - s.y)) / (s.tx * s.tx + s.ty * s.ty) :
                                     kalman_z_end_velo - s.z;
    s.x = s.x + s.tx * delta_z;
    s.y = s.y + s.ty * delta_z;
    s.z = s.z + delta_z;
    const float dz2 = delta_z * delta_z;
    s.c00 += dz2 * s.c22 + 2.f * delta_z * s.c20;
    s.c20 += s.c22 * delta_z;
    s.c11 = s.c00;
    s.c31 = s.c20;
    s.c33 = s.c22;
    return s;
  }

  // Velo::Consolidated::States (VeloConsolidated.cuh:388-598): x y z tx ty qop per track,
  // then c00 c20 c22 c11 c31 c33 chi2 ndof per track after all tracks' first block.
  __device__ __forceinline__ void store_state(float* base, unsigned total, unsigned i, const KalmanState& s)
  {
    float2* st = reinterpret_cast<float2*>(base + 6u * i);
    st[0] = make_float2(s.x, s.y);
    st[1] = make_float2(s.z, s.tx);
    st[2] = make_float2(s.ty, 0.f);
    float2* cov = reinterpret_cast<float2*>(base + 6u * total + 8u * i);
    cov[0] = make_float2(s.c00, s.c20);
    cov[1] = make_float2(s.c22, s.c11);
    cov[2] = make_float2(s.c31, s.c33);
    cov[3] = make_float2(0.f, 0.f);
  }

  __global__ void __launch_bounds__(kalman_threads, kalman_ctas_per_sm) kalman_filter_kernel(KalmanParams p)
  {
    // in the chain: a stage before this one found the slice too large and wrote no tracks
    if (p.abort_flags != 0 && p.status != nullptr && (*p.status & p.abort_flags)) return;
    const unsigned total_tracks = p.offsets_all_velo_tracks[p.n_events];
    if (total_tracks > p.track_capacity) {
      if (threadIdx.x == 0 && blockIdx.x == 0 && p.status != nullptr) set_error(p.status, err_output_capacity);
      return;
    }
    const unsigned* hn = p.offsets_velo_track_hit_number;
    const unsigned total_hits = hn[total_tracks];
    const float* coords = reinterpret_cast<const float*>(p.velo_track_hits) + total_hits;
    // The hits of a warp's 32 consecutive tracks are one contiguous span of the container: the warp
    // copies it into its shared-memory slot with coalesced loads, and each lane fits its track from
    // there.  A span above the slot's capacity is read from global memory in place.
    __shared__ float staged[kalman_threads / 32][3 * kalman_warp_hits];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    float* slot = staged[warp];
    for (unsigned base = blockIdx.x * blockDim.x + warp * 32u; base < total_tracks; base += gridDim.x * blockDim.x) {
      const unsigned end = min(base + 32u, total_tracks);
      const unsigned span_first = hn[base];
      const unsigned span_hits = hn[end] - span_first;
      const bool in_slot = span_hits <= min(p.warp_hits, kalman_warp_hits);
      if (in_slot) {
        const float* src = coords + 3 * size_t(span_first);
        for (unsigned j = lane; j < 3u * span_hits; j += 32u) slot[j] = src[j];
      }
      __syncwarp();
      const unsigned t = base + lane;
      if (t < end) {
        const unsigned first = hn[t], n = hn[t + 1] - first;
        if (n < 2) {
          // a track needs two hits for the linear fit (consolidated tracks have three or more)
          if (p.status != nullptr) set_error(p.status, err_input_capacity);
          p.is_backward[t] = 0;
        }
        else {
          const float* hits = in_slot ? slot + 3u * (first - span_first) : coords + 3 * size_t(first);
          // linear_fit (VeloKalmanFilter.cu:333-353) between the first and last hit
          const float* a = hits;
          const float* b = hits + 3 * (n - 1);
          const float tx = (b[0] - a[0]) / (b[2] - a[2]);
          const float ty = (b[1] - a[1]) / (b[2] - a[2]);
          const float delta_z = (tx * (p.beamline_x - b[0]) + ty * (p.beamline_y - b[1])) / (tx * tx + ty * ty);
          const float lin_z = b[2] + delta_z;
          const bool backward = lin_z > a[2];
          p.is_backward[t] = backward ? 1 : 0;
          const KalmanState up = simplified_fit<true>(hits, int(n), tx, ty, p.beamline_x, p.beamline_y, backward);
          const KalmanState down =
            simplified_fit<false>(hits, int(n), up.tx, up.ty, p.beamline_x, p.beamline_y, backward);
          store_state(p.beamline_states, total_tracks, t, up);
          store_state(p.endvelo_states, total_tracks, t, down);
        }
      }
      __syncwarp(); // every lane done with the slot before the next span overwrites it
    }
  }

} // namespace velo
