// Host side of the C ABI (include/velo_b200.h): geometry and lookup tables, the device
// workspace, the launch sequence of the chain, CUDA-graph capture and the host-buffer path.
//
// Launch sequence for one slice of N events, on the caller's stream, no host sync:
//   memset(bank index, status)
//   estimate_kernel        [N CTAs]  velo_calculate_number_of_candidates + velo_estimate_input_size
//   exclusive_scan_kernel  [2 jobs]  prefix_sum_offsets_velo_candidates, event estimate bases
//   cluster_sort_kernel    [N CTAs]  velo_masked_clustering + velo_sort_by_phi
//                                    (+ prefix_sum_offsets_estimated_input_size, per event)
//   search_by_triplet_kernel [N]     velo_search_by_triplet + velo_three_hit_tracks_filter
//   exclusive_scan_kernel  [3 jobs]  prefix_sum_offsets_velo_tracks,
//                                    prefix_sum_offsets_number_of_three_hit_tracks_filtered,
//                                    per-event track-hit bases
//   consolidate_kernel     [N CTAs]  velo_copy_track_hit_number + prefix_sum_offsets_velo_track_hit_number
//                                    + velo_consolidate_tracks
//   totals_kernel + one 40-byte device-to-host copy of the host scalars.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "velo_b200.h"
#include "velo_kernels.cuh"

namespace {
  thread_local std::string last_error;

  VeloStatus fail(VeloStatus s, const std::string& what)
  {
    last_error = what;
    return s;
  }

} // namespace

namespace velo_host {
  void set_last_error(const std::string& what) { last_error = what; }

  // ClusteringCommon.cpp:6-104 restated: 8-connected groups of the 2 x 4 super pixel,
  // seeded in ascending bit order (bit = col * 4 + row); per group the centroid
  // (row | col << 2, shifted by 4 for the second group), bit 3 set for a second group,
  // and the fractional centroid offsets.
  void build_sp_tables(uint8_t* patterns, float* fx, float* fy)
  {
    std::memset(patterns, 0, 256);
    std::memset(fx, 0, 512 * sizeof(float));
    std::memset(fy, 0, 512 * sizeof(float));
    for (unsigned sp = 0; sp < 256; ++sp) {
      unsigned left = sp, clu = 0;
      for (unsigned seed = 0; seed < 8; ++seed) {
        if (!(left & (1u << seed))) continue;
        unsigned group = 1u << seed, before;
        do {
          before = group;
          for (unsigned b = 0; b < 8; ++b) {
            if (!(left & (1u << b)) || (group & (1u << b))) continue;
            for (unsigned o = 0; o < 8; ++o) {
              if (!(group & (1u << o))) continue;
              const int dc = int(b / 4) - int(o / 4), dr = int(b % 4) - int(o % 4);
              if (dc >= -1 && dc <= 1 && dr >= -1 && dr <= 1) {
                group |= 1u << b;
                break;
              }
            }
          }
        } while (group != before);
        left &= ~group;
        unsigned x = 0, y = 0, n = 0;
        for (unsigned b = 0; b < 8; ++b)
          if (group & (1u << b)) {
            x += b / 4;
            y += b % 4;
            ++n;
          }
        const unsigned cx = x / n, cy = y / n;
        fx[2 * sp + clu] = float(x) / float(n) - float(cx);
        fy[2 * sp + clu] = float(y) / float(n) - float(cy);
        patterns[sp] |= uint8_t(((cx << 2) | cy) << (4 * clu));
        patterns[sp] |= uint8_t(clu << 3);
        ++clu;
      }
    }
  }

  bool parse_geometry(const char* p, size_t size, velo::Geometry& g)
  {
    const char* end = p + size;
    auto read = [&](size_t n, float* dst) {
      uint64_t count;
      if (p + 8 > end) return false;
      std::memcpy(&count, p, 8);
      p += 8;
      if (count != n || p + n * 4 > end) return false;
      std::memcpy(dst, p, n * 4);
      p += n * 4;
      return true;
    };
    if (!read(velo::n_modules, g.module_zs) || !read(velo::n_cols, g.local_x) || !read(velo::n_cols, g.x_pitch))
      return false;
    uint64_t n_ltg, n_trans;
    if (p + 16 > end) return false;
    std::memcpy(&n_ltg, p, 8);
    std::memcpy(&n_trans, p + 8, 8);
    p += 16;
    if (n_ltg != velo::n_sensors || n_trans != 12 || p + velo::n_sensors * 12 * 4 > end) return false;
    std::memcpy(g.ltg, p, velo::n_sensors * 12 * 4);
    return true;
  }
} // namespace velo_host

namespace {
#define VELO_CUDA(call)                                                                                 \
  do {                                                                                                  \
    const cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return fail(VELO_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

  // A device buffer the chain allocated (owned) or a piece of memory it was given (bound).
  template<typename T>
  struct DeviceBuffer {
    using value_type = T;
    T* p = nullptr;
    size_t n = 0;
    bool owned = false;
    cudaError_t reserve(size_t count)
    {
      if (count <= n && p && owned) return cudaSuccess;
      release();
      const cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
      if (e == cudaSuccess) {
        n = count;
        owned = true;
      }
      else {
        p = nullptr;
      }
      return e;
    }
    void bind(void* ptr, size_t count)
    {
      release();
      p = static_cast<T*>(ptr);
      n = count;
    }
    void release()
    {
      if (p && owned) cudaFree(p);
      p = nullptr;
      n = 0;
      owned = false;
    }
  };

  constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

  // Bounds of a slice that a workspace is laid out for: events, estimated clusters T (two per
  // super pixel at most, EstimateInputSize.cu:66,176-203), track container entries, track hits.
  struct SliceBounds {
    size_t n = 0, T = 0, tracks = 0, track_hits = 0, super_pixels = 0;
  };

  struct DeviceTotals {
    unsigned n_events;
    unsigned total_clusters;
    unsigned candidates;
    unsigned four_hit;
    unsigned three_hit;
    unsigned reconstructed;
    unsigned track_hits;
    unsigned track_container_size;
    unsigned flags;
  };

  __global__ void totals_kernel(
    unsigned n,
    const unsigned* event_base,
    const unsigned* candidates_offsets,
    const unsigned* offsets_tracks,
    const unsigned* offsets_three,
    const unsigned* track_hit_base,
    const unsigned* status,
    DeviceTotals* out)
  {
    const unsigned T = event_base[n];
    const float by_clusters = __uint2float_rn(T) * 0.34f;
    out->n_events = n;
    out->total_clusters = T;
    out->candidates = candidates_offsets[n];
    out->four_hit = offsets_tracks[n];
    out->three_hit = offsets_three[n];
    out->reconstructed = offsets_tracks[n] + offsets_three[n];
    out->track_hits = track_hit_base[n];
    out->track_container_size = by_clusters < __uint2float_rn(n * velo::minimum_container_size) ?
                                  n * velo::minimum_container_size :
                                  static_cast<unsigned>(by_clusters);
    out->flags = *status;
  }
} // namespace

// search_by_triplet_kernel instantiations (block size, lanes per seed candidate, ring place)
using SearchKernel = void (*)(velo::SearchParams);
struct SearchVariant {
  unsigned threads, lanes, ring_global;
  SearchKernel fn;
};
static const SearchVariant search_variants[] = {
#define VELO_SEARCH_VARIANT(T, L, R) {T, L, R, velo::search_by_triplet_kernel<T, L, R>},
  VELO_SEARCH_CONFIGS(VELO_SEARCH_VARIANT)
#undef VELO_SEARCH_VARIANT
};

// Retina decoding: keys of an event in L2-resident global scratch (shared memory would hold 24 KiB
// for 3072 keys and allow six CTAs per SM instead of eight), the bucket order of up to 8192
// clusters in shared memory (16 KiB).
static constexpr unsigned retina_key_capacity = 0;
static constexpr unsigned retina_order_capacity_max = 8192;
static constexpr size_t n_sensors_total = velo::n_sensors;

// search_by_triplet_gated_kernel instantiations (block size, ring place)
static SearchKernel gated_search_kernel(unsigned threads, unsigned ring_global)
{
#define VELO_GATED_VARIANT(T, R) \
  if (threads == T && ring_global == R) return velo::search_by_triplet_gated_kernel<T, R>;
  VELO_GATED_CONFIGS(VELO_GATED_VARIANT)
#undef VELO_GATED_VARIANT
  return nullptr;
}

static const SearchVariant* find_search_variant(unsigned threads, unsigned lanes, unsigned ring_global = 0)
{
  for (const auto& v : search_variants)
    if (v.threads == threads && v.lanes == lanes && v.ring_global == ring_global) return &v;
  return nullptr;
}

static constexpr unsigned n_timed_kernels = 9;
static const char* const kernel_names[n_timed_kernels] = {
  "estimate_kernel", "exclusive_scan_kernel(candidates, estimates)", "cluster_sort_kernel", "seed_gate_kernel",
  "search_by_triplet_kernel", "exclusive_scan_kernel(tracks, three-hit, track hits)", "consolidate_kernel",
  "kalman_filter_kernel", "totals_kernel"};

struct VeloChain {
  int device = 0;
  velo::Constants k {};
  DeviceBuffer<velo::Geometry> geo;

  // capacities
  unsigned cap_events = 0;
  size_t cap_clusters = 0; // T
  size_t cap_tracks = 0;   // track container entries
  size_t cap_track_hits = 0;

  // launch configuration (autotuned by allen_b200/autotune.py)
  unsigned estimate_blob_bytes = 32 * 1024;
  unsigned cluster_blob_bytes = 16 * 1024;
  unsigned cluster_stage_capacity = 3072;
  unsigned search_hit_capacity = 3072;
  unsigned search_threads = 256;
  unsigned search_lanes = 2;
  unsigned persistent = 0;
  unsigned events_per_claim = 1;
  unsigned search_ring_global = 0; // rings of tracks to follow in global scratch (persistent only)
  unsigned cluster_threads = 256;  // block size of the clustering kernel (128 or 256)
  unsigned retina_order_capacity = retina_order_capacity_max; // retina clusters ranked through key buckets
  unsigned kalman_warp_hits = velo::kalman_warp_hits;         // Kalman: hits of a warp's tracks staged
  unsigned seed_window = 0;                                   // learned mode: h0 candidates per seed candidate
  unsigned resident_kalman = 0;                               // Kalman CTAs resident on the device
  unsigned resident_export = 0;                               // half-layout export CTAs
  unsigned resident_estimate = 0, resident_cluster = 0, resident_search = 0; // CTAs that fit the device

  // workspace
  DeviceBuffer<unsigned long long> bank_index_key;
  DeviceBuffer<unsigned> status;
  DeviceBuffer<unsigned> number_of_candidates, candidates_offsets, estimated, candidate_num, event_estimate,
    event_base, offsets_est, cluster_num, atomics, n_tracks, offsets_tracks, n_three_out, offsets_three,
    event_track_hits, event_track_hit_base, offsets_all, track_hit_number, offsets_hit_number;
  DeviceBuffer<char> sorted, staging, track_hits, hit_scratch;
  DeviceBuffer<uint64_t> ring_scratch; // search_ring_global: one ring of 2048 entries per resident search CTA
  DeviceBuffer<uint32_t> sp_scratch;   // sorted bank copies (the estimate kernel's, which the clustering kernel reads)
  DeviceBuffer<unsigned> sp_base, sp_alloc; // each event's place in sp_scratch, the allocation counter
  DeviceBuffer<velo::TrackHits> tracks;
  DeviceBuffer<velo::TrackletHits> three_hit, three_out;
  DeviceBuffer<uint8_t> hit_used, accepted;
  DeviceBuffer<DeviceTotals> totals_dev;
  DeviceTotals* totals_host = nullptr;
  cudaEvent_t done = nullptr;
  cudaStream_t capture_stream = nullptr; // graphs are captured here (the legacy stream cannot be)

  // learned seed gate and training-record recording
  DeviceBuffer<velo::MlpModelDevice> seed_model;
  bool learned = false;
  float kept_lo = 0.f, kept_hi = 1.f; // per-event bounds of the gate's kept fraction
  DeviceBuffer<uint8_t> seed_gate, h1_outcome;
  DeviceBuffer<unsigned> gate_stats;
  DeviceBuffer<unsigned> seed_stats;
  DeviceBuffer<unsigned> queue_next, event_order; // persistent launches: 3 claim counters, event order
  // velo_kalman_filter after consolidation (optional)
  bool kalman = false;
  float beamline[2] = {0.f, 0.f};
  DeviceBuffer<uint8_t> is_backward;
  // retina-cluster front end (VPRetinaCluster banks) instead of super pixels
  bool retina = false;
  DeviceBuffer<unsigned> retina_sizes, retina_offsets, retina_bank_index;
  DeviceBuffer<long long> retina_keys;
  DeviceBuffer<float> kalman_beamline_states, kalman_endvelo_states;
  velo::SeedRecord* records = nullptr;
  unsigned* record_count = nullptr;
  unsigned record_capacity = 0, record_every = 1;

  // per-slice workspace: an arena the chain allocated (velo_chain_reserve), or caller memory
  // (velo_chain_bind); the key of the last binding decides whether cached graphs still hold
  DeviceBuffer<char> arena;
  struct BindKey {
    const void* workspace = nullptr;
    SliceBounds bounds;
    long long layout = 0;
    VeloChainOutputBuffers outputs {};
  } bind_key;
  bool bound_external = false;
  // half-precision layout: the caller's coordinate containers, written from the FP32 ones
  char* half_sorted_out = nullptr;
  char* half_track_hits_out = nullptr;

  // host-buffer path
  DeviceBuffer<char> in_raw;
  DeviceBuffer<unsigned> in_offsets, in_sizes, in_types;

  // CUDA graphs, one per slice (pointers, event range), with optional per-kernel timing
  // events captured into them.
  struct GraphEntry {
    VeloDeviceSlice key;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[n_timed_kernels + 1] = {};
  };
  std::vector<GraphEntry> graphs;
  cudaEvent_t direct_ev[n_timed_kernels + 1] = {};
  bool timing = false;
  bool direct_timed = false;
  unsigned last_n = 0;

  void release_graph()
  {
    for (auto& g : graphs) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      for (auto& e : g.ev)
        if (e) cudaEventDestroy(e);
    }
    graphs.clear();
    direct_timed = false;
  }
};

namespace {
  bool slice_bounds(unsigned max_events, unsigned long long max_super_pixels, SliceBounds& b)
  {
    b.n = max_events;
    b.super_pixels = size_t(max_super_pixels);
    b.T = 2 * size_t(max_super_pixels) + 64;
    if (max_events == 0 || b.T > 0xFFFFFFFFull / velo::element_size) return false;
    b.tracks = std::max<size_t>(size_t(double(b.T) * 0.34) + 64, b.n * velo::minimum_container_size + 64);
    b.track_hits = b.T;
    return true;
  }

  // Every buffer whose size follows from the slice bounds, in workspace order:
  // f(buffer, element count, kind).  Outputs are the buffers a caller that binds its own memory
  // supplies separately (the reference's DEVICE_OUTPUTs that later algorithms read); the two
  // coordinate containers are outputs too, unless the caller takes them in the half-precision
  // layout, which the chain exports from its FP32 containers (those then stay in the workspace).
  enum BufferKind { scratch_buffer, output_buffer, coordinate_buffer };

  template<typename F>
  void for_each_slice_buffer(VeloChain* c, const SliceBounds& b, F&& f)
  {
    const size_t n = b.n, T = b.T, tracks = b.tracks;
    f(c->number_of_candidates, n, scratch_buffer);
    f(c->candidates_offsets, n + 1, scratch_buffer);
    f(c->estimated, 26 * n, scratch_buffer);
    f(c->candidate_num, n, scratch_buffer);
    f(c->event_estimate, n, scratch_buffer);
    f(c->event_base, n + 1, scratch_buffer);
    f(c->atomics, 3 * n, scratch_buffer);
    f(c->n_tracks, n, scratch_buffer);
    f(c->offsets_tracks, n + 1, scratch_buffer);
    f(c->n_three_out, n, scratch_buffer);
    f(c->offsets_three, n + 1, scratch_buffer);
    f(c->event_track_hits, n, scratch_buffer);
    f(c->event_track_hit_base, n + 1, scratch_buffer);
    f(c->staging, 24 * T, scratch_buffer);
    f(c->hit_scratch, 16 * T, scratch_buffer);
    f(c->sp_scratch, b.super_pixels + 64, scratch_buffer);
    f(c->sp_base, n, scratch_buffer);
    f(c->sp_alloc, 1, scratch_buffer);
    f(c->tracks, tracks, scratch_buffer);
    f(c->three_hit, tracks, scratch_buffer);
    f(c->three_out, tracks, scratch_buffer);
    f(c->hit_used, T, scratch_buffer);
    f(c->seed_stats, 3 * n, scratch_buffer);
    f(c->seed_gate, T, scratch_buffer);
    f(c->h1_outcome, T, scratch_buffer);
    f(c->gate_stats, 2 * n, scratch_buffer);
    f(c->queue_next, 3, scratch_buffer);
    f(c->is_backward, tracks, scratch_buffer);
    f(c->retina_sizes, n * n_sensors_total, scratch_buffer);
    f(c->retina_offsets, n * n_sensors_total + 1, scratch_buffer);
    f(c->retina_bank_index, n_sensors_total, scratch_buffer);
    f(c->retina_keys, T, scratch_buffer);
    f(c->kalman_beamline_states, 14 * tracks, scratch_buffer);
    f(c->kalman_endvelo_states, 14 * tracks, scratch_buffer);
    f(c->event_order, n, scratch_buffer);
    // outputs
    f(c->offsets_est, 26 * n + 1, output_buffer);
    f(c->cluster_num, 26 * n, output_buffer);
    f(c->sorted, velo::element_size * T, coordinate_buffer);
    f(c->offsets_all, n + 1, output_buffer);
    f(c->track_hit_number, tracks, output_buffer);
    f(c->offsets_hit_number, tracks + 1, output_buffer);
    f(c->track_hits, velo::element_size * b.track_hits, coordinate_buffer);
    f(c->accepted, 2 * tracks, output_buffer);
  }

  // Which buffers a workspace holds: all of them (the chain's own arena), or all but the
  // caller's outputs (FP32 layout), or all but the outputs other than the coordinate containers
  // (half layout).
  enum WorkspaceScope { whole_chain, without_outputs, without_outputs_but_coordinates };

  bool in_workspace(BufferKind k, WorkspaceScope w)
  {
    return k == scratch_buffer || w == whole_chain || (k == coordinate_buffer && w == without_outputs_but_coordinates);
  }

  size_t workspace_bytes(VeloChain* c, const SliceBounds& b, WorkspaceScope w)
  {
    size_t bytes = 0;
    for_each_slice_buffer(c, b, [&](auto& buf, size_t count, BufferKind k) {
      if (in_workspace(k, w)) bytes += align256(count * sizeof(typename std::decay_t<decltype(buf)>::value_type));
    });
    return bytes;
  }

  // Carves the buffers out of `base` (256-byte aligned pieces); the chain's capacities follow.
  void bind_workspace(VeloChain* c, char* base, const SliceBounds& b, WorkspaceScope w)
  {
    size_t at = 0;
    for_each_slice_buffer(c, b, [&](auto& buf, size_t count, BufferKind k) {
      if (!in_workspace(k, w)) return;
      buf.bind(base + at, count);
      at += align256(count * sizeof(typename std::decay_t<decltype(buf)>::value_type));
    });
    c->cap_events = unsigned(b.n);
    c->cap_clusters = b.T;
    c->cap_tracks = b.tracks;
    c->cap_track_hits = b.track_hits;
  }

  // The element counts of the output buffers of a slice bound (set_arguments_size).
  void output_sizes(const SliceBounds& b, int layout, VeloChainSizes* s)
  {
    const size_t element = layout == VELO_COORDINATES_FP16 ? velo::element_size_half : velo::element_size;
    s->offsets_estimated_input_size = 26 * b.n + 1;
    s->module_cluster_num = 26 * b.n;
    s->sorted_velo_cluster_container_bytes = element * b.T;
    s->offsets_all_velo_tracks = b.n + 1;
    s->velo_track_hit_number = b.tracks;
    s->offsets_velo_track_hit_number = b.tracks + 1;
    s->velo_track_hits_bytes = element * b.track_hits;
    s->accepted_velo_tracks = 2 * b.tracks;
    s->max_reconstructed_tracks = b.tracks;
  }
} // namespace

namespace {
  VeloStatus launch_kalman(VeloChain* c, unsigned n, cudaStream_t stream)
  {
    velo::KalmanParams p {};
    p.n_events = n;
    p.offsets_all_velo_tracks = c->offsets_all.p;
    p.offsets_velo_track_hit_number = c->offsets_hit_number.p;
    p.velo_track_hits = c->track_hits.p;
    p.beamline_x = c->beamline[0];
    p.beamline_y = c->beamline[1];
    p.track_capacity = static_cast<unsigned>(c->cap_tracks);
    p.warp_hits = c->kalman_warp_hits;
    p.abort_flags = velo::err_input_capacity | velo::err_output_capacity;
    p.is_backward = c->is_backward.p;
    p.beamline_states = c->kalman_beamline_states.p;
    p.endvelo_states = c->kalman_endvelo_states.p;
    p.status = c->status.p;
    // one wave of the device (grid-stride loop over the tracks)
    const unsigned blocks = std::min<unsigned>(unsigned((c->cap_tracks + 255) / 256), c->resident_kalman);
    velo::kalman_filter_kernel<<<std::max(blocks, 1u), velo::kalman_threads, 0, stream>>>(p);
    VELO_CUDA(cudaGetLastError());
    return VELO_OK;
  }

  VeloStatus enqueue_chain(VeloChain* c, const VeloDeviceSlice& s, cudaStream_t stream, cudaEvent_t* ev, bool capturing)
  {
    using namespace velo;
    const unsigned n = s.n_events;
    RawInput in {s.raw, s.offsets, s.sizes, s.types, s.event_start, s.n_events, s.bank_version, s.mep_layout};
    unsigned stage = 0;
    // inside a capture the records must become graph nodes of their own (external events)
    auto mark = [&]() -> cudaError_t {
      if (!ev) return cudaSuccess;
      return capturing ? cudaEventRecordWithFlags(ev[stage++], stream, cudaEventRecordExternal) :
                         cudaEventRecord(ev[stage++], stream);
    };

    VELO_CUDA(cudaMemsetAsync(c->bank_index_key.p, 0, n_sensors * sizeof(unsigned long long), stream));
    VELO_CUDA(cudaMemsetAsync(c->status.p, 0, sizeof(unsigned), stream));
    // persistent launches: claim counters at zero, events ordered by raw size (largest first)
    const bool persistent = c->persistent != 0;
    auto queue = [&](unsigned k) {
      return persistent ? WorkQueue {c->queue_next.p + k, c->event_order.p, c->events_per_claim} : WorkQueue {};
    };
    auto grid = [&](unsigned resident) { return persistent ? std::min(n, std::max(resident, 1u)) : n; };
    if (persistent) {
      VELO_CUDA(cudaMemsetAsync(c->queue_next.p, 0, 3 * sizeof(unsigned), stream));
      event_order_kernel<<<1, scan_threads, 0, stream>>>(in, c->event_order.p);
      VELO_CUDA(cudaGetLastError());
    }
    VELO_CUDA(mark());

    if (c->retina) {
      // retina-cluster front end (velo_reconstruction.py:18-71): count, scan, decode + sort
      RetinaParams rp {};
      rp.in = in;
      rp.geo = c->geo.p;
      rp.k = c->k;
      rp.each_sensor_pair_size = c->retina_sizes.p;
      rp.bank_index = c->retina_bank_index.p;
      rp.event_total = c->event_estimate.p;
      rp.event_base = c->event_base.p;
      rp.offsets_each_sensor_pair_size = c->retina_offsets.p;
      rp.offsets_module_pair_cluster = c->offsets_est.p;
      rp.module_cluster_num = c->cluster_num.p;
      rp.container = c->sorted.p;
      rp.key_scratch = c->retina_keys.p;
      rp.status = c->status.p;
      rp.smem_key_capacity = retina_key_capacity;
      rp.smem_order_capacity = c->retina_order_capacity;
      rp.cluster_capacity = static_cast<unsigned>(c->cap_clusters);
      VELO_CUDA(cudaMemsetAsync(c->retina_bank_index.p, 0, n_sensors * sizeof(unsigned), stream));
      VELO_CUDA(cudaMemsetAsync(c->candidates_offsets.p, 0, (n + 1) * sizeof(unsigned), stream));
      retina_count_kernel<<<n, decode_threads, 0, stream>>>(rp);
      VELO_CUDA(cudaGetLastError());
      VELO_CUDA(mark());
      ScanParams rs {};
      rs.jobs[0] = {c->event_estimate.p, c->event_base.p, n};
      exclusive_scan_kernel<<<1, scan_threads, 0, stream>>>(rs);
      VELO_CUDA(cudaGetLastError());
      VELO_CUDA(mark());
      retina_decode_kernel<<<n, decode_threads,
                             retina_key_capacity * sizeof(long long) + c->retina_order_capacity * sizeof(uint16_t), stream>>>(rp);
      VELO_CUDA(cudaGetLastError());
      VELO_CUDA(mark());
    }
    else {
      EstimateParams ep {};
      ep.in = in;
      ep.estimated_input_size = c->estimated.p;
      ep.number_of_candidates = c->number_of_candidates.p;
      ep.module_candidate_num = c->candidate_num.p;
      ep.event_estimate = c->event_estimate.p;
      ep.bank_index_key = c->bank_index_key.p;
      ep.designated_stride = (n + 255) / 256;
      ep.status = c->status.p;
      ep.smem_blob_bytes = c->estimate_blob_bytes;
      ep.sp_scratch = c->sp_scratch.p;
      ep.sp_capacity = static_cast<unsigned>(c->sp_scratch.n);
      ep.sp_alloc = c->sp_alloc.p;
      ep.sp_base = c->sp_base.p;
      ep.queue = queue(0);
      VELO_CUDA(cudaMemsetAsync(c->sp_alloc.p, 0, sizeof(unsigned), stream));
      estimate_kernel<<<grid(c->resident_estimate), decode_threads, c->estimate_blob_bytes, stream>>>(ep);
      VELO_CUDA(cudaGetLastError());
      VELO_CUDA(mark());

      ScanParams sp1 {};
      sp1.jobs[0] = {c->event_estimate.p, c->event_base.p, n};
      sp1.jobs[1] = {c->number_of_candidates.p, c->candidates_offsets.p, n};
      exclusive_scan_kernel<<<2, scan_threads, 0, stream>>>(sp1);
      VELO_CUDA(cudaGetLastError());
      VELO_CUDA(mark());

      ClusterSortParams cp {};
      cp.in = in;
      cp.geo = c->geo.p;
      cp.k = c->k;
      cp.estimated_input_size = c->estimated.p;
      cp.event_base = c->event_base.p;
      cp.bank_index_key = c->bank_index_key.p;
      cp.offsets_estimated_input_size = c->offsets_est.p;
      cp.module_cluster_num = c->cluster_num.p;
      cp.sorted_container = c->sorted.p;
      cp.staging = c->staging.p;
      cp.candidates_offsets = c->candidates_offsets.p;
      cp.sp_scratch = c->sp_scratch.p;
      cp.sp_capacity = static_cast<unsigned>(c->sp_scratch.n);
      cp.sp_base = c->sp_base.p;
      cp.status = c->status.p;
      cp.smem_blob_bytes = c->cluster_blob_bytes;
      cp.smem_cluster_capacity = c->cluster_stage_capacity;
      cp.cluster_capacity = static_cast<unsigned>(c->cap_clusters);
      const unsigned cluster_smem = cluster_sort_blob_offset(c->cluster_stage_capacity) + c->cluster_blob_bytes;
      cp.queue = queue(1);
      if (c->cluster_threads == 128)
        cluster_sort_kernel<128><<<grid(c->resident_cluster), 128, cluster_smem, stream>>>(cp);
      else
        cluster_sort_kernel<256><<<grid(c->resident_cluster), 256, cluster_smem, stream>>>(cp);
      VELO_CUDA(cudaGetLastError());
      VELO_CUDA(mark());
    }

    SearchParams sp {};
    sp.geo = c->geo.p;
    sp.k = c->k;
    sp.n_events = n;
    sp.offsets_estimated_input_size = c->offsets_est.p;
    sp.module_cluster_num = c->cluster_num.p;
    sp.sorted_container = c->sorted.p;
    sp.track_capacity = static_cast<unsigned>(c->cap_tracks);
    sp.tracks = c->tracks.p;
    sp.three_hit_tracks = c->three_hit.p;
    sp.hit_used = reinterpret_cast<bool*>(c->hit_used.p);
    sp.atomics_velo = c->atomics.p;
    sp.number_of_velo_tracks = c->n_tracks.p;
    sp.three_hit_tracks_output = c->three_out.p;
    sp.number_of_three_hit_tracks_output = c->n_three_out.p;
    sp.event_track_hits = c->event_track_hits.p;
    sp.status = c->status.p;
    sp.smem_hit_capacity = c->search_hit_capacity;
    sp.hit_scratch = c->hit_scratch.p;
    sp.ring_scratch = c->ring_scratch.p;
    sp.cluster_capacity = static_cast<unsigned>(c->cap_clusters);
    sp.seed_stats = c->seed_stats.p;
    sp.seed_gate = c->learned ? c->seed_gate.p : nullptr;
    sp.gate_stats = c->gate_stats.p;
    sp.kept_lo = c->kept_lo;
    sp.kept_hi = c->kept_hi;
    sp.h1_outcome = c->records ? c->h1_outcome.p : nullptr;
    sp.seed_window = c->seed_window;
    sp.queue = queue(2);
    GateParams gp {};
    gp.geo = c->geo.p;
    gp.k = c->k;
    gp.n_events = n;
    gp.offsets_estimated_input_size = c->offsets_est.p;
    gp.module_cluster_num = c->cluster_num.p;
    gp.sorted_container = c->sorted.p;
    gp.cluster_capacity = static_cast<unsigned>(c->cap_clusters);
    gp.model = c->seed_model.p;
    gp.gate = c->seed_gate.p;
    gp.gate_stats = c->gate_stats.p;
    gp.h1_outcome = c->h1_outcome.p;
    gp.records = c->records;
    gp.record_count = c->record_count;
    gp.record_capacity = c->record_capacity;
    gp.record_every = c->record_every;
    gp.status = c->status.p;
    if (c->learned) {
      // the gate of every seed candidate, before the search
      seed_gate_kernel<false><<<n, gate_threads, 0, stream>>>(gp);
      VELO_CUDA(cudaGetLastError());
    }
    VELO_CUDA(mark());
    if (c->records) VELO_CUDA(cudaMemsetAsync(c->h1_outcome.p, 0, c->cap_clusters, stream));
    const unsigned search_smem = c->search_hit_capacity * search_hit_bytes;
    {
      const SearchKernel fn =
        (c->learned || c->records) ? gated_search_kernel(c->search_threads, c->search_ring_global) : nullptr;
      const SearchVariant* v = find_search_variant(c->search_threads, c->search_lanes, c->search_ring_global);
      if (!fn && !v) return fail(VELO_ERR_ARGUMENT, "no compiled search kernel for this launch configuration");
      void* args[] = {&sp};
      VELO_CUDA(cudaLaunchKernel(reinterpret_cast<const void*>(fn ? fn : v->fn), dim3(grid(c->resident_search)),
                                 dim3(c->search_threads), args, search_smem, stream));
    }
    if (c->records) {
      // training records: the features of the candidates the search met, with its outcomes
      seed_gate_kernel<true><<<n, gate_threads, 0, stream>>>(gp);
      VELO_CUDA(cudaGetLastError());
    }
    VELO_CUDA(mark());

    ScanParams sp2 {};
    sp2.jobs[0] = {c->n_tracks.p, c->offsets_tracks.p, n};
    sp2.jobs[1] = {c->n_three_out.p, c->offsets_three.p, n};
    sp2.jobs[2] = {c->event_track_hits.p, c->event_track_hit_base.p, n};
    exclusive_scan_kernel<<<3, scan_threads, 0, stream>>>(sp2);
    VELO_CUDA(cudaGetLastError());
    VELO_CUDA(mark());

    ConsolidateParams kp {};
    kp.n_events = n;
    kp.offsets_estimated_input_size = c->offsets_est.p;
    kp.sorted_container = c->sorted.p;
    kp.tracks = c->tracks.p;
    kp.three_hit_tracks_output = c->three_out.p;
    kp.offsets_velo_tracks = c->offsets_tracks.p;
    kp.offsets_three_hit = c->offsets_three.p;
    kp.event_track_hit_base = c->event_track_hit_base.p;
    kp.offsets_all_velo_tracks = c->offsets_all.p;
    kp.velo_track_hit_number = c->track_hit_number.p;
    kp.offsets_velo_track_hit_number = c->offsets_hit_number.p;
    kp.velo_track_hits = c->track_hits.p;
    kp.accepted_velo_tracks = reinterpret_cast<bool*>(c->accepted.p);
    kp.track_capacity = static_cast<unsigned>(c->cap_tracks);
    kp.track_hit_capacity = static_cast<unsigned>(c->cap_track_hits);
    kp.track_container_capacity = static_cast<unsigned>(c->cap_tracks);
    kp.cluster_capacity = static_cast<unsigned>(c->cap_clusters);
    kp.status = c->status.p;
    consolidate_kernel<<<n, consolidate_threads, 0, stream>>>(kp);
    VELO_CUDA(cudaGetLastError());
    VELO_CUDA(mark());

    if (c->half_sorted_out) {
      // the caller's containers in the half-precision layout of Allen's CUDA build
      HalfExportParams hp {};
      hp.n_events = n;
      hp.offsets_estimated_input_size = c->offsets_est.p;
      hp.sorted_container = c->sorted.p;
      hp.offsets_all_velo_tracks = c->offsets_all.p;
      hp.offsets_velo_track_hit_number = c->offsets_hit_number.p;
      hp.velo_track_hits = c->track_hits.p;
      hp.cluster_capacity = static_cast<unsigned>(c->cap_clusters);
      hp.track_capacity = static_cast<unsigned>(c->cap_tracks);
      hp.track_hit_capacity = static_cast<unsigned>(c->cap_track_hits);
      hp.sorted_half = c->half_sorted_out;
      hp.track_hits_half = c->half_track_hits_out;
      hp.status = c->status.p;
      export_half_kernel<<<c->resident_export, 256, 0, stream>>>(hp);
      VELO_CUDA(cudaGetLastError());
    }
    if (c->kalman) {
      const VeloStatus st = launch_kalman(c, n, stream);
      if (st != VELO_OK) return st;
    }
    VELO_CUDA(mark());

    totals_kernel<<<1, 1, 0, stream>>>(
      n,
      c->event_base.p,
      c->candidates_offsets.p,
      c->offsets_tracks.p,
      c->offsets_three.p,
      c->event_track_hit_base.p,
      c->status.p,
      c->totals_dev.p);
    VELO_CUDA(cudaGetLastError());
    VELO_CUDA(mark());
    VELO_CUDA(cudaMemcpyAsync(c->totals_host, c->totals_dev.p, sizeof(DeviceTotals), cudaMemcpyDeviceToHost, stream));
    return VELO_OK;
  }

  VeloStatus configure_kernels(VeloChain* c)
  {
    using namespace velo;
    const int cluster_smem = int(cluster_sort_blob_offset(c->cluster_stage_capacity) + c->cluster_blob_bytes);
    const int search_smem = int(c->search_hit_capacity * search_hit_bytes);
    VELO_CUDA(raise_dynamic_smem_limit(reinterpret_cast<const void*>(estimate_kernel), int(c->estimate_blob_bytes)));
    VELO_CUDA(raise_dynamic_smem_limit(reinterpret_cast<const void*>(cluster_sort_kernel<128>), cluster_smem));
    VELO_CUDA(raise_dynamic_smem_limit(reinterpret_cast<const void*>(cluster_sort_kernel<256>), cluster_smem));
    for (const auto& v : search_variants)
      VELO_CUDA(raise_dynamic_smem_limit(reinterpret_cast<const void*>(v.fn), search_smem));
#define VELO_GATED_LIMIT(T, R) \
    VELO_CUDA(raise_dynamic_smem_limit(reinterpret_cast<const void*>(search_by_triplet_gated_kernel<T, R>), search_smem));
    VELO_GATED_CONFIGS(VELO_GATED_LIMIT)
#undef VELO_GATED_LIMIT
    // CTAs of each kernel resident on the device at once: the grid of a persistent launch
    int sms = 0, per_sm = 0;
    VELO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    VELO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, estimate_kernel, decode_threads, c->estimate_blob_bytes));
    c->resident_estimate = unsigned(std::max(per_sm, 1) * sms);
    VELO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kalman_filter_kernel, kalman_threads, 0));
    c->resident_kalman = unsigned(std::max(per_sm, 1) * sms);
    VELO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, export_half_kernel, 256, 0));
    c->resident_export = unsigned(std::max(per_sm, 1) * sms);
    if (c->cluster_threads == 128)
      VELO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cluster_sort_kernel<128>, 128, cluster_smem));
    else
      VELO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cluster_sort_kernel<256>, 256, cluster_smem));
    c->resident_cluster = unsigned(std::max(per_sm, 1) * sms);
    const SearchVariant* v = find_search_variant(c->search_threads, c->search_lanes, c->search_ring_global);
    const SearchKernel learned = gated_search_kernel(c->search_threads, c->search_ring_global);
    SearchKernel fn = (c->learned || c->records) && learned ? learned : (v ? v->fn : nullptr);
    if (fn) {
      VELO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, int(c->search_threads), search_smem));
      c->resident_search = unsigned(std::max(per_sm, 1) * sms);
    }
    // the global rings: one per CTA of the persistent search grid (plain or learned kernel,
    // whichever has more resident CTAs, so that switching modes needs no new allocation)
    if (c->search_ring_global) {
      size_t ctas = 0;
      for (SearchKernel k : {v ? v->fn : nullptr, learned}) {
        if (!k) continue;
        VELO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, int(c->search_threads), search_smem));
        ctas = std::max(ctas, size_t(std::max(per_sm, 1)) * sms);
      }
      VELO_CUDA(c->ring_scratch.reserve(ctas * max_tracks_to_follow));
    }
    return VELO_OK;
  }
} // namespace

extern "C" {

const char* velo_last_error_string(void) { return last_error.c_str(); }

void velo_default_properties(VeloChainProperties* props)
{
  props->phi_tolerance = 0.045f;
  props->max_scatter = 0.08f;
  props->max_skipped_modules = 1;
  props->max_chi2 = 20.0f;
}

VeloStatus velo_device_check(void)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(VELO_ERR_NO_DEVICE, "no CUDA device");
  cudaDeviceProp prop {};
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return fail(VELO_ERR_NO_DEVICE, "cannot query the device");
  if (prop.major != 10) return fail(VELO_ERR_NO_DEVICE, std::string("sm_100 required, found ") + prop.name);
  cudaFuncAttributes attr {};
  if (cudaFuncGetAttributes(&attr, reinterpret_cast<const void*>(search_variants[0].fn)) != cudaSuccess)
    return fail(VELO_ERR_NO_DEVICE, "kernels not loadable on this device");
  return VELO_OK;
}

VeloStatus velo_chain_create(
  const void* geometry, size_t geometry_size, const VeloChainProperties* props, VeloChain** out)
{
  if (!geometry || !out) return fail(VELO_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  const VeloStatus dev_ok = velo_device_check();
  if (dev_ok != VELO_OK) return dev_ok;
  velo::Geometry g {};
  if (!velo_host::parse_geometry(static_cast<const char*>(geometry), geometry_size, g))
    return fail(VELO_ERR_ARGUMENT, "malformed velo geometry blob");
  velo_host::build_sp_tables(g.sp_patterns, g.sp_fx, g.sp_fy);

  VeloChainProperties pr;
  velo_default_properties(&pr);
  if (props) pr = *props;

  auto* c = new VeloChain;
  cudaGetDevice(&c->device);
  // IEEE single-precision constants, as the reference's constexpr values (VeloTools.cuh:18-63)
  const float pi_f = 3.141592654f;
  c->k.convert_factor_i16 = 32768.f / pi_f;
  c->k.c1 = .25f * pi_f;
  c->k.c2 = .75f * pi_f;
  c->k.max_scatter = pr.max_scatter;
  c->k.max_chi2 = pr.max_chi2;
  c->k.max_skipped_modules = pr.max_skipped_modules;
  // hit_phi_float_to_16 (VeloTools.cuh:55-60): float -> int16 through int32
  c->k.phi_tolerance_i16 = static_cast<int16_t>(static_cast<int32_t>(pr.phi_tolerance * c->k.convert_factor_i16));

  auto cleanup = [&](VeloStatus s) {
    velo_chain_destroy(c);
    return s;
  };
  if (c->geo.reserve(1) != cudaSuccess) return cleanup(fail(VELO_ERR_CUDA, "geometry allocation failed"));
  if (cudaMemcpy(c->geo.p, &g, sizeof(g), cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(fail(VELO_ERR_CUDA, "geometry upload failed"));
  if (c->bank_index_key.reserve(velo::n_sensors) != cudaSuccess || c->status.reserve(1) != cudaSuccess ||
      c->totals_dev.reserve(1) != cudaSuccess)
    return cleanup(fail(VELO_ERR_CUDA, "allocation failed"));
  if (cudaMallocHost(&c->totals_host, sizeof(DeviceTotals)) != cudaSuccess)
    return cleanup(fail(VELO_ERR_CUDA, "pinned allocation failed"));
  std::memset(c->totals_host, 0, sizeof(DeviceTotals));
  if (cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming) != cudaSuccess)
    return cleanup(fail(VELO_ERR_CUDA, "event creation failed"));
  if (cudaStreamCreateWithFlags(&c->capture_stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(VELO_ERR_CUDA, "stream creation failed"));
  const VeloStatus cfg = configure_kernels(c);
  if (cfg != VELO_OK) return cleanup(cfg);
  *out = c;
  return VELO_OK;
}

VeloStatus velo_chain_reserve(
  VeloChain* c, unsigned max_events, unsigned long long max_super_pixels, unsigned long long max_raw_bytes)
{
  if (!c || max_events == 0) return fail(VELO_ERR_ARGUMENT, "bad reserve arguments");
  SliceBounds b;
  if (!slice_bounds(max_events, max_super_pixels, b)) return fail(VELO_ERR_CAPACITY, "slice too large for 32-bit offsets");
  c->release_graph();
  // one owned arena for every per-slice buffer, outputs included; it only grows
  const size_t bytes = workspace_bytes(c, b, whole_chain);
  if (!c->arena.owned || c->arena.n < bytes) {
    c->arena.release();
    if (c->arena.reserve(bytes) != cudaSuccess) return fail(VELO_ERR_CUDA, "workspace allocation failed");
  }
  bind_workspace(c, c->arena.p, b, whole_chain);
  c->bound_external = false;
  c->half_sorted_out = c->half_track_hits_out = nullptr;
  c->bind_key = VeloChain::BindKey {};
  if (max_raw_bytes && c->in_raw.reserve(max_raw_bytes + 16) != cudaSuccess)
    return fail(VELO_ERR_CUDA, "workspace allocation failed: input staging");
  return VELO_OK;
}

VeloStatus velo_chain_sizes(
  const VeloChain* c, unsigned max_events, unsigned long long max_super_pixels, int layout, VeloChainSizes* sizes)
{
  if (!sizes || max_events == 0) return fail(VELO_ERR_ARGUMENT, "bad size arguments");
  if (layout != VELO_COORDINATES_FP32 && layout != VELO_COORDINATES_FP16) return fail(VELO_ERR_ARGUMENT, "unknown layout");
  SliceBounds b;
  if (!slice_bounds(max_events, max_super_pixels, b)) return fail(VELO_ERR_CAPACITY, "slice too large for 32-bit offsets");
  output_sizes(b, layout, sizes);
  VeloChain buffers; // the sizes depend on the bounds only, not on a chain's state
  sizes->workspace_bytes =
    workspace_bytes(&buffers, b, layout == VELO_COORDINATES_FP16 ? without_outputs_but_coordinates : without_outputs);
  return VELO_OK;
}

VeloStatus velo_chain_bind(
  VeloChain* c,
  void* workspace,
  unsigned long long workspace_size,
  unsigned max_events,
  unsigned long long max_super_pixels,
  int layout,
  const VeloChainOutputBuffers* o)
{
  if (!c || !workspace || !o || max_events == 0) return fail(VELO_ERR_ARGUMENT, "null argument");
  if (layout != VELO_COORDINATES_FP32 && layout != VELO_COORDINATES_FP16) return fail(VELO_ERR_ARGUMENT, "unknown layout");
  if (!o->dev_offsets_estimated_input_size || !o->dev_module_cluster_num || !o->dev_sorted_velo_cluster_container ||
      !o->dev_offsets_all_velo_tracks || !o->dev_velo_track_hit_number || !o->dev_offsets_velo_track_hit_number ||
      !o->dev_velo_track_hits || !o->dev_accepted_velo_tracks)
    return fail(VELO_ERR_ARGUMENT, "every output buffer is required");
  if (reinterpret_cast<uintptr_t>(workspace) & 255) return fail(VELO_ERR_ARGUMENT, "workspace must be 256-byte aligned");
  const uintptr_t any = reinterpret_cast<uintptr_t>(o->dev_offsets_estimated_input_size) |
                        reinterpret_cast<uintptr_t>(o->dev_module_cluster_num) |
                        reinterpret_cast<uintptr_t>(o->dev_sorted_velo_cluster_container) |
                        reinterpret_cast<uintptr_t>(o->dev_offsets_all_velo_tracks) |
                        reinterpret_cast<uintptr_t>(o->dev_velo_track_hit_number) |
                        reinterpret_cast<uintptr_t>(o->dev_offsets_velo_track_hit_number) |
                        reinterpret_cast<uintptr_t>(o->dev_velo_track_hits);
  if (any & 15) return fail(VELO_ERR_ARGUMENT, "output buffers must be 16-byte aligned");
  SliceBounds b;
  if (!slice_bounds(max_events, max_super_pixels, b)) return fail(VELO_ERR_CAPACITY, "slice too large for 32-bit offsets");
  const bool half = layout == VELO_COORDINATES_FP16;
  const WorkspaceScope scope = half ? without_outputs_but_coordinates : without_outputs;
  if (workspace_size < workspace_bytes(c, b, scope)) return fail(VELO_ERR_CAPACITY, "workspace smaller than velo_chain_sizes()");
  VeloChain::BindKey key {};
  key.workspace = workspace;
  key.bounds = b;
  key.layout = layout;
  key.outputs = *o;
  const bool same = c->bound_external && std::memcmp(&key, &c->bind_key, sizeof(key)) == 0;
  if (same) return VELO_OK;
  c->release_graph();
  c->arena.release();
  bind_workspace(c, static_cast<char*>(workspace), b, scope);
  c->offsets_est.bind(o->dev_offsets_estimated_input_size, 26 * b.n + 1);
  c->cluster_num.bind(o->dev_module_cluster_num, 26 * b.n);
  c->offsets_all.bind(o->dev_offsets_all_velo_tracks, b.n + 1);
  c->track_hit_number.bind(o->dev_velo_track_hit_number, b.tracks);
  c->offsets_hit_number.bind(o->dev_offsets_velo_track_hit_number, b.tracks + 1);
  c->accepted.bind(o->dev_accepted_velo_tracks, 2 * b.tracks);
  if (half) {
    c->half_sorted_out = o->dev_sorted_velo_cluster_container;
    c->half_track_hits_out = o->dev_velo_track_hits;
  }
  else {
    c->sorted.bind(o->dev_sorted_velo_cluster_container, velo::element_size * b.T);
    c->track_hits.bind(o->dev_velo_track_hits, velo::element_size * b.track_hits);
    c->half_sorted_out = c->half_track_hits_out = nullptr;
  }
  c->bind_key = key;
  c->bound_external = true;
  return VELO_OK;
}

VeloStatus velo_chain_run(VeloChain* c, const VeloDeviceSlice* s, VeloStream stream_, int use_graph)
{
  if (!c || !s || !s->raw || !s->offsets || !s->sizes || !s->types) return fail(VELO_ERR_ARGUMENT, "null argument");
  if (s->bank_version != 2 && s->bank_version != 3 && s->bank_version != 4)
    return fail(VELO_ERR_ARGUMENT, "VELO SP bank version not supported (" + std::to_string(s->bank_version) + ")");
  if (s->n_events == 0) return fail(VELO_ERR_ARGUMENT, "empty slice");
  if (s->n_events > c->cap_events) return fail(VELO_ERR_CAPACITY, "slice has more events than reserved");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  c->last_n = s->n_events;
  if (!use_graph) {
    if (c->timing && !c->direct_ev[0])
      for (auto& e : c->direct_ev)
        VELO_CUDA(cudaEventCreate(&e));
    const VeloStatus st = enqueue_chain(c, *s, stream, c->timing ? c->direct_ev : nullptr, false);
    if (st != VELO_OK) return st;
    c->direct_timed = c->timing;
    VELO_CUDA(cudaEventRecord(c->done, stream));
    return VELO_OK;
  }
  VeloChain::GraphEntry* entry = nullptr;
  for (auto& g : c->graphs) {
    const VeloDeviceSlice& k = g.key;
    if (k.raw == s->raw && k.offsets == s->offsets && k.sizes == s->sizes && k.types == s->types &&
        k.event_start == s->event_start && k.n_events == s->n_events && k.bank_version == s->bank_version &&
        k.mep_layout == s->mep_layout) {
      entry = &g;
      break;
    }
  }
  if (!entry) {
    if (c->graphs.size() >= 64) c->release_graph();
    c->graphs.emplace_back();
    entry = &c->graphs.back();
    entry->key = *s;
    if (c->timing)
      for (auto& e : entry->ev)
        VELO_CUDA(cudaEventCreate(&e));
    cudaGraph_t graph;
    VELO_CUDA(cudaStreamBeginCapture(c->capture_stream, cudaStreamCaptureModeThreadLocal));
    const VeloStatus st = enqueue_chain(c, *s, c->capture_stream, c->timing ? entry->ev : nullptr, true);
    const cudaError_t end = cudaStreamEndCapture(c->capture_stream, &graph);
    if (st != VELO_OK) {
      c->graphs.pop_back();
      return st;
    }
    if (end != cudaSuccess) {
      c->graphs.pop_back();
      return fail(VELO_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(end));
    }
    const cudaError_t inst = cudaGraphInstantiate(&entry->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (inst != cudaSuccess) {
      c->graphs.pop_back();
      return fail(VELO_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(inst));
    }
  }
  VELO_CUDA(cudaGraphLaunch(entry->exec, stream));
  VELO_CUDA(cudaEventRecord(c->done, stream));
  return VELO_OK;
}

VeloStatus velo_chain_configure(VeloChain* c, const VeloLaunchConfig* cfg)
{
  if (!c || !cfg) return fail(VELO_ERR_ARGUMENT, "null argument");
  if (!find_search_variant(cfg->search_threads, cfg->search_lanes_per_seed, cfg->search_ring_global))
    return fail(VELO_ERR_ARGUMENT, "no compiled search kernel for (" + std::to_string(cfg->search_threads) + ", " +
                                     std::to_string(cfg->search_lanes_per_seed) + ", ring " +
                                     std::to_string(cfg->search_ring_global) + ")");
  if (cfg->search_ring_global && !cfg->persistent)
    return fail(VELO_ERR_ARGUMENT, "search_ring_global needs persistent launches (one ring per resident CTA)");
  if (cfg->cluster_threads != 128 && cfg->cluster_threads != 256)
    return fail(VELO_ERR_ARGUMENT, "cluster_threads must be 128 or 256");
  if (cfg->retina_order_capacity > retina_order_capacity_max)
    return fail(VELO_ERR_ARGUMENT, "retina_order_capacity above 8192");
  if (cfg->kalman_warp_hits > velo::kalman_warp_hits)
    return fail(VELO_ERR_ARGUMENT, "kalman_warp_hits above 368");
  if (cfg->seed_window > 4) return fail(VELO_ERR_ARGUMENT, "seed_window above 4");
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  const unsigned search_static = 32 * 1024; // upper bound of the kernel's static shared memory
  const unsigned cluster_dyn = velo::cluster_sort_blob_offset(cfg->cluster_stage_capacity) + cfg->cluster_blob_bytes;
  if (cfg->search_hit_capacity * velo::search_hit_bytes + search_static > unsigned(optin) ||
      cluster_dyn + 16 * 1024 > unsigned(optin) || cfg->estimate_blob_bytes + 16 * 1024 > unsigned(optin) ||
      cfg->search_hit_capacity > 65536 || cfg->cluster_stage_capacity > 65535 || (cfg->cluster_blob_bytes & 15) ||
      (cfg->estimate_blob_bytes & 15) || cfg->persistent > 1 || cfg->events_per_claim < 1 || cfg->events_per_claim > 64)
    return fail(VELO_ERR_ARGUMENT, "launch configuration exceeds the device's shared memory");
  c->release_graph();
  c->search_threads = cfg->search_threads;
  c->search_lanes = cfg->search_lanes_per_seed;
  c->search_hit_capacity = cfg->search_hit_capacity;
  c->cluster_stage_capacity = cfg->cluster_stage_capacity;
  c->cluster_blob_bytes = cfg->cluster_blob_bytes;
  c->estimate_blob_bytes = cfg->estimate_blob_bytes;
  c->persistent = cfg->persistent;
  c->events_per_claim = cfg->events_per_claim;
  c->search_ring_global = cfg->search_ring_global;
  c->cluster_threads = cfg->cluster_threads;
  c->retina_order_capacity = cfg->retina_order_capacity;
  c->kalman_warp_hits = cfg->kalman_warp_hits;
  c->seed_window = cfg->seed_window;
  return configure_kernels(c);
}

VeloStatus velo_chain_get_config(const VeloChain* c, VeloLaunchConfig* cfg)
{
  if (!c || !cfg) return fail(VELO_ERR_ARGUMENT, "null argument");
  cfg->search_threads = c->search_threads;
  cfg->search_lanes_per_seed = c->search_lanes;
  cfg->search_hit_capacity = c->search_hit_capacity;
  cfg->cluster_stage_capacity = c->cluster_stage_capacity;
  cfg->cluster_blob_bytes = c->cluster_blob_bytes;
  cfg->estimate_blob_bytes = c->estimate_blob_bytes;
  cfg->persistent = c->persistent;
  cfg->events_per_claim = c->events_per_claim;
  cfg->search_ring_global = c->search_ring_global;
  cfg->cluster_threads = c->cluster_threads;
  cfg->retina_order_capacity = c->retina_order_capacity;
  cfg->kalman_warp_hits = c->kalman_warp_hits;
  cfg->seed_window = c->seed_window;
  return VELO_OK;
}

VeloStatus velo_chain_set_timing(VeloChain* c, int enable)
{
  if (!c) return fail(VELO_ERR_ARGUMENT, "null chain");
  if (bool(enable) != c->timing) c->release_graph();
  c->timing = enable != 0;
  return VELO_OK;
}

unsigned velo_chain_kernel_count(void) { return n_timed_kernels; }

const char* velo_chain_kernel_name(unsigned i) { return i < n_timed_kernels ? kernel_names[i] : ""; }

VeloStatus velo_chain_kernel_times(VeloChain* c, float* ms_sum, unsigned* n_runs)
{
  if (!c || !ms_sum) return fail(VELO_ERR_ARGUMENT, "null argument");
  for (unsigned k = 0; k < n_timed_kernels; ++k)
    ms_sum[k] = 0.f;
  unsigned runs = 0;
  auto add = [&](cudaEvent_t* ev) -> VeloStatus {
    for (unsigned k = 0; k < n_timed_kernels; ++k) {
      float ms = 0.f;
      VELO_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      ms_sum[k] += ms;
    }
    ++runs;
    return VELO_OK;
  };
  VELO_CUDA(cudaEventSynchronize(c->done));
  for (auto& g : c->graphs)
    if (g.ev[0]) {
      const VeloStatus st = add(g.ev);
      if (st != VELO_OK) return st;
    }
  if (c->direct_timed) {
    const VeloStatus st = add(c->direct_ev);
    if (st != VELO_OK) return st;
  }
  if (n_runs) *n_runs = runs;
  return VELO_OK;
}

VeloStatus velo_chain_synchronize(VeloChain* c, VeloChainTotals* t)
{
  if (!c) return fail(VELO_ERR_ARGUMENT, "null chain");
  VELO_CUDA(cudaEventSynchronize(c->done));
  const DeviceTotals& d = *c->totals_host;
  if (t) {
    t->n_events = d.n_events;
    t->host_total_number_of_velo_clusters = d.total_clusters;
    t->host_number_of_cluster_candidates = d.candidates;
    t->host_number_of_velo_tracks_at_least_four_hits = d.four_hit;
    t->host_number_of_three_hit_tracks_filtered = d.three_hit;
    t->host_number_of_reconstructed_velo_tracks = d.reconstructed;
    t->host_accumulated_number_of_hits_in_velo_tracks = d.track_hits;
    t->track_container_size = d.track_container_size;
    t->device_flags = d.flags;
  }
  if (d.flags) return fail(VELO_ERR_DEVICE_FLAGS, "device flags raised: " + std::to_string(d.flags));
  return VELO_OK;
}

VeloStatus velo_chain_outputs(const VeloChain* c, VeloChainOutputs* o)
{
  if (!c || !o) return fail(VELO_ERR_ARGUMENT, "null argument");
  o->dev_number_of_candidates = c->number_of_candidates.p;
  o->dev_estimated_input_size = c->estimated.p;
  o->dev_module_candidate_num = c->candidate_num.p;
  o->dev_offsets_estimated_input_size = c->offsets_est.p;
  o->dev_module_cluster_num = c->cluster_num.p;
  o->dev_sorted_velo_cluster_container = c->sorted.p;
  o->dev_tracks = c->tracks.p;
  o->dev_three_hit_tracks = c->three_hit.p;
  o->dev_hit_used = c->hit_used.p;
  o->dev_atomics_velo = c->atomics.p;
  o->dev_number_of_velo_tracks = c->n_tracks.p;
  o->dev_offsets_velo_tracks = c->offsets_tracks.p;
  o->dev_three_hit_tracks_output = c->three_out.p;
  o->dev_number_of_three_hit_tracks_output = c->n_three_out.p;
  o->dev_offsets_number_of_three_hit_tracks_filtered = c->offsets_three.p;
  o->dev_offsets_all_velo_tracks = c->offsets_all.p;
  o->dev_velo_track_hit_number = c->track_hit_number.p;
  o->dev_offsets_velo_track_hit_number = c->offsets_hit_number.p;
  o->dev_velo_track_hits = c->track_hits.p;
  o->dev_accepted_velo_tracks = c->accepted.p;
  o->dev_seed_stats = c->seed_stats.p;
  o->dev_is_backward = c->is_backward.p;
  o->dev_each_sensor_pair_size = c->retina ? c->retina_sizes.p : nullptr;
  o->dev_offsets_each_sensor_pair_size = c->retina ? c->retina_offsets.p : nullptr;
  o->dev_retina_bank_index = c->retina ? c->retina_bank_index.p : nullptr;
  o->dev_seed_gate = c->seed_gate.p;
  o->dev_gate_stats = c->gate_stats.p;
  o->dev_velo_kalman_beamline_states = reinterpret_cast<char*>(c->kalman_beamline_states.p);
  o->dev_velo_kalman_endvelo_states = reinterpret_cast<char*>(c->kalman_endvelo_states.p);
  return VELO_OK;
}

VeloStatus velo_chain_run_host(
  VeloChain* c,
  const VeloHostSlice* s,
  VeloStream stream_,
  unsigned* host_offsets_all,
  size_t offsets_all_capacity,
  unsigned* host_offsets_hit_number,
  size_t offsets_hit_number_capacity,
  char* host_track_hits,
  size_t track_hits_capacity,
  VeloChainTotals* totals,
  unsigned long long* h2d_bytes,
  unsigned long long* d2h_bytes)
{
  if (!c || !s || !s->raw || !s->offsets || !s->sizes || !s->types) return fail(VELO_ERR_ARGUMENT, "null argument");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  const size_t n = s->n_events;
  if (c->in_raw.reserve(s->raw_bytes + 16) != cudaSuccess || c->in_offsets.reserve(n + 1) != cudaSuccess ||
      c->in_sizes.reserve(s->sizes_bytes / 4 + 1) != cudaSuccess || c->in_types.reserve(s->types_bytes / 4 + 1) != cudaSuccess)
    return fail(VELO_ERR_CUDA, "input staging allocation failed");
  VELO_CUDA(cudaMemcpyAsync(c->in_raw.p, s->raw, s->raw_bytes, cudaMemcpyHostToDevice, stream));
  VELO_CUDA(cudaMemcpyAsync(c->in_offsets.p, s->offsets, (n + 1) * sizeof(unsigned), cudaMemcpyHostToDevice, stream));
  VELO_CUDA(cudaMemcpyAsync(c->in_sizes.p, s->sizes, s->sizes_bytes, cudaMemcpyHostToDevice, stream));
  VELO_CUDA(cudaMemcpyAsync(c->in_types.p, s->types, s->types_bytes, cudaMemcpyHostToDevice, stream));
  unsigned long long up = s->raw_bytes + (n + 1) * sizeof(unsigned) + s->sizes_bytes + s->types_bytes;
  VeloDeviceSlice ds {c->in_raw.p, c->in_offsets.p, c->in_sizes.p, c->in_types.p, 0, s->n_events, s->bank_version};
  VeloStatus st = velo_chain_run(c, &ds, stream, 1);
  if (st != VELO_OK) return st;
  VeloChainTotals t {};
  st = velo_chain_synchronize(c, &t);
  if (totals) *totals = t;
  if (st != VELO_OK) return st;
  const size_t n_tracks = t.host_number_of_reconstructed_velo_tracks;
  const size_t b_all = (n + 1) * sizeof(unsigned);
  const size_t b_hn = (n_tracks + 1) * sizeof(unsigned);
  const size_t b_hits = size_t(t.host_accumulated_number_of_hits_in_velo_tracks) * velo::element_size;
  if (b_all > offsets_all_capacity || b_hn > offsets_hit_number_capacity || b_hits > track_hits_capacity)
    return fail(VELO_ERR_CAPACITY, "host output buffers too small");
  VELO_CUDA(cudaMemcpyAsync(host_offsets_all, c->offsets_all.p, b_all, cudaMemcpyDeviceToHost, stream));
  VELO_CUDA(cudaMemcpyAsync(host_offsets_hit_number, c->offsets_hit_number.p, b_hn, cudaMemcpyDeviceToHost, stream));
  VELO_CUDA(cudaMemcpyAsync(host_track_hits, c->track_hits.p, b_hits, cudaMemcpyDeviceToHost, stream));
  VELO_CUDA(cudaStreamSynchronize(stream));
  if (h2d_bytes) *h2d_bytes = up;
  if (d2h_bytes) *d2h_bytes = b_all + b_hn + b_hits + sizeof(DeviceTotals);
  return VELO_OK;
}

VeloStatus velo_copy_to_host(void* host, const void* device, size_t bytes)
{
  VELO_CUDA(cudaMemcpy(host, device, bytes, cudaMemcpyDeviceToHost));
  return VELO_OK;
}

VeloStatus velo_copy_to_host_async(void* host, const void* device, size_t bytes, VeloStream stream)
{
  VELO_CUDA(cudaMemcpyAsync(host, device, bytes, cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
  return VELO_OK;
}

VeloStatus velo_copy_to_device(void* device, const void* host, size_t bytes)
{
  VELO_CUDA(cudaMemcpy(device, host, bytes, cudaMemcpyHostToDevice));
  return VELO_OK;
}

VeloStatus velo_chain_set_front_end(VeloChain* c, int retina_clusters)
{
  if (!c) return fail(VELO_ERR_ARGUMENT, "null chain");
  if (bool(retina_clusters) != c->retina) c->release_graph();
  c->retina = retina_clusters != 0;
  return VELO_OK;
}

VeloStatus velo_chain_set_kalman(VeloChain* c, int enable, float beamline_x, float beamline_y)
{
  if (!c) return fail(VELO_ERR_ARGUMENT, "null chain");
  c->release_graph();
  c->kalman = enable != 0;
  c->beamline[0] = beamline_x;
  c->beamline[1] = beamline_y;
  return VELO_OK;
}

VeloStatus velo_run_kalman_filter(
  unsigned n_events,
  const unsigned* dev_offsets_all_velo_tracks,
  const unsigned* dev_offsets_velo_track_hit_number,
  const char* dev_velo_track_hits,
  unsigned track_capacity,
  float beamline_x,
  float beamline_y,
  uint8_t* dev_is_backward,
  char* dev_velo_kalman_beamline_states,
  char* dev_velo_kalman_endvelo_states,
  unsigned* dev_status,
  VeloStream stream)
{
  if (!dev_offsets_all_velo_tracks || !dev_offsets_velo_track_hit_number || !dev_velo_track_hits || !dev_is_backward ||
      !dev_velo_kalman_beamline_states || !dev_velo_kalman_endvelo_states)
    return fail(VELO_ERR_ARGUMENT, "null argument");
  if ((reinterpret_cast<uintptr_t>(dev_velo_kalman_beamline_states) |
       reinterpret_cast<uintptr_t>(dev_velo_kalman_endvelo_states)) & 7u)
    return fail(VELO_ERR_ARGUMENT, "state buffers must be 8-byte aligned");
  velo::KalmanParams p {};
  p.n_events = n_events;
  p.offsets_all_velo_tracks = dev_offsets_all_velo_tracks;
  p.offsets_velo_track_hit_number = dev_offsets_velo_track_hit_number;
  p.velo_track_hits = dev_velo_track_hits;
  p.beamline_x = beamline_x;
  p.beamline_y = beamline_y;
  p.track_capacity = track_capacity;
  p.warp_hits = velo::kalman_warp_hits;
  p.is_backward = dev_is_backward;
  p.beamline_states = reinterpret_cast<float*>(dev_velo_kalman_beamline_states);
  p.endvelo_states = reinterpret_cast<float*>(dev_velo_kalman_endvelo_states);
  p.status = dev_status;
  // one wave of the current device (grid-stride loop over the tracks)
  int device = 0, sms = 0, per_sm = 0;
  VELO_CUDA(cudaGetDevice(&device));
  VELO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  VELO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, velo::kalman_filter_kernel, velo::kalman_threads, 0));
  const unsigned blocks = std::min<unsigned>((track_capacity + 255) / 256, unsigned(std::max(per_sm, 1) * sms));
  velo::kalman_filter_kernel<<<std::max(blocks, 1u), velo::kalman_threads, 0, static_cast<cudaStream_t>(stream)>>>(p);
  VELO_CUDA(cudaGetLastError());
  return VELO_OK;
}

VeloStatus velo_chain_set_seed_model(VeloChain* c, const VeloSeedModel* model)
{
  if (!c) return fail(VELO_ERR_ARGUMENT, "null chain");
  c->release_graph();
  if (!model) {
    c->learned = false;
    return configure_kernels(c); // the persistent grid follows the kernel the chain launches
  }
  if (!gated_search_kernel(c->search_threads, c->search_ring_global))
    return fail(VELO_ERR_ARGUMENT, "the learned search needs flat seeding (search_lanes_per_seed 0)");
  std::vector<float> params(VELO_SEED_PARAMS);
  velo::model_params(*model, params.data());
  velo::MlpModelDevice d;
  velo::make_model_device(params.data(), *model, d);
  if (c->seed_model.reserve(1) != cudaSuccess) return fail(VELO_ERR_CUDA, "seed model allocation failed");
  VELO_CUDA(cudaMemcpy(c->seed_model.p, &d, sizeof(d), cudaMemcpyHostToDevice));
  c->kept_lo = model->kept_lo;
  c->kept_hi = model->kept_hi;
  c->learned = true;
  return configure_kernels(c);
}

VeloStatus velo_chain_record_seeds(
  VeloChain* c, VeloSeedRecord* records, unsigned capacity, unsigned record_every, unsigned* dev_count)
{
  if (!c) return fail(VELO_ERR_ARGUMENT, "null chain");
  if (records && (!dev_count || record_every == 0)) return fail(VELO_ERR_ARGUMENT, "recording needs a counter and record_every > 0");
  if (records && !gated_search_kernel(c->search_threads, c->search_ring_global))
    return fail(VELO_ERR_ARGUMENT, "recording needs flat seeding (search_lanes_per_seed 0)");
  c->release_graph();
  c->records = reinterpret_cast<velo::SeedRecord*>(records);
  c->record_count = records ? dev_count : nullptr;
  c->record_capacity = records ? capacity : 0;
  c->record_every = records ? record_every : 1;
  return configure_kernels(c);
}

void velo_chain_destroy(VeloChain* c)
{
  if (!c) return;
  c->release_graph();
  for (auto& e : c->direct_ev)
    if (e) cudaEventDestroy(e);
  c->arena.release();
  c->geo.release();
  c->bank_index_key.release();
  c->status.release();
  c->number_of_candidates.release();
  c->candidates_offsets.release();
  c->estimated.release();
  c->candidate_num.release();
  c->event_estimate.release();
  c->event_base.release();
  c->offsets_est.release();
  c->cluster_num.release();
  c->atomics.release();
  c->n_tracks.release();
  c->offsets_tracks.release();
  c->n_three_out.release();
  c->offsets_three.release();
  c->event_track_hits.release();
  c->event_track_hit_base.release();
  c->offsets_all.release();
  c->track_hit_number.release();
  c->offsets_hit_number.release();
  c->sorted.release();
  c->staging.release();
  c->hit_scratch.release();
  c->ring_scratch.release();
  c->sp_scratch.release();
  c->track_hits.release();
  c->tracks.release();
  c->three_hit.release();
  c->three_out.release();
  c->hit_used.release();
  c->accepted.release();
  c->seed_stats.release();
  c->queue_next.release();
  c->is_backward.release();
  c->retina_sizes.release();
  c->retina_offsets.release();
  c->retina_bank_index.release();
  c->retina_keys.release();
  c->kalman_beamline_states.release();
  c->kalman_endvelo_states.release();
  c->event_order.release();
  c->seed_model.release();
  c->totals_dev.release();
  c->in_raw.release();
  c->in_offsets.release();
  c->in_sizes.release();
  c->in_types.release();
  if (c->totals_host) cudaFreeHost(c->totals_host);
  if (c->done) cudaEventDestroy(c->done);
  if (c->capture_stream) cudaStreamDestroy(c->capture_stream);
  delete c;
}

} // extern "C"
