// Allocation-free decoding entry point: velo_decode_noalloc() (include/velo_b200.h).
//
// Who needs it.  Inside an Allen sequence every device buffer belongs to the stream's
// arena, which the scheduler carves up before each algorithm runs; algorithms are not
// meant to allocate on their own, and a caller that pre-reserved all of its device memory
// (or works under a memory budget that forbids growth mid-run) cannot call cudaMalloc.
// velo_chain_* owns a workspace it allocates in velo_chain_reserve(); this entry point
// instead keeps its scratch in a fixed-size array of static device memory, loaded with the
// library, so a call allocates nothing: the caller passes the raw banks in and the three
// decoding outputs (offsets, cluster counts, sorted container) out.
//
// What it runs: the decoding half of the chain (candidate count + input-size estimate,
// the device scan, masked clustering + sort by phi) with the same kernels as
// velo_chain_run(), so its outputs are identical.
//
// Limits and rules:
//   * at most velo_noalloc_max_events events and velo_noalloc_max_clusters estimated
//     clusters per call (the estimate is bounded by twice the super-pixel count, which
//     the caller knows from the bank sizes); larger slices are rejected with
//     VELO_ERR_CAPACITY before any work is queued;
//   * every GPU that loads the library holds the array (8 MiB) until the process exits;
//   * the first call on a device looks up the array's device address, uploads the
//     geometry and sets the kernels' shared-memory limits (synchronous CUDA calls), so
//     make that first call before any stream capture;
//   * all calls share the array and it keeps the last call's contents; the parts that
//     must start at zero are cleared on the stream at every call.  Calls that overlap on
//     the GPU (different streams, no ordering between them) race on it;
//   * the geometry is device-wide too: a call with another geometry blob uploads it on its
//     own stream, which rewrites it under any overlapping call on another stream (the same
//     race), and inside a stream capture that upload fails (pageable source).
#include <cstring>
#include <mutex>
#include <string>

#include "velo_b200.h"
#include "velo_kernels.cuh"

namespace {
  constexpr unsigned max_events = 1024;
  constexpr unsigned max_clusters = 262144;
  constexpr unsigned max_devices = 64;

  // Scratch layout (bytes, 256-aligned pieces)
  constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
  constexpr size_t off_bank_index = 0;
  constexpr size_t off_status = align256(off_bank_index + velo::n_sensors * sizeof(unsigned long long));
  constexpr size_t off_estimated = align256(off_status + sizeof(unsigned));
  constexpr size_t off_n_candidates = align256(off_estimated + size_t(velo::n_module_pairs) * max_events * 4);
  constexpr size_t off_candidate_num = align256(off_n_candidates + size_t(max_events) * 4);
  constexpr size_t off_event_estimate = align256(off_candidate_num + size_t(max_events) * 4);
  constexpr size_t off_event_base = align256(off_event_estimate + size_t(max_events) * 4);
  constexpr size_t off_candidates_offsets = align256(off_event_base + size_t(max_events + 1) * 4);
  constexpr size_t off_staging = align256(off_candidates_offsets + size_t(max_events + 1) * 4);
  constexpr size_t scratch_bytes = align256(off_staging + size_t(24) * max_clusters);
  static_assert(scratch_bytes <= 8u * 1024 * 1024, "scratch array above its stated 8 MiB");

  constexpr unsigned estimate_blob_bytes = 32 * 1024;
  constexpr unsigned cluster_blob_bytes = 16 * 1024;
  constexpr unsigned cluster_stage_capacity = 3072;

  std::mutex setup_mutex;
  unsigned char* scratch_address[max_devices] = {};
  std::string geometry_loaded[max_devices];
  thread_local std::string noalloc_error;

  VeloStatus fail(VeloStatus s, const std::string& what)
  {
    noalloc_error = what;
    return s;
  }
} // namespace

// File-scope static device memory: the scratch and the geometry of this entry point.
// In host code these names are host-side stand-ins, never device addresses: the device
// address of the scratch comes from cudaGetSymbolAddress() below.
static __device__ __align__(256) unsigned char velo_noalloc_scratch[scratch_bytes];
static __device__ __align__(16) velo::Geometry velo_noalloc_geometry;

namespace {
  // Once per device, with that device current: the scratch address, the kernels'
  // shared-memory limits, and (when it changes) the geometry.
  VeloStatus setup(int device, const void* geometry, size_t geometry_size, cudaStream_t stream, unsigned char** scratch)
  {
    std::lock_guard<std::mutex> lock(setup_mutex);
    if (device < 0 || device >= int(max_devices)) return fail(VELO_ERR_ARGUMENT, "device index out of range");
    if (!scratch_address[device]) {
      void* ptr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&ptr, velo_noalloc_scratch);
      if (e != cudaSuccess) return fail(VELO_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      const int cluster_smem = int(velo::cluster_sort_blob_offset(cluster_stage_capacity) + cluster_blob_bytes);
      if (velo::raise_dynamic_smem_limit(reinterpret_cast<const void*>(velo::estimate_kernel), int(estimate_blob_bytes)) !=
            cudaSuccess ||
          velo::raise_dynamic_smem_limit(reinterpret_cast<const void*>(velo::cluster_sort_kernel<velo::decode_threads>), cluster_smem) !=
            cudaSuccess)
        return fail(VELO_ERR_CUDA, "cannot set the kernels' shared-memory limits");
      scratch_address[device] = static_cast<unsigned char*>(ptr);
    }
    // the blob is compared in place with the one last uploaded to this device
    std::string& loaded = geometry_loaded[device];
    if (loaded.size() != geometry_size || std::memcmp(loaded.data(), geometry, geometry_size) != 0) {
      velo::Geometry g {};
      if (!velo_host::parse_geometry(static_cast<const char*>(geometry), geometry_size, g))
        return fail(VELO_ERR_ARGUMENT, "malformed velo geometry blob");
      velo_host::build_sp_tables(g.sp_patterns, g.sp_fx, g.sp_fy);
      // on the caller's stream, after the earlier calls queued there; the source is pageable,
      // so the copy has read it when the call returns
      const cudaError_t e = cudaMemcpyToSymbolAsync(velo_noalloc_geometry, &g, sizeof(g), 0, cudaMemcpyHostToDevice, stream);
      if (e != cudaSuccess) return fail(VELO_ERR_CUDA, std::string("geometry upload: ") + cudaGetErrorString(e));
      loaded.assign(static_cast<const char*>(geometry), geometry_size);
    }
    *scratch = scratch_address[device];
    return VELO_OK;
  }
} // namespace

extern "C" {

unsigned velo_noalloc_max_events(void) { return max_events; }
unsigned velo_noalloc_max_clusters(void) { return max_clusters; }
unsigned long long velo_noalloc_scratch_bytes(void) { return scratch_bytes; }
const char* velo_noalloc_last_error_string(void) { return noalloc_error.c_str(); }

VeloStatus velo_decode_noalloc(
  const void* geometry,
  size_t geometry_size,
  const VeloDeviceSlice* s,
  unsigned long long super_pixels,
  VeloStream stream_,
  unsigned* dev_offsets_estimated_input_size,
  unsigned* dev_module_cluster_num,
  char* dev_sorted_velo_cluster_container,
  unsigned long long container_bytes,
  unsigned* dev_status)
{
  using namespace velo;
  if (!geometry || !s || !s->raw || !s->offsets || !s->sizes || !s->types || !dev_offsets_estimated_input_size ||
      !dev_module_cluster_num || !dev_sorted_velo_cluster_container)
    return fail(VELO_ERR_ARGUMENT, "null argument");
  if (s->bank_version != 2 && s->bank_version != 3 && s->bank_version != 4)
    return fail(VELO_ERR_ARGUMENT, "VELO SP bank version not supported (" + std::to_string(s->bank_version) + ")");
  if (s->n_events == 0) return fail(VELO_ERR_ARGUMENT, "empty slice");
  const unsigned long long bound = 2 * super_pixels; // estimated clusters <= 2 per super pixel
  if (s->n_events > max_events)
    return fail(VELO_ERR_CAPACITY, "slice of " + std::to_string(s->n_events) + " events above the limit of " +
                                     std::to_string(max_events));
  if (bound > max_clusters)
    return fail(VELO_ERR_CAPACITY, "slice of up to " + std::to_string(bound) + " clusters above the limit of " +
                                     std::to_string(max_clusters));
  if (container_bytes < bound * element_size)
    return fail(VELO_ERR_CAPACITY, "output container smaller than 18 bytes x 2 x super pixels");
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return fail(VELO_ERR_NO_DEVICE, "no CUDA device");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  unsigned char* scratch = nullptr;
  const VeloStatus st = setup(device, geometry, geometry_size, stream, &scratch);
  if (st != VELO_OK) return st;
  Geometry* geo = nullptr;
  if (cudaGetSymbolAddress(reinterpret_cast<void**>(&geo), velo_noalloc_geometry) != cudaSuccess)
    return fail(VELO_ERR_CUDA, "geometry address");

  const unsigned n = s->n_events;
  RawInput in {s->raw, s->offsets, s->sizes, s->types, s->event_start, s->n_events, s->bank_version, s->mep_layout};
  auto* bank_index = reinterpret_cast<unsigned long long*>(scratch + off_bank_index);
  auto* status = reinterpret_cast<unsigned*>(scratch + off_status);
  auto* estimated = reinterpret_cast<unsigned*>(scratch + off_estimated);
  auto* n_candidates = reinterpret_cast<unsigned*>(scratch + off_n_candidates);
  auto* candidate_num = reinterpret_cast<unsigned*>(scratch + off_candidate_num);
  auto* event_estimate = reinterpret_cast<unsigned*>(scratch + off_event_estimate);
  auto* event_base = reinterpret_cast<unsigned*>(scratch + off_event_base);
  auto* candidates_offsets = reinterpret_cast<unsigned*>(scratch + off_candidates_offsets);
  char* staging = reinterpret_cast<char*>(scratch + off_staging);

  // what must start at zero: the max-reduced bank index and the status word
  if (cudaMemsetAsync(bank_index, 0, n_sensors * sizeof(unsigned long long), stream) != cudaSuccess ||
      cudaMemsetAsync(status, 0, sizeof(unsigned), stream) != cudaSuccess)
    return fail(VELO_ERR_CUDA, "memset");

  EstimateParams ep {};
  ep.in = in;
  ep.estimated_input_size = estimated;
  ep.number_of_candidates = n_candidates;
  ep.module_candidate_num = candidate_num;
  ep.event_estimate = event_estimate;
  ep.bank_index_key = bank_index;
  ep.designated_stride = (n + 255) / 256;
  ep.status = status;
  ep.smem_blob_bytes = estimate_blob_bytes;
  estimate_kernel<<<n, decode_threads, estimate_blob_bytes, stream>>>(ep);

  ScanParams sp {};
  sp.jobs[0] = {event_estimate, event_base, n};
  sp.jobs[1] = {n_candidates, candidates_offsets, n};
  exclusive_scan_kernel<<<2, scan_threads, 0, stream>>>(sp);

  ClusterSortParams cp {};
  cp.in = in;
  cp.geo = geo;
  const float pi_f = 3.141592654f;
  cp.k.convert_factor_i16 = 32768.f / pi_f;
  cp.k.c1 = .25f * pi_f;
  cp.k.c2 = .75f * pi_f;
  cp.estimated_input_size = estimated;
  cp.event_base = event_base;
  cp.bank_index_key = bank_index;
  cp.offsets_estimated_input_size = dev_offsets_estimated_input_size;
  cp.module_cluster_num = dev_module_cluster_num;
  cp.sorted_container = dev_sorted_velo_cluster_container;
  cp.staging = staging;
  cp.status = status;
  cp.smem_blob_bytes = cluster_blob_bytes;
  cp.smem_cluster_capacity = cluster_stage_capacity;
  cp.cluster_capacity = static_cast<unsigned>(bound);
  const unsigned cluster_smem = cluster_sort_blob_offset(cluster_stage_capacity) + cluster_blob_bytes;
  cluster_sort_kernel<decode_threads><<<n, decode_threads, cluster_smem, stream>>>(cp);
  const cudaError_t launch = cudaGetLastError();
  if (launch != cudaSuccess) return fail(VELO_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(launch));
  if (dev_status && cudaMemcpyAsync(dev_status, status, sizeof(unsigned), cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
    return fail(VELO_ERR_CUDA, "status copy");
  return VELO_OK;
}

} // extern "C"
