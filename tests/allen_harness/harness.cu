/*
 * Test infrastructure: runs the Allen adaptor (integration/VeloB200Chain.cu) the way Allen's
 * scheduler does, and the reference's own velo_kalman_filter on its outputs.
 *
 *  1. Constants as Allen's VPGeometry consumer fills them (integration/non_event_data/src/
 *     VPGeometry.cpp:58-67: the reference's VeloGeometry(std::vector<char>) copied to the device).
 *  2. One Allen::Store::AllenArgument per parameter of velo_b200_chain_t, bound into the
 *     ArgumentReferences<Parameters> that the algorithm's methods take (stream/store/include/
 *     Store.cuh:236-440); inputs point at the caller's device slice.
 *  3. set_arguments_size(), then device (cudaMalloc, standing in for the per-stream arena) and host
 *     memory of those sizes for every output, then operator() on a stream of its own.
 *  4. The reference's velo_kalman_filter kernel (device/velo/simplified_kalman_filter/src/
 *     VeloKalmanFilter.cu:362-399, compiled here for sm_100a) reads the adaptor's
 *     dev_velo_tracks_view and dev_offsets_all_velo_tracks, as velo_reconstruction.py:295-307
 *     wires it.
 *  5. A kernel that walks the adaptor's dev_imec_velo_tracks with the reference's own view types
 *     (dyn_cast to MultiEventTracks, container(e).track(i).hit(j)) and writes every hit's id and
 *     coordinates at its consolidated position.
 * Every buffer is then readable through allen_harness_buffer() until allen_harness_free().
 */
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "VeloB200Chain.cuh"
#include "VeloKalmanFilter.cuh"
#include "ClusteringDefinitions.cuh"

namespace {
  using Chain = velo_b200_chain::velo_b200_chain_t;
  using Refs = ArgumentReferences<velo_b200_chain::Parameters>;
  using Tuple = typename Refs::parameters_tuple_t;

  struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    bool device = true;
  };

  struct Harness {
    std::vector<std::unique_ptr<Allen::Store::AllenArgument>> args;
    std::map<std::string, Buffer> buffers; // every output by its parameter name, plus the harness's own
    std::vector<void*> device_allocations, host_allocations;
    std::unique_ptr<Chain> algorithm;
    VeloGeometry* dev_geometry = nullptr;
    float* dev_beamline = nullptr;
    cudaStream_t stream = nullptr;
    std::string error;
    ~Harness()
    {
      algorithm.reset(); // destroys the library chains first
      for (void* p : device_allocations)
        cudaFree(p);
      for (void* p : host_allocations)
        std::free(p);
      if (dev_geometry) cudaFree(dev_geometry);
      if (dev_beamline) cudaFree(dev_beamline);
      if (stream) cudaStreamDestroy(stream);
    }
  };

  std::string last_error;

  template<typename P>
  constexpr bool is_output = Allen::is_template_base_of_v<Allen::Store::output_datatype, P>;
  template<typename P>
  constexpr bool is_host = std::is_base_of_v<Allen::Store::host_datatype, P>;

  // a readable name for each parameter: the last component of its nested name, e.g.
  // dev_velo_track_hits_t from the mangled N16velo_b200_chain10Parameters21dev_velo_track_hits_tE
  template<typename P>
  std::string parameter_name()
  {
    const std::string s = typeid(P).name();
    std::string last;
    size_t i = s.size() > 0 && s[0] == 'N' ? 1 : 0;
    while (i < s.size() && std::isdigit(static_cast<unsigned char>(s[i]))) {
      size_t len = 0;
      while (i < s.size() && std::isdigit(static_cast<unsigned char>(s[i])))
        len = 10 * len + size_t(s[i++] - '0');
      last = s.substr(i, len);
      i += len;
    }
    return last.empty() ? s : last;
  }

  template<size_t... I>
  auto make_arguments(Harness& h, std::index_sequence<I...>)
  {
    (h.args.emplace_back(std::make_unique<Allen::Store::AllenArgument>(
       std::in_place_type<std::remove_const_t<typename std::tuple_element_t<I, Tuple>::type>>,
       parameter_name<std::tuple_element_t<I, Tuple>>(),
       is_host<std::tuple_element_t<I, Tuple>> ? Allen::Store::Scope::Host : Allen::Store::Scope::Device)),
     ...);
    return typename Refs::arguments_t {std::ref(static_cast<Allen::Store::BaseArgument&>(*h.args[I]))...};
  }

  template<typename P>
  Allen::Store::AllenArgument& arg(Harness& h)
  {
    return *h.args[index_of_v<P, Tuple>];
  }

  // memory of the size set_arguments_size gave, for every output
  template<size_t... I>
  void allocate_outputs(Harness& h, const Refs& refs, std::index_sequence<I...>)
  {
    auto one = [&](auto tag) {
      using P = typename decltype(tag)::type;
      if constexpr (is_output<P>) {
        using T = std::remove_const_t<typename P::type>;
        const size_t bytes = std::max<size_t>(refs.template size<P>(), 1) * sizeof(T);
        void* p = nullptr;
        if constexpr (is_host<P>) {
          p = std::calloc(bytes, 1);
          h.host_allocations.push_back(p);
        }
        else {
          if (cudaMalloc(&p, bytes) != cudaSuccess) throw std::runtime_error("harness allocation failed");
          h.device_allocations.push_back(p);
        }
        arg<P>(h).set_pointer(p);
      }
    };
    (one(std::type_identity<std::tuple_element_t<I, Tuple>> {}), ...);
  }

  // after operator(): every output's pointer and (possibly reduced) size, by name
  template<size_t... I>
  void record_outputs(Harness& h, const Refs& refs, std::index_sequence<I...>)
  {
    auto one = [&](auto tag) {
      using P = typename decltype(tag)::type;
      if constexpr (is_output<P>) {
        using T = std::remove_const_t<typename P::type>;
        h.buffers[parameter_name<P>()] =
          Buffer {const_cast<void*>(static_cast<const void*>(refs.template data<P>())), refs.template size<P>() * sizeof(T),
                  !is_host<P>};
      }
    };
    (one(std::type_identity<std::tuple_element_t<I, Tuple>> {}), ...);
  }

  void* device_alloc(Harness& h, size_t bytes)
  {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 1)) != cudaSuccess) throw std::runtime_error("harness allocation failed");
    h.device_allocations.push_back(p);
    return p;
  }

  struct HitRecord {
    unsigned id;
    float x, y, z;
  };

  // Every hit of every track, read through the reference's own view types from the type-erased
  // multi-event container; one thread walks events, tracks and hits in order, which is the
  // consolidated container's order, and writes each hit at its running position.
  __global__ void walk_views(Allen::IMultiEventContainer* const* imec, HitRecord* out, unsigned capacity, unsigned* counts)
  {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const auto* m = Allen::dyn_cast<const Allen::Views::Velo::Consolidated::MultiEventTracks*>(imec[0]);
    if (m == nullptr) {
      counts[0] = 0xFFFFFFFFu; // not a VELO tracks container
      return;
    }
    unsigned at = 0, tracks_seen = 0;
    for (unsigned e = 0; e < m->number_of_events(); ++e) {
      const auto& tracks = m->container(e);
      if (tracks.offset() != tracks_seen) counts[2] = 0xFFFFFFFFu; // offsets out of order
      for (unsigned i = 0; i < tracks.size(); ++i) {
        const auto& t = tracks.track(i);
        for (unsigned j = 0; j < t.number_of_hits(); ++j) {
          const ::Velo::Hit v = t.hit(j);
          if (at < capacity) out[at] = HitRecord {v.LHCbID, v.x, v.y, v.z};
          ++at;
        }
      }
      tracks_seen += tracks.size();
    }
    counts[0] = m->number_of_events();
    counts[1] = tracks_seen;
    if (counts[2] != 0xFFFFFFFFu) counts[2] = at;
  }
} // namespace

// HarnessInput: the slice on the device and what Allen's non-event data would hold.
struct HarnessInput {
  const char* raw;
  const unsigned* offsets;
  const unsigned* sizes;
  const unsigned* types;
  size_t raw_bytes, sizes_words, types_words;
  unsigned event_start;
  unsigned n_events;   // host_number_of_events
  unsigned n_slice;    // events in the raw arrays
  int bank_version;
  const char* geometry; // velo_geometry.bin
  size_t geometry_size;
  float beamline_x, beamline_y;
};

extern "C" {

const char* allen_harness_error(void) { return last_error.c_str(); }

// Runs the adaptor and the reference's Kalman filter; returns a handle, or null (see the error).
void* allen_harness_run(const HarnessInput* in)
{
  auto h = std::make_unique<Harness>();
  try {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
      throw std::runtime_error("stream creation failed");
    // 1. Constants
    Constants constants {};
    {
      const VeloGeometry g {std::vector<char>(in->geometry, in->geometry + in->geometry_size)};
      if (cudaMalloc(&h->dev_geometry, sizeof(VeloGeometry)) != cudaSuccess ||
          cudaMemcpy(h->dev_geometry, &g, sizeof(VeloGeometry), cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("geometry upload failed");
      constants.dev_velo_geometry = h->dev_geometry;
      const float beamline[2] = {in->beamline_x, in->beamline_y};
      if (cudaMalloc(&h->dev_beamline, sizeof(beamline)) != cudaSuccess ||
          cudaMemcpy(h->dev_beamline, beamline, sizeof(beamline), cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("beamline upload failed");
      constants.dev_beamline = gsl::span<float> {h->dev_beamline, 2};
    }
    // 2. the algorithm's arguments
    Refs refs {make_arguments(*h, std::make_index_sequence<std::tuple_size_v<Tuple>> {})};
    unsigned host_n = in->n_events;
    int host_version = in->bank_version;
    auto bind = [&](auto& a, const void* p, size_t n) {
      a.set_pointer(const_cast<void*>(p));
      a.set_size(n);
    };
    using namespace velo_b200_chain;
    bind(arg<Parameters::host_number_of_events_t>(*h), &host_n, 1);
    bind(arg<Parameters::host_raw_bank_version_t>(*h), &host_version, 1);
    bind(arg<Parameters::dev_velo_raw_input_t>(*h), in->raw, in->raw_bytes);
    bind(arg<Parameters::dev_velo_raw_input_offsets_t>(*h), in->offsets, in->n_slice + 1);
    bind(arg<Parameters::dev_velo_raw_input_sizes_t>(*h), in->sizes, in->sizes_words);
    bind(arg<Parameters::dev_velo_raw_input_types_t>(*h), in->types, in->types_words);
    // 3. sizes, memory, operator()
    h->algorithm = std::make_unique<Chain>();
    const RuntimeOptions runtime_options {
      nullptr, 0, {in->event_start, in->event_start + in->n_events}, 1, false, 0, nullptr, nullptr};
    h->algorithm->set_arguments_size(refs, runtime_options, constants);
    allocate_outputs(*h, refs, std::make_index_sequence<std::tuple_size_v<Tuple>> {});
    Allen::Context context;
    context.initialize();
    (*h->algorithm)(refs, runtime_options, constants, context);
    if (cudaStreamSynchronize(context.stream()) != cudaSuccess) throw std::runtime_error("adaptor run failed");
    record_outputs(*h, refs, std::make_index_sequence<std::tuple_size_v<Tuple>> {});

    // 4. the reference's velo_kalman_filter on the adaptor's outputs
    const unsigned n = in->n_events;
    const unsigned reco = refs.template first<Parameters::host_number_of_reconstructed_velo_tracks_t>();
    {
      auto* event_list = static_cast<mask_t*>(device_alloc(*h, n * sizeof(mask_t)));
      std::vector<mask_t> list(n);
      for (unsigned e = 0; e < n; ++e)
        list[e] = mask_t {e};
      auto* dev_n = static_cast<unsigned*>(device_alloc(*h, sizeof(unsigned)));
      auto* is_backward = static_cast<bool*>(device_alloc(*h, std::max(reco, 1u)));
      const size_t state_bytes = size_t(std::max(reco, 1u)) * Velo::Consolidated::States::size;
      auto* beam = static_cast<char*>(device_alloc(*h, state_bytes));
      auto* end = static_cast<char*>(device_alloc(*h, state_bytes));
      auto* beam_view = static_cast<Allen::Views::Physics::KalmanStates*>(
        device_alloc(*h, n * sizeof(Allen::Views::Physics::KalmanStates)));
      auto* end_view = static_cast<Allen::Views::Physics::KalmanStates*>(
        device_alloc(*h, n * sizeof(Allen::Views::Physics::KalmanStates)));
      auto* histograms = static_cast<unsigned*>(device_alloc(*h, 9 * 64 * sizeof(unsigned)));
      if (cudaMemcpy(event_list, list.data(), n * sizeof(mask_t), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dev_n, &n, sizeof(unsigned), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemset(histograms, 0, 9 * 64 * sizeof(unsigned)) != cudaSuccess)
        throw std::runtime_error("Kalman inputs");
      velo_kalman_filter::Parameters k {};
      auto sp = [](auto* p, size_t count) { return Allen::device::span<std::remove_pointer_t<decltype(p)>> {p, count}; };
      k.host_number_of_reconstructed_velo_tracks = sp(static_cast<const unsigned*>(&reco), 1);
      k.host_number_of_events = sp(static_cast<const unsigned*>(&n), 1);
      k.dev_event_list = sp(static_cast<const mask_t*>(event_list), n);
      k.dev_number_of_events = sp(static_cast<const unsigned*>(dev_n), 1);
      k.dev_offsets_all_velo_tracks = sp(static_cast<const unsigned*>(refs.template data<Parameters::dev_offsets_all_velo_tracks_t>()), n + 1);
      k.dev_velo_tracks_view = sp(
        static_cast<const Allen::Views::Velo::Consolidated::Tracks*>(refs.template data<Parameters::dev_velo_tracks_view_t>()), n);
      k.dev_is_backward = sp(is_backward, reco);
      k.dev_velo_kalman_beamline_states = sp(beam, state_bytes);
      k.dev_velo_kalman_endvelo_states = sp(end, state_bytes);
      k.dev_velo_kalman_beamline_states_view = sp(beam_view, n);
      k.dev_velo_kalman_endvelo_states_view = sp(end_view, n);
      k.histogram_velo_track_eta_min = -10.f;
      k.histogram_velo_track_eta_max = 10.f;
      k.histogram_velo_track_eta_nbins = 40u;
      k.histogram_velo_track_phi_min = -4.f;
      k.histogram_velo_track_phi_max = 4.f;
      k.histogram_velo_track_phi_nbins = 16u;
      k.histogram_velo_track_nhits_min = 0.f;
      k.histogram_velo_track_nhits_max = 50.f;
      k.histogram_velo_track_nhits_nbins = 50u;
      auto hs = [&](unsigned i, unsigned nb) { return gsl::span<unsigned> {histograms + 64 * i, nb}; };
      velo_kalman_filter::velo_kalman_filter<<<n, 256, 0, h->stream>>>(
        k, h->dev_beamline, hs(0, 40), hs(1, 16), hs(2, 50), hs(3, 40), hs(4, 16), hs(5, 50), hs(6, 40), hs(7, 16),
        hs(8, 50));
      if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
        throw std::runtime_error("reference velo_kalman_filter failed");
      h->buffers["ref_kalman_is_backward"] = Buffer {is_backward, reco, true};
      h->buffers["ref_kalman_beamline_states"] = Buffer {beam, size_t(reco) * Velo::Consolidated::States::size, true};
      h->buffers["ref_kalman_endvelo_states"] = Buffer {end, size_t(reco) * Velo::Consolidated::States::size, true};
    }
    // 5. the views walked with the reference's types
    {
      const unsigned th = refs.template first<Parameters::host_accumulated_number_of_hits_in_velo_tracks_t>();
      auto* hits = static_cast<HitRecord*>(device_alloc(*h, size_t(std::max(th, 1u)) * sizeof(HitRecord)));
      auto* counts = static_cast<unsigned*>(device_alloc(*h, 3 * sizeof(unsigned)));
      if (cudaMemset(counts, 0, 3 * sizeof(unsigned)) != cudaSuccess) throw std::runtime_error("memset");
      walk_views<<<1, 1, 0, h->stream>>>(
        reinterpret_cast<Allen::IMultiEventContainer* const*>(refs.template data<Parameters::dev_imec_velo_tracks_t>()),
        hits, th, counts);
      if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
        throw std::runtime_error("view walk failed");
      h->buffers["walked_hits"] = Buffer {hits, size_t(th) * sizeof(HitRecord), true};
      h->buffers["walked_counts"] = Buffer {counts, 3 * sizeof(unsigned), true};
    }
  } catch (const std::exception& e) {
    last_error = e.what();
    return nullptr;
  }
  return h.release();
}

// One buffer by name: its pointer, bytes and whether it is device memory; 0 if unknown.
int allen_harness_buffer(void* handle, const char* name, void** ptr, size_t* bytes, int* device)
{
  auto* h = static_cast<Harness*>(handle);
  auto it = h->buffers.find(name);
  if (it == h->buffers.end()) return 0;
  *ptr = it->second.ptr;
  *bytes = it->second.bytes;
  *device = it->second.device ? 1 : 0;
  return 1;
}

// The names of every buffer, separated by spaces.
const char* allen_harness_names(void* handle)
{
  static thread_local std::string names;
  names.clear();
  for (auto& kv : static_cast<Harness*>(handle)->buffers)
    names += kv.first + " ";
  return names.c_str();
}

void allen_harness_free(void* handle) { delete static_cast<Harness*>(handle); }

// Host-only check of the view layouts (no GPU): the reference's view constructors, run on the
// host over small offset arrays, give byte for byte the structs of include/velo_b200.h filled
// as velo_create_velo_views fills them.  Returns 0 if they agree, else the number of the first
// view that differs (1 Hits, 2 Track, 3 Tracks, 4 MultiEventTracks).
int allen_harness_layout_check(void)
{
  namespace V = Allen::Views::Velo::Consolidated;
  constexpr unsigned n = 3, n_tracks = 5;
  const unsigned offsets_all[n + 1] = {0, 2, 2, 5};
  const unsigned hit_offsets[n_tracks + 1] = {0, 4, 9, 9, 13, 16};
  const char* base = reinterpret_cast<const char*>(0x1000);
  // the reference's objects in raw storage (constructed in place, never destroyed: trivial types)
  alignas(16) static unsigned char hits_raw[n][sizeof(V::Hits)];
  alignas(16) static unsigned char track_raw[n_tracks][sizeof(V::Track)];
  alignas(16) static unsigned char tracks_raw[n][sizeof(V::Tracks)];
  alignas(16) static unsigned char multi_raw[sizeof(V::MultiEventTracks)];
  std::memset(hits_raw, 0, sizeof(hits_raw));
  std::memset(track_raw, 0, sizeof(track_raw));
  std::memset(tracks_raw, 0, sizeof(tracks_raw));
  std::memset(multi_raw, 0, sizeof(multi_raw));
  const auto* ref_hits = reinterpret_cast<const V::Hits*>(hits_raw);
  const auto* ref_track = reinterpret_cast<const V::Track*>(track_raw);
  const auto* ref_tracks = reinterpret_cast<const V::Tracks*>(tracks_raw);
  for (unsigned e = 0; e < n; ++e) {
    new (hits_raw[e]) V::Hits(base, offsets_all, hit_offsets, e, n);
    VeloHitsView ours;
    std::memset(&ours, 0, sizeof(ours));
    ours.base_pointer = base;
    ours.offset = hit_offsets[offsets_all[e]];
    ours.size = hit_offsets[offsets_all[e + 1]] - hit_offsets[offsets_all[e]];
    ours.total_number_of_hits = hit_offsets[offsets_all[n]];
    if (std::memcmp(hits_raw[e], &ours, sizeof(ours)) != 0) return 1;
  }
  for (unsigned e = 0; e < n; ++e)
    for (unsigned t = 0; t < offsets_all[e + 1] - offsets_all[e]; ++t) {
      const unsigned g = offsets_all[e] + t;
      new (track_raw[g]) V::Track(ref_hits, offsets_all, hit_offsets, t, e);
      const unsigned* hn = hit_offsets + offsets_all[e];
      VeloTrackView ours;
      std::memset(&ours, 0, sizeof(ours));
      ours.hits = reinterpret_cast<const VeloHitsView*>(hits_raw[e]);
      ours.track_index = t;
      ours.track_container_offset = offsets_all[e];
      ours.offset = hn[t] - hn[0];
      ours.number_of_hits = hn[t + 1] - hn[t];
      if (std::memcmp(track_raw[g], &ours, sizeof(ours)) != 0) return 2;
    }
  for (unsigned e = 0; e < n; ++e) {
    new (tracks_raw[e]) V::Tracks(ref_track, offsets_all, e);
    VeloTracksView ours;
    std::memset(&ours, 0, sizeof(ours));
    ours.track = reinterpret_cast<const VeloTrackView*>(track_raw[offsets_all[e]]);
    ours.size = offsets_all[e + 1] - offsets_all[e];
    ours.offset = offsets_all[e];
    if (std::memcmp(tracks_raw[e], &ours, sizeof(ours)) != 0) return 3;
  }
  new (multi_raw) V::MultiEventTracks(ref_tracks, n);
  VeloMultiEventTracksView ours;
  std::memset(&ours, 0, sizeof(ours));
  ours.type_id = 1;
  ours.container = reinterpret_cast<const VeloTracksView*>(tracks_raw);
  ours.number_of_events = n;
  if (std::memcmp(multi_raw, &ours, sizeof(ours)) != 0) return 4;
  return 0;
}

} // extern "C"
