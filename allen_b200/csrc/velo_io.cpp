// Host-side raw input path: MDF record index and the transpose of the VELO banks into the
// Allen non-MEP layout (C ABI in include/velo_io.h).
//
// Reference behaviour restated:
//   * record walk: mdf/src/read_mdf.cpp:113-241 (read_banks), main/src/Transpose.cpp:112-176
//     (read_events); header sizes mdf/include/mdf_header.hpp:149-161; checksum
//     mdf/src/raw_helpers.cpp:10-23 (Bob Jenkins' one-at-a-time hash, public domain);
//   * subdetector of a bank: main/src/Transpose.cpp:34-95 and main/include/BankMapping.h;
//   * bank order: main/include/Transpose.h:73-101 (sort_by_bank_type / sort_by_sourceID,
//     std::stable_sort at main/src/Transpose.cpp:282);
//   * slice layout: main/src/Transpose.cpp:293-454 and :475-483.
//
// The reference transposes one event after the other into a growing slice.  Here the events
// are independent work items: pass 1 sizes every event (and keeps its sorted bank list),
// an exclusive scan gives each event its offsets, and pass 2 writes the events in parallel.
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "velo_io.h"

namespace {

  thread_local std::string last_error;

  VeloIoStatus fail(VeloIoStatus s, const std::string& what)
  {
    last_error = what;
    return s;
  }

  // LHCb raw bank types used here (mdf/lhcb/Event/RawBank.h:69-134).
  constexpr unsigned type_velo = 8;
  constexpr unsigned type_daq = 15;
  constexpr unsigned type_odin = 16;
  constexpr unsigned type_hlt_dec_reports = 17;
  constexpr unsigned type_hlt_routing_bits = 53;
  constexpr unsigned type_hlt_sel_reports = 54;
  constexpr unsigned type_hlt_lumi_summary = 56;
  constexpr unsigned type_vp = 63;
  constexpr unsigned type_vp_retina_cluster = 73;
  // Source-ID subdetector codes of the VELO halves (mdf/daq40/sourceid.h:20-21).
  constexpr unsigned source_velo_a = 2;
  constexpr unsigned source_velo_c = 3;
  constexpr uint16_t bank_magic = 0xCBCB;
  constexpr unsigned bank_header_bytes = 8;
  constexpr unsigned mdf_base_header_bytes = 20;

  struct BankHeader {
    uint16_t magic;
    uint16_t length; // header + payload, without padding
    uint8_t type;
    uint8_t version;
    uint16_t source_id;
  };
  static_assert(sizeof(BankHeader) == bank_header_bytes, "raw bank header is 8 bytes");

  inline BankHeader read_bank_header(const unsigned char* p)
  {
    BankHeader h;
    std::memcpy(&h, p, sizeof(h));
    return h;
  }

  inline unsigned padded_length(unsigned length) { return (length + 3u) & ~3u; }

  // Types the reference never assigns to a subdetector (main/src/Transpose.cpp:6-11).
  inline bool uncounted_type(unsigned type)
  {
    return type == type_daq || type == type_hlt_dec_reports || type == type_hlt_sel_reports ||
           type == type_hlt_routing_bits || type == type_hlt_lumi_summary;
  }

  inline bool velo_bank_type(unsigned type)
  {
    return type == type_vp || type == type_velo || type == type_vp_retina_cluster;
  }

  // The bank-order functions treat only VP and VPRetinaCluster as VELO types (the legacy Velo
  // type goes with the other subdetectors), main/include/Transpose.h:75-76 and :97-98.
  inline bool ordered_as_velo(unsigned type) { return type == type_vp || type == type_vp_retina_cluster; }

  inline bool in_velo_slice(const BankHeader& h, bool by_source_id)
  {
    if (!by_source_id) return velo_bank_type(h.type);
    const unsigned sys = h.source_id >> 11;
    return (sys == source_velo_a || sys == source_velo_c) && !uncounted_type(h.type);
  }

  // MDF header size by header version; 0 for an unknown version.
  inline unsigned mdf_header_bytes(unsigned version)
  {
    switch (version) {
    case 0: return 40; // 20 + Header0 (22 bytes packed) - 2
    case 1: return 48; // 20 + Header1 (28 bytes)
    case 2: return 20;
    case 3: return 48;
    default: return 0;
    }
  }

  uint32_t one_at_a_time(const unsigned char* p, size_t n)
  {
    uint32_t hash = 0;
    for (size_t i = 0; i < n; ++i) {
      // the reference adds the byte as a (signed) char
      hash += static_cast<uint32_t>(static_cast<int32_t>(static_cast<signed char>(p[i])));
      hash += hash << 10;
      hash ^= hash >> 6;
    }
    hash += hash << 3;
    hash ^= hash >> 11;
    hash += hash << 15;
    return hash;
  }

  // One VELO bank of an event, as pass 1 leaves it for pass 2.
  struct Selected {
    uint64_t offset; // of the bank header in the stream
    uint16_t length;
    uint8_t type;
    uint8_t version;
    uint16_t source_id;
  };

  struct EventPlan {
    uint64_t first = 0; // index of the event's first bank in its worker's list
    uint32_t n_banks = 0;
    uint64_t bytes = 0; // of the event in the raw slice
    int version = -1;
  };

  struct WorkerError {
    VeloIoStatus status = VELO_IO_OK;
    unsigned event = 0;
    std::string what;
  };

  // Collect and order the VELO banks of one event; returns VELO_IO_OK or a format error.
  VeloIoStatus plan_event(
    const unsigned char* stream,
    const VeloMdfEvent& ev,
    bool by_source_id,
    std::vector<Selected>& list,
    std::vector<uint64_t>& keys,
    std::vector<Selected>& scratch,
    EventPlan& plan,
    std::string& what)
  {
    const uint64_t begin = ev.banks_offset, end = ev.banks_offset + ev.banks_bytes;
    plan.first = list.size();
    for (uint64_t p = begin; p < end;) {
      if (end - p < bank_header_bytes) {
        what = "bank header past the end of its record";
        return VELO_IO_ERR_FORMAT;
      }
      // the next header's address depends on this one's length: fetch the stream ahead
      __builtin_prefetch(stream + p + 1024);
      __builtin_prefetch(stream + p + 2048);
      const BankHeader h = read_bank_header(stream + p);
      if (h.magic != bank_magic) {
        what = "bad bank magic";
        return VELO_IO_ERR_FORMAT;
      }
      if (h.length < bank_header_bytes || padded_length(h.length) > end - p) {
        what = "bank length outside its record";
        return VELO_IO_ERR_FORMAT;
      }
      if (in_velo_slice(h, by_source_id)) list.push_back(Selected {p, h.length, h.type, h.version, h.source_id});
      p += padded_length(h.length);
    }
    auto first = list.begin() + static_cast<std::ptrdiff_t>(plan.first);
    const auto by_type = [](const Selected& a, const Selected& b) {
      const bool a_velo = ordered_as_velo(a.type), b_velo = ordered_as_velo(b.type);
      if (a_velo != b_velo) return a_velo;
      return a.type == b.type ? a.source_id < b.source_id : a.type < b.type;
    };
    // Selecting by type, and selecting by source ID when every selected bank is VP or
    // VPRetinaCluster, the order is the total order (VELO-type flag, type, source ID) with
    // ties in stream order: one sort of packed keys, no allocation.  Otherwise the reference's
    // comparator need not be a strict weak order, and std::stable_sort with it is used as is.
    bool keyed = !by_source_id;
    if (by_source_id) {
      keyed = true;
      for (auto it = first; it != list.end() && keyed; ++it)
        keyed = ordered_as_velo(it->type);
    }
    const size_t n = list.size() - plan.first;
    if (keyed && n <= (1u << 20)) {
      keys.resize(n);
      for (size_t i = 0; i < n; ++i) {
        const Selected& b = first[static_cast<std::ptrdiff_t>(i)];
        keys[i] = (uint64_t(ordered_as_velo(b.type) ? 0u : 1u) << 63) | (uint64_t(b.type) << 55) |
                  (uint64_t(b.source_id) << 39) | i;
      }
      std::sort(keys.begin(), keys.end());
      scratch.assign(first, list.end());
      for (size_t i = 0; i < n; ++i)
        first[static_cast<std::ptrdiff_t>(i)] = scratch[keys[i] & ((uint64_t(1) << 39) - 1)];
    }
    else if (by_source_id) {
      std::stable_sort(first, list.end(), [&by_type](const Selected& a, const Selected& b) {
        if (ordered_as_velo(a.type) && ordered_as_velo(b.type)) return by_type(a, b);
        return a.source_id < b.source_id;
      });
    }
    else {
      std::stable_sort(first, list.end(), by_type);
    }
    plan.n_banks = static_cast<uint32_t>(list.size() - plan.first);
    uint64_t bytes = 4ull * (2 + plan.n_banks);
    for (size_t i = plan.first; i < list.size(); ++i)
      bytes += 4 + padded_length(list[i].length) - bank_header_bytes;
    plan.bytes = bytes;
    plan.version = plan.n_banks ? list[plan.first].version : -1;
    return VELO_IO_OK;
  }

  inline void put32(unsigned char* dst, uint32_t v) { std::memcpy(dst, &v, 4); }
  inline void put16(unsigned char* dst, uint16_t v) { std::memcpy(dst, &v, 2); }

  template<typename F>
  void run_workers(unsigned n_threads, unsigned n_events, F&& body)
  {
    if (n_threads <= 1) {
      body(0u, 0u, n_events);
      return;
    }
    std::vector<std::thread> pool;
    pool.reserve(n_threads);
    for (unsigned t = 0; t < n_threads; ++t) {
      const unsigned lo = static_cast<unsigned>(uint64_t(n_events) * t / n_threads);
      const unsigned hi = static_cast<unsigned>(uint64_t(n_events) * (t + 1) / n_threads);
      pool.emplace_back([&body, t, lo, hi] { body(t, lo, hi); });
    }
    for (auto& th : pool)
      th.join();
  }

} // namespace

extern "C" VeloIoStatus velo_mdf_scan(
  const void* stream,
  size_t stream_bytes,
  int check_checksum,
  VeloMdfEvent* events,
  unsigned max_events,
  unsigned* n_events,
  size_t* bytes_used)
{
  if (!n_events || !bytes_used || (!stream && stream_bytes) || (!events && max_events))
    return fail(VELO_IO_ERR_ARGUMENT, "velo_mdf_scan: null argument");
  const auto* s = static_cast<const unsigned char*>(stream);
  *n_events = 0;
  *bytes_used = 0;
  size_t pos = 0;
  unsigned n = 0;
  while (n < max_events && stream_bytes - pos >= mdf_base_header_bytes) {
    uint32_t size0, checksum;
    std::memcpy(&size0, s + pos, 4);
    std::memcpy(&checksum, s + pos + 12, 4);
    const unsigned compression = s[pos + 16];
    const unsigned hdr = s[pos + 17];
    const unsigned header_bytes = mdf_header_bytes(hdr >> 4);
    const unsigned sub_header_bytes = (hdr & 0x0Fu) * 4u;
    if (header_bytes == 0 || mdf_base_header_bytes + sub_header_bytes != header_bytes || size0 < header_bytes) {
      *n_events = n;
      *bytes_used = pos;
      return fail(VELO_IO_ERR_FORMAT, "velo_mdf_scan: record " + std::to_string(n) + ": bad MDF header");
    }
    if (size0 > stream_bytes - pos) break; // incomplete record: resume from here
    if (compression & 0x0Fu) {
      *n_events = n;
      *bytes_used = pos;
      return fail(VELO_IO_ERR_UNSUPPORTED, "velo_mdf_scan: record " + std::to_string(n) + " is compressed");
    }
    if (check_checksum && checksum != 0 && one_at_a_time(s + pos + 16, size0 - 16) != checksum) {
      *n_events = n;
      *bytes_used = pos;
      return fail(VELO_IO_ERR_CHECKSUM, "velo_mdf_scan: record " + std::to_string(n) + ": checksum mismatch");
    }
    events[n] = VeloMdfEvent {pos, pos + header_bytes, size0 - header_bytes, size0};
    ++n;
    pos += size0;
  }
  *n_events = n;
  *bytes_used = pos;
  return VELO_IO_OK;
}

extern "C" int velo_mdf_select_by_source_id(const void* stream, const VeloMdfEvent* event)
{
  if (!stream || !event) return -1;
  const auto* s = static_cast<const unsigned char*>(stream);
  const uint64_t end = event->banks_offset + event->banks_bytes;
  uint64_t n_banks = 0, with_subdetector = 0;
  for (uint64_t p = event->banks_offset; p < end;) {
    if (end - p < bank_header_bytes) return -1;
    const BankHeader h = read_bank_header(s + p);
    if (h.magic != bank_magic || h.length < bank_header_bytes || padded_length(h.length) > end - p) return -1;
    if (!uncounted_type(h.type)) {
      with_subdetector += (h.source_id >> 11) != 0;
      ++n_banks;
    }
    p += padded_length(h.length);
  }
  // In real data only the ODIN bank has no subdetector bits.
  return n_banks - with_subdetector == 1 ? 1 : 0;
}

extern "C" VeloIoStatus velo_transpose_vp(
  const void* stream,
  const VeloMdfEvent* events,
  unsigned n_events,
  int select_by_source_id,
  unsigned n_threads,
  void* raw,
  size_t raw_capacity,
  uint32_t* offsets,
  uint32_t* sizes,
  size_t sizes_capacity,
  uint32_t* types,
  size_t types_capacity,
  VeloTransposeInfo* info)
{
  if (!info || (n_events && (!stream || !events)))
    return fail(VELO_IO_ERR_ARGUMENT, "velo_transpose_vp: null argument");
  const auto* s = static_cast<const unsigned char*>(stream);
  const bool by_source_id = select_by_source_id != 0;
  if (n_threads == 0) n_threads = std::max(1u, std::thread::hardware_concurrency());
  n_threads = std::min(n_threads, std::max(1u, n_events / 64u)); // at least 64 events per thread

  // Pass 1: per event its ordered VELO banks and its size.
  std::vector<EventPlan> plans(n_events);
  std::vector<std::vector<Selected>> lists(n_threads);
  std::vector<WorkerError> errors(n_threads);
  run_workers(n_threads, n_events, [&](unsigned t, unsigned lo, unsigned hi) {
    auto& list = lists[t];
    list.reserve(size_t(hi - lo) * 256);
    std::vector<uint64_t> keys;
    std::vector<Selected> scratch;
    for (unsigned e = lo; e < hi; ++e) {
      std::string what;
      const VeloIoStatus st = plan_event(s, events[e], by_source_id, list, keys, scratch, plans[e], what);
      if (st != VELO_IO_OK) {
        errors[t] = WorkerError {st, e, what};
        return;
      }
    }
  });
  for (const auto& err : errors) // workers cover increasing event ranges: the first error is the lowest event
    if (err.status != VELO_IO_OK)
      return fail(err.status, "velo_transpose_vp: event " + std::to_string(err.event) + ": " + err.what);

  // Exclusive scan of event sizes, bank counts; the slice version is the last event's.
  uint64_t raw_bytes = 0, n_banks = 0;
  int version = -1;
  unsigned empty = 0;
  for (unsigned e = 0; e < n_events; ++e) {
    raw_bytes += plans[e].bytes;
    n_banks += plans[e].n_banks;
    if (plans[e].n_banks) version = plans[e].version;
    else ++empty;
  }
  info->raw_bytes = raw_bytes;
  info->sizes_bytes = (4ull * (n_events + 1) + 2ull * n_banks + 3) & ~3ull;
  info->types_bytes = (4ull * (n_events + 1) + n_banks + 3) & ~3ull;
  info->n_banks = n_banks;
  info->bank_version = version;
  info->empty_events = empty;
  if (raw_bytes > 0xFFFFFFFFull || 2ull * (n_events + 1) + n_banks > 0xFFFFFFFFull)
    return fail(VELO_IO_ERR_CAPACITY, "velo_transpose_vp: slice exceeds 32-bit offsets; transpose fewer events");
  if (!raw || !offsets || !sizes || !types || raw_capacity < raw_bytes || sizes_capacity < info->sizes_bytes ||
      types_capacity < info->types_bytes)
    return fail(VELO_IO_ERR_CAPACITY, "velo_transpose_vp: output buffers too small");

  // Offsets of every event in the three arrays.
  auto* sizes8 = reinterpret_cast<unsigned char*>(sizes);
  auto* types8 = reinterpret_cast<unsigned char*>(types);
  uint32_t raw_off = 0, size_off = 2u * (n_events + 1), type_off = 4u * (n_events + 1);
  for (unsigned e = 0; e < n_events; ++e) {
    put32(reinterpret_cast<unsigned char*>(offsets + e), raw_off);
    put32(sizes8 + 4ull * e, size_off);
    put32(types8 + 4ull * e, type_off);
    raw_off += static_cast<uint32_t>(plans[e].bytes);
    size_off += plans[e].n_banks;
    type_off += plans[e].n_banks;
  }
  put32(reinterpret_cast<unsigned char*>(offsets + n_events), raw_off);
  put32(sizes8 + 4ull * n_events, size_off);
  put32(types8 + 4ull * n_events, type_off);
  std::memset(sizes8 + 2ull * size_off, 0, info->sizes_bytes - 2ull * size_off);
  std::memset(types8 + type_off, 0, info->types_bytes - type_off);

  // Pass 2: every event at its offsets.
  auto* out = static_cast<unsigned char*>(raw);
  run_workers(n_threads, n_events, [&](unsigned t, unsigned lo, unsigned hi) {
    const auto& list = lists[t];
    for (unsigned e = lo; e < hi; ++e) {
      const EventPlan& plan = plans[e];
      uint32_t ev_off, sz_off, ty_off;
      std::memcpy(&ev_off, offsets + e, 4);
      std::memcpy(&sz_off, sizes8 + 4ull * e, 4);
      std::memcpy(&ty_off, types8 + 4ull * e, 4);
      unsigned char* w = out + ev_off;
      put32(w, plan.n_banks);
      put32(w + 4, 0);
      unsigned char* payload = w + 4ull * (2 + plan.n_banks);
      uint32_t bank_off = 0;
      for (uint32_t i = 0; i < plan.n_banks; ++i) {
        const Selected& b = list[plan.first + i];
        const unsigned data_bytes = padded_length(b.length) - bank_header_bytes;
        put32(payload + bank_off, b.source_id);
        std::memcpy(payload + bank_off + 4, s + b.offset + bank_header_bytes, data_bytes);
        bank_off += 4 + data_bytes;
        put32(w + 4ull * (2 + i), bank_off);
        put16(sizes8 + 2ull * (sz_off + i), static_cast<uint16_t>(b.length - bank_header_bytes));
        types8[ty_off + i] = b.type;
      }
    }
  });
  last_error.clear();
  return VELO_IO_OK;
}

extern "C" const char* velo_io_last_error(void) { return last_error.c_str(); }
