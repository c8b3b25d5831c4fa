/*
 * Test infrastructure (oracle side): runs the reference's own MDF reader and transpose,
 * compiled as CPU C++ from their source files (main/src/Transpose.cpp,
 * mdf/src/read_mdf.cpp, mdf/src/raw_helpers.cpp, main/src/BankTypes.cpp), on an MDF byte
 * stream held in memory, and returns the VP slice it writes.
 *
 * Steps followed, as the reference's MDF provider takes them
 * (main/include/MDFProvider.h:150-175 and :540-560): read the first header, read_events()
 * into a prefetch buffer, check_sourceIDs() on the first event to pick the subdetector
 * and bank-order functions, fill_counts() on the first event, then transpose_events() into
 * one slice of bank type VP whose buffers are the caller's (zeroed first, as reset_slice()
 * does, main/src/SliceUtils.cpp:22-40).
 *
 * This file contains no reference code; it includes the reference headers and links the
 * reference objects built by oracle/Makefile.  Output goes to oracle/_ref/.
 */
#include <algorithm>
#include <chrono>
#include <cstring>
#include <unordered_set>
#include <vector>

#include <Transpose.h>

extern "C" int ref_transpose_vp(
  const char* stream,
  size_t stream_bytes,
  unsigned max_events,
  int check_checksum,
  char* raw,
  size_t raw_capacity,
  unsigned* offsets,  // [max_events + 1]
  unsigned* sizes,    // sizes_words
  size_t sizes_words,
  unsigned* types,    // types_words
  size_t types_words,
  unsigned* n_events, // events read
  unsigned* n_offsets,
  int* bank_version,
  int* by_source_id,
  double* transpose_seconds) // wall time of transpose_events alone
{
  size_t pos = 0;
  Allen::IO input;
  input.good = true;
  input.read = [&](char* dst, size_t n) -> ssize_t {
    const size_t k = std::min(n, stream_bytes - pos);
    std::memcpy(dst, stream + pos, k);
    pos += k;
    return static_cast<ssize_t>(k);
  };
  input.write = [](char const*, size_t) -> ssize_t { return -1; };
  input.close = [] {};

  LHCb::MDFHeader header;
  if (input.read(reinterpret_cast<char*>(&header), mdf_header_size) != static_cast<ssize_t>(mdf_header_size)) return 1;

  Allen::ReadBuffer read_buffer {0, std::vector<unsigned>(max_events + 1, 0), std::vector<char>(stream_bytes * 2 + (1 << 20)), 0};
  std::vector<char> compress_buffer(stream_bytes + (1 << 20));
  auto [eof, error, n_bytes] = read_events(input, read_buffer, header, compress_buffer, max_events, check_checksum != 0);
  (void) eof;
  (void) n_bytes;
  if (error) return 2;
  auto& [n_filled, event_offsets, buffer, transpose_start] = read_buffer;
  *n_events = static_cast<unsigned>(n_filled);
  if (n_filled == 0) return 3;

  gsl::span<char const> first_event {buffer.data(), event_offsets[1]};
  const bool is_mc = check_sourceIDs(first_event);
  Allen::sd_from_raw_bank sd_from_raw = is_mc ? Allen::sd_from_raw_bank {sd_from_bank_type} : Allen::sd_from_raw_bank {sd_from_sourceID};
  Allen::bank_sorter bank_sort = is_mc ? Allen::bank_sorter {sort_by_bank_type} : Allen::bank_sorter {sort_by_sourceID};
  *by_source_id = is_mc ? 0 : 1;
  std::unordered_set<LHCb::RawBank::BankType> skip_banks;
  auto [count_ok, mfp_count] = fill_counts(first_event, sd_from_raw, skip_banks);
  if (!count_ok) return 4;

  std::fill(offsets, offsets + max_events + 1, 0u);
  std::fill(sizes, sizes + sizes_words, 0u);
  std::fill(types, types + types_words, 0u);
  Allen::Slices slices;
  for (auto& s : slices)
    s.resize(1);
  auto& slice = slices[to_integral(BankTypes::VP)][0];
  slice.fragments.emplace_back(raw, raw_capacity);
  slice.fragments_mem_size = raw_capacity;
  slice.offsets = {offsets, static_cast<size_t>(max_events + 1)};
  slice.n_offsets = 1;
  slice.sizes = {sizes, sizes_words};
  slice.types = {types, types_words};

  std::array<int, NBankTypes> banks_version;
  banks_version.fill(-1);
  EventIDs event_ids;
  std::vector<char> event_mask(n_filled + 1, 0);
  std::unordered_set<BankTypes> bank_types {BankTypes::VP};
  const auto t0 = std::chrono::steady_clock::now();
  auto [ok, full, n_transposed] = transpose_events(
    read_buffer, slices, 0, bank_types, sd_from_raw, bank_sort, mfp_count, skip_banks, banks_version, event_ids,
    event_mask, n_filled, false);
  *transpose_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  (void) full;
  if (!ok || slice.fragments.size() != 1 || slice.fragments[0].data() != raw) return 5; // no re-allocation
  *n_offsets = static_cast<unsigned>(slice.n_offsets);
  *bank_version = banks_version[to_integral(BankTypes::VP)];
  return n_transposed == n_filled ? 0 : 6;
}
