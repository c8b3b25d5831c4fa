/*
 * C ABI of the host-side raw input path (libvelo_io.so): MDF records -> the Allen
 * non-MEP layout of the VELO banks, which is what velo_chain_run() reads.
 *
 * The reference reads MDF files record by record into a prefetch buffer
 * (main/src/Transpose.cpp:112-176 read_events, mdf/src/read_mdf.cpp:113-241 read_banks)
 * and then transposes each event's banks into one Allen-layout slice per subdetector
 * (main/src/Transpose.cpp:220-454 transpose_event, :456-498 transpose_events), one slice
 * per thread.  This library does the same for the VELO slice, in two steps:
 *
 *   velo_mdf_scan()      indexes the records of an MDF byte stream held in host memory
 *                        (no copy: the transpose reads the banks where they lie);
 *   velo_transpose_vp()  writes the VELO slice of a range of indexed events: a parallel
 *                        pass that sizes every event, one prefix sum, and a parallel pass
 *                        that writes each event at its offset (any number of threads).
 *
 * The output buffers are what velo_chain_run() takes as dev_velo_raw_input,
 * dev_velo_raw_input_offsets, dev_velo_raw_input_sizes, dev_velo_raw_input_types and
 * host_raw_bank_version once copied to the device; written into page-locked host memory
 * they are copied with one cudaMemcpyAsync each.
 *
 * Why on the host: an MDF event carries every subdetector's banks (the 2018 minbias sample:
 * 1238 banks, 118-349 KB per event, of which the VELO banks are about 10 %), so moving whole
 * records over PCIe to transpose them on the GPU would copy ten times the bytes the chain
 * needs.  MEP input needs no transpose at all: the kernels read MEP fragments in place
 * (VeloDeviceSlice.mep_layout).
 *
 * Plain pointers and sizes; every function returns a VeloIoStatus.  No CUDA dependency.
 */
#ifndef VELO_IO_H
#define VELO_IO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  VELO_IO_OK = 0,
  VELO_IO_ERR_ARGUMENT = 1,    /* null pointer or inconsistent sizes */
  VELO_IO_ERR_CAPACITY = 3,    /* an output buffer is too small; VeloTransposeInfo holds the sizes needed */
  VELO_IO_ERR_FORMAT = 6,      /* unknown MDF header version, bad bank magic, bank past its record */
  VELO_IO_ERR_CHECKSUM = 7,    /* record checksum differs from the header's (only when checking) */
  VELO_IO_ERR_UNSUPPORTED = 8  /* compressed record (the reference inflates these with ROOT's zip) */
} VeloIoStatus;

/* One MDF record.  Offsets are bytes from the start of the scanned stream. */
typedef struct {
  uint64_t record_offset; /* the MDF header */
  uint64_t banks_offset;  /* the first raw bank (after header and sub-header) */
  uint32_t banks_bytes;   /* raw banks of the event: record size - header size */
  uint32_t record_bytes;  /* bytes from record_offset to the next record */
} VeloMdfEvent;

/* Index the complete MDF records of `stream` (host memory).
 *
 * Replaces the record loop of read_events / read_banks (main/src/Transpose.cpp:112-176,
 * mdf/src/read_mdf.cpp:113-241): the header gives the record size, the header version
 * the header size (40, 48, 20 and 48 bytes for versions 0-3,
 * mdf/include/mdf_header.hpp:149-161), which the 20-byte header and its sub-header (4 x the
 * low nibble of the header-type byte) must fill; the banks follow it up to the record
 * size.  With check_checksum != 0 a non-zero header checksum is compared with the
 * one-at-a-time hash of the record from its compression byte on
 * (mdf/src/read_mdf.cpp:166-179, mdf/src/raw_helpers.cpp:10-23).
 * Stops at the end of the stream, after max_events records, or before an incomplete record;
 * *bytes_used = the end of the last record indexed (where a next call resumes).
 * Errors: a compressed record (VELO_IO_ERR_UNSUPPORTED), an unknown header version or a
 * record smaller than its header (VELO_IO_ERR_FORMAT), a checksum mismatch
 * (VELO_IO_ERR_CHECKSUM); the records before the bad one stay indexed in *n_events. */
VeloIoStatus velo_mdf_scan(
  const void* stream,
  size_t stream_bytes,
  int check_checksum,
  VeloMdfEvent* events,
  unsigned max_events,
  unsigned* n_events,
  size_t* bytes_used);

/* 1 when the banks of one event name their subdetector in the five top bits of the source
 * ID (real data, recent simulation), 0 when only the bank type does (older simulation,
 * e.g. the 2018 minbias sample).  Restates check_sourceIDs (main/src/Transpose.cpp:34-58),
 * which the reference applies to the first event of a file (main/include/MDFProvider.h:158-169).
 * Returns -1 on a bad bank magic or a bank past the end. */
int velo_mdf_select_by_source_id(const void* stream, const VeloMdfEvent* event);

typedef struct {
  size_t raw_bytes;         /* bytes of dev_velo_raw_input written (= offsets[n_events]) */
  size_t sizes_bytes;       /* bytes of dev_velo_raw_input_sizes: 4 (n+1) + 2 banks, rounded up to 4 */
  size_t types_bytes;       /* bytes of dev_velo_raw_input_types: 4 (n+1) + banks, rounded up to 4 */
  uint64_t n_banks;         /* VELO banks in the slice */
  int bank_version;         /* host_raw_bank_version: version of the last event's first VELO bank; -1 if none */
  unsigned empty_events;    /* events without any VELO bank (written with zero banks) */
} VeloTransposeInfo;

/* Write the VELO slice (Allen non-MEP layout) of events[0 .. n_events) of `stream`.
 *
 * Replaces transpose_event / transpose_events (main/src/Transpose.cpp:220-498) for the VP
 * slice.  A bank belongs to the slice when its type is VP (63), Velo (8) or VPRetinaCluster
 * (73) (select_by_source_id = 0; main/include/BankMapping.h:13-16), or when the five top
 * bits of its source ID are VELO_A or VELO_C and its type is not DAQ or an Hlt summary
 * (select_by_source_id = 1; main/src/Transpose.cpp:83-95).  Per event the banks are ordered
 * as the reference orders them (main/include/Transpose.h:73-101, stable): selecting by type,
 * VP and VPRetinaCluster banks first, then by bank type and source ID; selecting by source
 * ID, by source ID except between two VP / VPRetinaCluster banks, which compare by type
 * first.  Each event is written as: bank count, n+1 bank offsets, then per bank its
 * source ID and its padded payload; the sizes array holds 16-bit payload sizes after n+1
 * offsets in 16-bit units (first = 2 (n+1)), the types array 8-bit bank types after n+1
 * offsets in bytes (first = 4 (n+1)).  Unused bytes of the last word of sizes and types are
 * zero.
 *
 * One difference: an event without any VELO bank is written as an event with zero banks,
 * where the reference writes nothing for it and so shifts every later event of the slice.
 *
 * n_threads = 0 uses all hardware threads.  When a buffer is too small nothing is written,
 * *info holds the sizes needed, and VELO_IO_ERR_CAPACITY is returned; info may be passed
 * with null buffers to size them.  offsets has n_events + 1 entries. */
VeloIoStatus velo_transpose_vp(
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
  VeloTransposeInfo* info);

/* Text of the last error of the calling thread ("" if none). */
const char* velo_io_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
