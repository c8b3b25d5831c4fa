"""MDF input: index the records of an MDF byte stream and transpose their VELO banks into
the Allen non-MEP layout that the chain reads (``include/velo_io.h``, ``libvelo_io.so``).

The reference's MDF provider reads records into a prefetch buffer and transposes one slice
per thread (main/include/MDFProvider.h, main/src/Transpose.cpp:112-498).  Here a slice is
transposed by all host threads at once: a sizing pass, a prefix sum, a writing pass.

    stream = mdf.read_file(path)              # bytes (or any buffer)
    index = mdf.scan(stream)                  # numpy structured array, one row per record
    slice_ = mdf.transpose_vp(stream, index)  # rawbanks.RawSlice for VeloChain.run()
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native
from .rawbanks import RawSlice

EVENT_DTYPE = np.dtype([("record_offset", "<u8"), ("banks_offset", "<u8"),
                        ("banks_bytes", "<u4"), ("record_bytes", "<u4")])

OK, ERR_ARGUMENT, ERR_CAPACITY, ERR_FORMAT, ERR_CHECKSUM, ERR_UNSUPPORTED = 0, 1, 3, 6, 7, 8


class TransposeInfoC(C.Structure):
    _fields_ = [("raw_bytes", C.c_size_t), ("sizes_bytes", C.c_size_t), ("types_bytes", C.c_size_t),
                ("n_banks", C.c_uint64), ("bank_version", C.c_int), ("empty_events", C.c_uint)]


class MdfError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what} (status {status})")
        self.status = status


_configured = False


def _lib():
    global _configured
    lib = _native.load_io()
    if not _configured:
        lib.velo_mdf_scan.restype = C.c_int
        lib.velo_mdf_scan.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_void_p, C.c_uint,
                                      C.POINTER(C.c_uint), C.POINTER(C.c_size_t)]
        lib.velo_mdf_select_by_source_id.restype = C.c_int
        lib.velo_mdf_select_by_source_id.argtypes = [C.c_void_p, C.c_void_p]
        lib.velo_transpose_vp.restype = C.c_int
        lib.velo_transpose_vp.argtypes = [C.c_void_p, C.c_void_p, C.c_uint, C.c_int, C.c_uint,
                                          C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t,
                                          C.c_void_p, C.c_size_t, C.POINTER(TransposeInfoC)]
        lib.velo_io_last_error.restype = C.c_char_p
        _configured = True
    return lib


def _as_u8(stream) -> np.ndarray:
    a = np.frombuffer(stream, dtype=np.uint8) if not isinstance(stream, np.ndarray) else stream.view(np.uint8)
    return np.ascontiguousarray(a.reshape(-1))


def read_file(path: str) -> np.ndarray:
    return np.fromfile(path, dtype=np.uint8)


def scan(stream, check_checksum: bool = False, max_events: int | None = None, batch: int = 65536) -> np.ndarray:
    """Index the complete records of ``stream``; raises MdfError on a bad, compressed or
    (with ``check_checksum``) corrupted record.  Indexes ``batch`` records per library call,
    each call resuming where the previous one stopped."""
    s = _as_u8(stream)
    lib = _lib()
    parts, pos = [], 0
    remaining = max_events if max_events is not None else None
    while pos < s.size and (remaining is None or remaining > 0):
        cap = batch if remaining is None else min(batch, remaining)
        events = np.zeros(cap, dtype=EVENT_DTYPE)
        n, used = C.c_uint(0), C.c_size_t(0)
        st = lib.velo_mdf_scan(s.ctypes.data + pos, s.size - pos, int(check_checksum), events.ctypes.data, cap,
                               C.byref(n), C.byref(used))
        if st != OK:
            raise MdfError(st, lib.velo_io_last_error().decode())
        if n.value == 0:
            break  # an incomplete record (or nothing) is left
        events = events[:n.value]
        events["record_offset"] += pos
        events["banks_offset"] += pos
        parts.append(events)
        pos += used.value
        if remaining is not None:
            remaining -= n.value
        if n.value < cap:
            break
    return np.concatenate(parts) if parts else np.zeros(0, dtype=EVENT_DTYPE)


def select_by_source_id(stream, event) -> bool:
    """Whether the stream's banks name their subdetector in their source IDs (decided, as the
    reference does, from one event: main/src/Transpose.cpp:34-58)."""
    s = _as_u8(stream)
    ev = np.asarray(event, dtype=EVENT_DTYPE).reshape(1)
    r = _lib().velo_mdf_select_by_source_id(s.ctypes.data, ev.ctypes.data)
    if r < 0:
        raise MdfError(ERR_FORMAT, "select_by_source_id: malformed banks")
    return bool(r)


def transpose_vp(stream, events: np.ndarray, by_source_id: bool | None = None,
                 n_threads: int = 0) -> RawSlice:
    """The VELO slice of ``events`` (Allen non-MEP layout) as a RawSlice."""
    s = _as_u8(stream)
    ev = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    if by_source_id is None:
        by_source_id = select_by_source_id(s, ev[0]) if ev.size else False
    lib = _lib()
    info = TransposeInfoC()
    n = int(ev.size)
    # upper bounds, so that one call does it: an event's slice bytes are at most its banks'
    # bytes plus the 8-byte preamble, and every bank takes at least 8 bytes of the record
    bank_bytes = int(ev["banks_bytes"].sum()) if n else 0
    raw = np.empty(max(bank_bytes + 8 * n, 1), dtype=np.uint8)
    offsets = np.empty(n + 1, dtype=np.uint32)
    sizes = np.empty((4 * (n + 1) + 2 * (bank_bytes // 8) + 3) // 4, dtype=np.uint32)
    types = np.empty((4 * (n + 1) + bank_bytes // 8 + 3) // 4, dtype=np.uint32)
    st = lib.velo_transpose_vp(s.ctypes.data, ev.ctypes.data, n, int(by_source_id), n_threads,
                               raw.ctypes.data, raw.size, offsets.ctypes.data, sizes.ctypes.data,
                               sizes.nbytes, types.ctypes.data, types.nbytes, C.byref(info))
    if st != OK:
        raise MdfError(st, lib.velo_io_last_error().decode())
    sizes = sizes[:info.sizes_bytes // 4]
    types = types[:info.types_bytes // 4]
    return RawSlice(raw=raw[:info.raw_bytes], offsets=offsets, sizes=sizes, types=types,
                    bank_version=int(info.bank_version))


def slices(stream, events_per_slice: int = 4000, check_checksum: bool = False, by_source_id: bool | None = None,
           n_threads: int = 0):
    """The VELO slices of consecutive groups of ``events_per_slice`` records of ``stream``, one
    RawSlice at a time (for HostPipeline: ``chain.pin_slice`` each)."""
    s = _as_u8(stream)
    index = scan(s, check_checksum=check_checksum)
    if by_source_id is None and index.size:
        by_source_id = select_by_source_id(s, index[0])
    for first in range(0, index.size, events_per_slice):
        yield transpose_vp(s, index[first:first + events_per_slice], by_source_id=bool(by_source_id),
                           n_threads=n_threads)


def write_records(events, header_version: int = 3, checksum: bool = True) -> bytes:
    """An MDF byte stream of uncompressed records (test and tooling helper).

    ``events``: per event a list of (bank_type, version, source_id, payload bytes).  Each bank
    is padded to 4 bytes; the header carries the one-at-a-time checksum when ``checksum``."""
    import struct
    sub_words = {0: 5, 1: 7, 2: 0, 3: 7}[header_version]
    out = bytearray()
    for banks in events:
        body = bytearray()
        for (btype, version, src, payload) in banks:
            length = 8 + len(payload)
            body += struct.pack("<HHBBH", 0xCBCB, length, btype, version, src) + bytes(payload)
            body += b"\0" * ((-length) % 4)
        size = 20 + 4 * sub_words + len(body)
        rest = bytes([0, (header_version << 4) | sub_words, 0, 0]) + b"\0" * (4 * sub_words) + bytes(body)
        csum = _one_at_a_time(rest) if checksum else 0
        out += struct.pack("<IIII", size, size, size, csum) + rest
    return bytes(out)


def _one_at_a_time(data: bytes) -> int:
    h = 0
    for b in data:
        h = (h + (b - 256 if b >= 128 else b)) & 0xFFFFFFFF  # the byte as a signed char
        h = (h + (h << 10)) & 0xFFFFFFFF
        h ^= h >> 6
    h = (h + (h << 3)) & 0xFFFFFFFF
    h ^= h >> 11
    h = (h + (h << 15)) & 0xFFFFFFFF
    return h
