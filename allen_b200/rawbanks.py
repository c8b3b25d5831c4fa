"""Allen raw-bank layout (non-MEP) for VP super-pixel banks, on the host.

A slice of N events is four arrays (main/src/Transpose.cpp:333-425; readers in
device/event_model/velo/include/ClusteringDefinitions.cuh:97-144 and
main/include/MEPTools.h:26-53):

* ``raw``      bytes; per event ``n_banks`` (u32), ``bank_offsets[n_banks + 1]``
               (u32, bytes from the payload start), then per bank its sourceID
               (u32) followed by the bank data padded to 4 bytes;
* ``offsets``  u32[N + 1], byte offset of each event blob in ``raw``;
* ``sizes``    u32[N + 1] offsets in u16 units from the array start, followed by
               the u16 payload size of every bank;
* ``types``    u32[N + 1] offsets in u8 units from the array start, followed by
               the u8 bank type of every bank (VP = 63, Velo = 8).

The MEP layout (``mep = True``; readers in main/include/MEPTools.h:55-205) keeps the
banks of one source together: ``offsets`` = [n_banks, n_events, source_id[n_banks],
then for each event the byte offset in ``raw`` of its fragment of every bank];
``sizes`` and ``types`` start with one u32 offset per bank (u16 and u8 units)
followed by that bank's per-event sizes and types.  A fragment is the bank data
without the sourceID word.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BANK_TYPE_VELO = 8
BANK_TYPE_VP = 63
BANK_TYPE_VP_RETINA = 73  # LHCb::RawBank::VPRetinaCluster


@dataclass
class RawSlice:
    raw: np.ndarray      # uint8
    offsets: np.ndarray  # uint32[N + 1]
    sizes: np.ndarray    # uint32
    types: np.ndarray    # uint32
    bank_version: int
    mep: bool = False    # MEP layout (banks of one source together)

    @property
    def n_events(self) -> int:
        if self.mep:
            return int(self.offsets[1])
        return int(self.offsets.shape[0] - 1)

    @property
    def retina(self) -> bool:
        """The slice carries retina-cluster banks (type 73) rather than super-pixel banks."""
        if self.n_events == 0:
            return False
        t8 = self.types.view(np.uint8)
        if self.mep:
            n_banks = int(self.offsets[0])
            return bool(any(np.any(t8[int(self.types[b]):int(self.types[b]) + self.n_events] == BANK_TYPE_VP_RETINA)
                            for b in range(n_banks)))
        first, last = int(self.types[0]), int(self.types[1]) if self.n_events > 1 else t8.size
        return bool(np.any(t8[first:first + max(last - first, 0)] == BANK_TYPE_VP_RETINA))

    def n_super_pixels(self) -> int:
        """Total super pixels of the slice, from the bank sizes alone (no payload read)."""
        return int(super_pixels_per_event(self).sum())


def build_slice(events, bank_version: int) -> RawSlice:
    """events: list (per event) of lists of (bank_type, source_id, payload bytes)."""
    n = len(events)
    blobs, sizes16, types8 = [], [], []
    for banks in events:
        words = [np.array([len(banks)], dtype=np.uint32)]
        offs = [0]
        datas = []
        for (btype, src, payload) in banks:
            pad = (-len(payload)) % 4
            d = np.frombuffer(bytes(payload) + b"\0" * pad, dtype=np.uint32)
            datas.append(np.concatenate([np.array([src], dtype=np.uint32), d]))
            offs.append(offs[-1] + 4 * (1 + d.size))
            sizes16.append(len(payload))
            types8.append(btype)
        words.append(np.array(offs, dtype=np.uint32))
        words.extend(datas)
        blobs.append(np.concatenate(words).view(np.uint8))
    offsets = np.zeros(n + 1, dtype=np.uint32)
    offsets[1:] = np.cumsum([b.size for b in blobs])
    raw = np.concatenate(blobs) if blobs else np.zeros(0, np.uint8)
    nb = np.array([len(b) for b in events], dtype=np.int64)
    first16, first8 = 2 * (n + 1), 4 * (n + 1)
    size_offs = first16 + np.concatenate([[0], np.cumsum(nb)])
    type_offs = first8 + np.concatenate([[0], np.cumsum(nb)])
    s16 = np.zeros(first16 + int(nb.sum()) + 1, dtype=np.uint16)
    s16.view(np.uint8)[: 4 * (n + 1)] = size_offs.astype(np.uint32).view(np.uint8)
    s16[first16:first16 + len(sizes16)] = np.array(sizes16, dtype=np.uint16)
    t8 = np.zeros(first8 + int(nb.sum()) + 3, dtype=np.uint8)
    t8[: 4 * (n + 1)] = type_offs.astype(np.uint32).view(np.uint8)
    t8[first8:first8 + len(types8)] = np.array(types8, dtype=np.uint8)
    sizes = np.frombuffer(s16.tobytes() + b"\0" * ((-s16.nbytes) % 4), dtype=np.uint32).copy()
    types = np.frombuffer(t8.tobytes() + b"\0" * ((-t8.nbytes) % 4), dtype=np.uint32).copy()
    return RawSlice(raw, offsets, sizes, types, bank_version)


def banks_of_event(s: RawSlice, event: int):
    """Decodes one event back into (bank_type, source_id, payload bytes) tuples."""
    base = int(s.offsets[event])
    blob = s.raw[base:int(s.offsets[event + 1])]
    w = blob.view(np.uint32)
    n_banks = int(w[0])
    offs = w[1:n_banks + 2]
    payload_start = 4 * (n_banks + 2)
    s16 = s.sizes.view(np.uint16)
    t8 = s.types.view(np.uint8)
    so, to = int(s.sizes[event]), int(s.types[event])
    out = []
    for b in range(n_banks):
        p = payload_start + int(offs[b])
        src = int(blob[p:p + 4].view(np.uint32)[0])
        size = int(s16[so + b])
        out.append((int(t8[to + b]), src, bytes(blob[p + 4:p + 4 + size])))
    return out


def super_pixels_per_event(s: RawSlice) -> np.ndarray:
    """Super pixels (or retina clusters) per event from the bank sizes: (size - 4) / 4 for
    v2/v3 (count word first), size / 4 for v4.  Upper bound used to size device buffers
    before launch."""
    n = s.n_events
    s16 = s.sizes.view(np.uint16)
    t8 = s.types.view(np.uint8)
    out = np.zeros(n, dtype=np.int64)
    if s.mep:
        for b in range(int(s.offsets[0])):
            sz = s16[int(s.sizes[b]):int(s.sizes[b]) + n].astype(np.int64)
            ty = t8[int(s.types[b]):int(s.types[b]) + n]
            words = np.where((ty == BANK_TYPE_VP) | (ty == BANK_TYPE_VELO) | (ty == BANK_TYPE_VP_RETINA), sz // 4, 0)
            if s.bank_version in (2, 3):
                words = np.maximum(words - 1, 0)
            out += words
        return out
    starts = s.sizes[:n + 1].astype(np.int64)
    tstarts = s.types[:n + 1].astype(np.int64)
    for e in range(n):
        sz = s16[starts[e]:starts[e + 1]].astype(np.int64)
        ty = t8[tstarts[e]:tstarts[e] + sz.size]
        sel = (ty == BANK_TYPE_VP) | (ty == BANK_TYPE_VELO) | (ty == BANK_TYPE_VP_RETINA)
        words = sz[sel] // 4
        if s.bank_version in (2, 3):
            words = np.maximum(words - 1, 0)
        out[e] = words.sum()
    return out


def to_mep(s: RawSlice) -> RawSlice:
    """The same events in the MEP layout.  Every event must have the same banks (sources) in
    the same order, as a MEP's events do."""
    assert not s.mep
    n = s.n_events
    per_event = [banks_of_event(s, e) for e in range(n)]
    n_banks = len(per_event[0]) if n else 0
    assert all(len(b) == n_banks and [x[1] for x in b] == [x[1] for x in per_event[0]] for b in per_event)
    offsets = np.zeros(2 + n_banks * (n + 1), dtype=np.uint32)
    offsets[0], offsets[1] = n_banks, n
    chunks, pos = [], 0
    for b in range(n_banks):
        offsets[2 + b] = per_event[0][b][1]
        for e in range(n):
            payload = per_event[e][b][2]
            offsets[2 + n_banks * (1 + e) + b] = pos
            data = payload + b"\0" * ((-len(payload)) % 4)
            chunks.append(data)
            pos += len(data)
    raw = np.frombuffer(b"".join(chunks), dtype=np.uint8).copy() if chunks else np.zeros(0, np.uint8)
    s16 = np.zeros(2 * n_banks + n_banks * n + 2, dtype=np.uint16)
    t8 = np.zeros(4 * n_banks + n_banks * n + 4, dtype=np.uint8)
    for b in range(n_banks):
        so, to = 2 * n_banks + b * n, 4 * n_banks + b * n
        s16.view(np.uint32)[b] = so
        t8.view(np.uint32)[b] = to
        s16[so:so + n] = [len(per_event[e][b][2]) for e in range(n)]
        t8[to:to + n] = [per_event[e][b][0] for e in range(n)]
    sizes = np.frombuffer(s16.tobytes() + b"\0" * ((-s16.nbytes) % 4), dtype=np.uint32).copy()
    types = np.frombuffer(t8.tobytes() + b"\0" * ((-t8.nbytes) % 4), dtype=np.uint32).copy()
    return RawSlice(raw, offsets, sizes, types, s.bank_version, mep=True)
