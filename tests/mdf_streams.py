"""Synthetic MDF byte streams for the raw input tests (test infrastructure).

An event of a generated RawSlice becomes an MDF record holding its VELO banks plus banks of
other subdetectors, an ODIN bank and a DAQ bank, in shuffled order, so that the transpose
has to select and re-order them.  With ``by_source_id`` every bank but ODIN carries its
subdetector in the five top bits of its source ID (real-data style), otherwise none does
(older simulation); the VELO banks' low source-ID bits are their sensor (pair) number.
"""
from __future__ import annotations

import numpy as np

from allen_b200 import mdf, rawbanks

OTHER_TYPES = [9, 13, 21, 22, 32, 33, 64, 66]   # UT, FT, Muon, Calo, ... (not VELO)
OTHER_SYSTEMS = [4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14]
VELO_TYPES = {8, 63, 73}


def velo_source(src: int, by_source_id: bool) -> int:
    if not by_source_id:
        return src
    return ((2 if src < 104 else 3) << 11) | (src & 0x7FF)


def event_banks(s: rawbanks.RawSlice, e: int, rng, by_source_id: bool, n_other: int,
                extra_velo: bool = False, drop_velo: bool = False):
    banks = []
    if not drop_velo:
        for (btype, src, payload) in rawbanks.banks_of_event(s, e):
            banks.append((btype, s.bank_version, velo_source(src, by_source_id), payload))
    if extra_velo:
        # more VELO-type banks, some with the source ID of an existing bank: order and stability.
        # Selecting by source ID, a legacy Velo (8) bank among VP banks makes the reference's
        # bank order depend on the other subdetectors' banks (its comparator is then not a
        # strict weak order), so that mode gets VP and VPRetinaCluster banks only.
        for k in range(6):
            btype = int(rng.choice([63, 73] if by_source_id else [8, 63, 73]))
            src = int(rng.integers(0, 208)) if k % 2 else (banks[0][2] & 0x7FF if banks else 5)
            payload = rng.integers(0, 256, int(rng.integers(4, 40))).astype(np.uint8).tobytes()
            banks.append((btype, int(rng.integers(2, 5)), velo_source(src, by_source_id), payload))
    for _ in range(n_other):
        btype = int(rng.choice(OTHER_TYPES))
        src = int(rng.integers(0, 1 << 11))
        if by_source_id:
            src |= int(rng.choice(OTHER_SYSTEMS)) << 11
        payload = rng.integers(0, 256, int(rng.integers(0, 90))).astype(np.uint8).tobytes()
        banks.append((btype, int(rng.integers(0, 8)), src, payload))
    odin = rng.integers(0, 1 << 32, 10, dtype=np.uint64).astype(np.uint32).tobytes()
    banks.append((16, 7, 0 if by_source_id else 0, odin))
    order = rng.permutation(len(banks))
    banks = [banks[i] for i in order]
    # the DAQ bank (type 15) is never counted or selected; put it first as the reader does
    daq = rng.integers(0, 256, 48).astype(np.uint8).tobytes()
    return [(15, 1, 0, daq)] + banks


def synthetic_stream(s: rawbanks.RawSlice, seed: int, by_source_id: bool = False, n_other: int = 40,
                     header_version: int = 3, extra_velo: bool = False, drop_velo_events=()) -> bytes:
    rng = np.random.default_rng(seed)
    events = [event_banks(s, e, rng, by_source_id, n_other, extra_velo, e in drop_velo_events)
              for e in range(s.n_events)]
    return mdf.write_records(events, header_version=header_version)
