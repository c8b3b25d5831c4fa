"""The reference's contract checks on the VELO chain's outputs, restated over numpy arrays.

The reference runs these as debug-build contracts after its algorithms:
  * cluster_container_checks, device/velo/search_by_triplet/src/SearchByTripletContracts.cu:6-81:
    per module pair the sorted container is strictly increasing in (phi, id, x, y), and every
    cluster has -100 < x < 100 and -100 < y < 100 (mm);
  * track_container_checks, SearchByTripletContracts.cu:83-120: every track of dev_tracks has
    at most 26 hits and no hit twice;
  * lhcb_id_container_checks, device/velo/consolidate_tracks/src/VeloConsolidateTracks.cu:194-269:
    every LHCb id of a consolidated track is non-zero and has the VELO detector type (0x2) in
    its top four bits, and each event's track count equals its id-sequence count (true by
    construction of the views from the same offsets, checked here as offsets that never
    decrease and end at the hit count).
They are invariants, not golden values: they hold for plain and learned modes alike, which
is what makes them the structural check of the learned search, whose tracks have no
bit-exact oracle.  ``check(outputs, n_events)`` returns the violated contracts (empty when
all hold), each with a count.
"""
from __future__ import annotations

import numpy as np

import parity

N_MP = 26
MAX_TRACK_SIZE = 26
VELO_TYPE = 0x2


def cluster_container(out: dict) -> list[str]:
    off = np.asarray(out["dev_offsets_estimated_input_size"], dtype=np.int64)
    num = np.asarray(out["dev_module_cluster_num"], dtype=np.int64)
    T = int(off[-1])
    ids, xyz, phi = parity.container_fields(out["dev_sorted_velo_cluster_container"], T)
    bad = []
    mask = parity.sorted_container_mask(off, num, T)
    x, y = xyz[:, 0], xyz[:, 1]
    n_xy = int((~((x > -100.0) & (x < 100.0) & (y > -100.0) & (y < 100.0)) & mask).sum())
    if n_xy:
        bad.append(f"cluster x or y outside (-100, 100) mm: {n_xy}")
    # consecutive slots inside one module pair: (phi, id, x, y) strictly increasing
    nxt = np.zeros(T, dtype=bool)  # slot i and i + 1 are in the same module pair
    for s, n in zip(off[:-1], num):
        if n > 1:
            nxt[s:s + n - 1] = True
    i = np.nonzero(nxt)[0]
    p0, p1 = phi[i].astype(np.int32), phi[i + 1].astype(np.int32)
    d0, d1 = ids[i], ids[i + 1]
    x0, x1, y0, y1 = x[i], x[i + 1], y[i], y[i + 1]
    ok = (p1 > p0) | ((p1 == p0) & (d1 > d0)) | ((p1 == p0) & (d1 == d0) & (x1 > x0)) | \
         ((p1 == p0) & (d1 == d0) & (x1 == x0) & (y1 > y0))
    n_unsorted = int((~ok).sum())
    if n_unsorted:
        bad.append(f"module pair not sorted in (phi, id): {n_unsorted} pairs of neighbours")
    return bad


def track_container(out: dict, n_events: int) -> list[str]:
    off = np.asarray(out["dev_offsets_estimated_input_size"])
    counts = np.asarray(out["dev_number_of_velo_tracks"])
    bad_size = repeated = 0
    for e in range(n_events):
        n = int(counts[e])
        if n == 0:
            continue
        hits, hits_num = parity.track_track_fields(out["dev_tracks"], parity.track_offset(off, e), n)
        bad_size += int((hits_num > MAX_TRACK_SIZE).sum())
        for t in range(n):
            k = min(int(hits_num[t]), MAX_TRACK_SIZE)
            h = np.sort(hits[t, :k])
            repeated += int(bool((h[1:] == h[:-1]).any()))
    bad = []
    if bad_size:
        bad.append(f"tracks above {MAX_TRACK_SIZE} hits: {bad_size}")
    if repeated:
        bad.append(f"tracks with a repeated hit: {repeated}")
    return bad


def lhcb_ids(out: dict) -> list[str]:
    offs = np.asarray(out["dev_offsets_all_velo_tracks"], dtype=np.int64)
    hit_off = np.asarray(out["dev_offsets_velo_track_hit_number"], dtype=np.int64)
    n_tracks = int(offs[-1])
    bad = []
    if (np.diff(offs) < 0).any() or (np.diff(hit_off[:n_tracks + 1]) < 0).any():
        bad.append("track or hit offsets decrease")
        return bad
    TH = int(hit_off[n_tracks])
    ids = parity._u8(out["dev_velo_track_hits"])[:4 * TH].view(np.uint32)
    if (ids == 0).any():
        bad.append(f"zero LHCb ids: {int((ids == 0).sum())}")
    n_type = int(((ids >> 28) != VELO_TYPE).sum())
    if n_type:
        bad.append(f"LHCb ids without the VELO preamble: {n_type}")
    return bad


def check(out: dict, n_events: int) -> list[str]:
    return cluster_container(out) + track_container(out, n_events) + lhcb_ids(out)
