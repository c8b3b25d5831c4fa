"""Parity rules between the chain's outputs and the oracle's (test infrastructure).

Everything is compared bit for bit.  Only the bytes the reference itself leaves
undefined are excluded:
  * sorted cluster container: the slots the estimate reserves beyond the clusters
    found (the reference fills them with a copy of container slot 0);
  * dev_tracks: the hit slots of a track beyond its hitsNum, and entries past the
    event's track count;
  * three-hit containers: entries past the event's count;
  * consolidated hits: the phi column, which the reference never writes.
"""
from __future__ import annotations

import numpy as np

N_MP = 26
EXACT = [
    "dev_number_of_candidates", "dev_estimated_input_size", "dev_module_candidate_num",
    "dev_offsets_estimated_input_size", "dev_module_cluster_num", "dev_hit_used", "dev_atomics_velo",
    "dev_number_of_velo_tracks", "dev_offsets_velo_tracks", "dev_number_of_three_hit_tracks_output",
    "dev_offsets_number_of_three_hit_tracks_filtered", "dev_offsets_all_velo_tracks",
    "dev_velo_track_hit_number", "dev_offsets_velo_track_hit_number", "dev_accepted_velo_tracks",
]


def _u8(a):
    return np.ascontiguousarray(a).view(np.uint8)


def sorted_container_mask(offsets_est, cluster_num, T):
    """Boolean mask over the T cluster slots that hold a cluster."""
    mask = np.zeros(T, dtype=bool)
    starts = offsets_est[:-1].astype(np.int64)
    nums = cluster_num.astype(np.int64)
    for s, n in zip(starts, nums):
        mask[s:s + n] = True
    return mask


def container_fields(buf, T):
    b = _u8(buf)
    ids = b[:4 * T].view(np.uint32)
    xyz = b[4 * T:16 * T].view(np.float32).reshape(T, 3)
    phi = b[16 * T:18 * T].view(np.int16)
    return ids, xyz, phi


def track_track_fields(tracks_bytes, to, n):
    t = _u8(tracks_bytes).reshape(-1, 54)[to:to + n]
    hits = t[:, :52].copy().view(np.uint16).reshape(n, 26)
    return hits, t[:, 52]


def track_offset(offsets_est, e):
    return int(np.float32(offsets_est[e * N_MP]) * np.float32(0.34))


# decoding buffers of the super-pixel front end that the retina-cluster front end does not have
SP_ONLY = {"dev_number_of_candidates", "dev_estimated_input_size", "dev_module_candidate_num"}


def compare(gpu: dict, ref: dict, n_events: int) -> list[str]:
    bad = []
    for k in EXACT:
        a, b = gpu.get(k), ref.get(k)
        if k in SP_ONLY and b is None:
            continue  # retina-cluster decoding
        if a is None or b is None:
            bad.append(f"{k}: missing")
            continue
        if _u8(a).shape != _u8(b).shape or not np.array_equal(_u8(a), _u8(b)):
            bad.append(f"{k}: differs ({_u8(a).size} vs {_u8(b).size} bytes)")
    off = ref["dev_offsets_estimated_input_size"]
    T = int(off[-1])
    mask = sorted_container_mask(off, ref["dev_module_cluster_num"], T)
    for name, (ga, ra) in zip(("id", "xyz", "phi"),
                              zip(container_fields(gpu["dev_sorted_velo_cluster_container"], T),
                                  container_fields(ref["dev_sorted_velo_cluster_container"], T))):
        if not np.array_equal(_u8(ga[mask]), _u8(ra[mask])):
            bad.append(f"sorted container {name}: {int((ga[mask] != ra[mask]).any(axis=-1).sum() if ga.ndim > 1 else (ga[mask] != ra[mask]).sum())} slots differ")
    n_tr = ref["dev_number_of_velo_tracks"]
    at = ref["dev_atomics_velo"].reshape(-1, 3)
    n3 = ref["dev_number_of_three_hit_tracks_output"]
    for e in range(n_events):
        to = track_offset(off, e)
        gh, gn = track_track_fields(gpu["dev_tracks"], to, int(n_tr[e]))
        rh, rn = track_track_fields(ref["dev_tracks"], to, int(n_tr[e]))
        if not np.array_equal(gn, rn):
            bad.append(f"event {e}: track hit counts differ")
            continue
        for i in range(int(n_tr[e])):
            if not np.array_equal(gh[i, :gn[i]], rh[i, :rn[i]]):
                bad.append(f"event {e}: track {i} hits differ")
                break
        for name, cnt in (("dev_three_hit_tracks", int(at[e, 0])), ("dev_three_hit_tracks_output", int(n3[e]))):
            g3 = np.asarray(gpu[name]).reshape(-1, 3)[to:to + cnt]
            r3 = np.asarray(ref[name]).reshape(-1, 3)[to:to + cnt]
            if not np.array_equal(g3, r3):
                bad.append(f"event {e}: {name} differ")
        if len(bad) > 20:
            break
    TH = int(ref["dev_offsets_velo_track_hit_number"][-1]) if ref["dev_offsets_velo_track_hit_number"].size else 0
    g = _u8(gpu["dev_velo_track_hits"])[:16 * TH]
    r = _u8(ref["dev_velo_track_hits"])[:16 * TH]
    if not np.array_equal(g, r):
        bad.append("dev_velo_track_hits (id, xyz) differ")
    return bad


def tracks_as_id_lists(out: dict) -> list[list[tuple]]:
    """Per event, the consolidated tracks as tuples of LHCb ids (order kept)."""
    off_all = out["dev_offsets_all_velo_tracks"]
    off_hn = out["dev_offsets_velo_track_hit_number"]
    TH = int(off_hn[-1]) if off_hn.size else 0
    ids = _u8(out["dev_velo_track_hits"])[:4 * TH].view(np.uint32)
    events = []
    for e in range(off_all.size - 1):
        evt = []
        for t in range(int(off_all[e]), int(off_all[e + 1])):
            evt.append(tuple(ids[off_hn[t]:off_hn[t + 1]].tolist()))
        events.append(evt)
    return events


def same_clusters_and_tracks(a: dict, b: dict) -> bool:
    """Two runs over the same events decoded to the same sorted clusters (occupied slots)
    and the same consolidated tracks; buffers indexed by candidate are not compared."""
    for k in ("dev_offsets_estimated_input_size", "dev_module_cluster_num", "dev_offsets_all_velo_tracks",
              "dev_offsets_velo_track_hit_number", "dev_velo_track_hits"):
        if not np.array_equal(_u8(a[k]), _u8(b[k])):
            return False
    off = a["dev_offsets_estimated_input_size"]
    T = int(off[-1])
    mask = sorted_container_mask(off, a["dev_module_cluster_num"], T)
    return all(np.array_equal(_u8(x[mask]), _u8(y[mask]))
               for x, y in zip(container_fields(a["dev_sorted_velo_cluster_container"], T),
                               container_fields(b["dev_sorted_velo_cluster_container"], T)))


def kalman_written_words(reco: int) -> np.ndarray:
    """Word indices of Velo::Consolidated::States that velo_kalman_filter writes: x y z tx ty
    of each track (qop not), and c00 c20 c22 c11 c31 c33 (chi2, ndof not)."""
    st = np.arange(6 * reco).reshape(reco, 6)[:, :5].ravel()
    cov = (6 * reco + np.arange(8 * reco).reshape(reco, 8)[:, :6]).ravel()
    return np.concatenate([st, cov])
