"""Tracking efficiency, ghost and clone rates against generator truth.

Rules of the reference's TrackChecker (checker/tracking/include/TrackChecker.h:180-320,
TrackCheckerCategories.h:28-30), applied to synthetic truth:
  * a track is matched to the particle owning at least 70% of its hits (m_minweight);
  * a track matched to no particle is a ghost;
  * further tracks matched to an already matched particle are clones;
  * efficiency denominator ("01_velo"): particles with hits on at least 3 distinct
    modules (the generator's stand-in for hasVelo) and 2 < eta < 5 (no electrons are
    generated).
A hit belongs to the particle that owns the pixel of the cluster's channel id (the
centroid pixel); noise pixels belong to nobody.
"""
from __future__ import annotations

import numpy as np

MIN_WEIGHT = 0.7
ID_MASK = 0xF3FFFFFF  # clears the retina fraction bits (VPChannelID orfx/orfy, bits 27 and 26)


def hit_owner_tables(gen):
    """Per event: (sorted lhcb ids, owning particle) from the generator's truth pixels."""
    tables = []
    tp, to = gen.truth_pixels, gen.truth_offsets
    for e in range(to.size - 1):
        sl = tp[to[e]:to[e + 1]]
        order = np.argsort(sl["lhcb_id"], kind="stable")
        tables.append((sl["lhcb_id"][order], sl["particle"][order]))
    return tables


def match_tracks(tracks_ids, table):
    """tracks_ids: list of tuples of LHCb ids for one event.  Returns the matched particle
    index per track (-1 for a ghost)."""
    ids, owner = table
    out = []
    for t in tracks_ids:
        a = np.asarray(t, dtype=np.uint32) & np.uint32(ID_MASK)
        pos = np.searchsorted(ids, a)
        pos = np.minimum(pos, max(ids.size - 1, 0))
        found = (ids.size > 0) & (ids[pos] == a) if ids.size else np.zeros(a.size, bool)
        parts = owner[pos][found] if ids.size else np.zeros(0, np.uint32)
        if parts.size == 0:
            out.append(-1)
            continue
        vals, cnt = np.unique(parts, return_counts=True)
        best = int(np.argmax(cnt))
        out.append(int(vals[best]) if cnt[best] >= MIN_WEIGHT * a.size else -1)
    return out


def evaluate(gen, tracks_per_event) -> dict:
    """gen: allen_b200.generator.Generated; tracks_per_event: list (per event) of lists
    of LHCb-id tuples.  Returns counts and rates."""
    tables = hit_owner_tables(gen)
    n_tracks = n_ghost = n_clone = 0
    n_recoble = n_reco = 0
    po = gen.particle_offsets
    for e, tracks in enumerate(tracks_per_event):
        parts = gen.particles[po[e]:po[e + 1]]
        matched = match_tracks(tracks, tables[e])
        n_tracks += len(matched)
        n_ghost += sum(1 for m in matched if m < 0)
        seen = {}
        for m in matched:
            if m >= 0:
                seen[m] = seen.get(m, 0) + 1
        recoble = (parts["n_modules"] >= 3) & (parts["eta"] > 2) & (parts["eta"] < 5)
        n_recoble += int(recoble.sum())
        for p, c in seen.items():
            if p < parts.size and recoble[p]:
                n_reco += 1
                n_clone += c - 1
    return {
        "tracks": n_tracks, "ghosts": n_ghost, "ghost_rate": n_ghost / max(n_tracks, 1),
        "reconstructible": n_recoble, "reconstructed": n_reco, "efficiency": n_reco / max(n_recoble, 1),
        "clones": n_clone, "clone_rate": n_clone / max(n_reco + n_clone, 1),
    }


def tracks_from_outputs(out: dict) -> list:
    """Per event, the LHCb ids of each consolidated track, from dev_offsets_all_velo_tracks,
    dev_offsets_velo_track_hit_number and dev_velo_track_hits (ids first in its SoA)."""
    off_all = np.asarray(out["dev_offsets_all_velo_tracks"]).view(np.uint32)
    off_hn = np.asarray(out["dev_offsets_velo_track_hit_number"]).view(np.uint32)
    th = int(off_hn[-1]) if off_hn.size else 0
    hits = np.asarray(out["dev_velo_track_hits"]).view(np.uint8)
    ids = hits[:4 * th].view(np.uint32)
    return [[tuple(ids[off_hn[t]:off_hn[t + 1]]) for t in range(int(off_all[e]), int(off_all[e + 1]))]
            for e in range(off_all.size - 1)]


class DeviceTruth:
    """Generator truth on the GPU for velo_validate_tracks: per event sorted truth-pixel ids
    with their owning particle, and per particle the reconstructible flag (hits on at least
    3 modules, 2 < eta < 5)."""

    def __init__(self, gen):
        import torch
        tables = hit_owner_tables(gen)
        ids = np.concatenate([t[0] for t in tables]) if tables else np.zeros(0, np.uint32)
        owner = np.concatenate([t[1] for t in tables]) if tables else np.zeros(0, np.uint32)
        offs = np.zeros(len(tables) + 1, np.uint32)
        offs[1:] = np.cumsum([t[0].size for t in tables])
        parts = gen.particles
        recoble = ((parts["n_modules"] >= 3) & (parts["eta"] > 2) & (parts["eta"] < 5)).astype(np.uint8)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        self.n_events = len(tables)
        self.n_particles = int(parts.size)
        self.truth_offsets = dev(offs.view(np.int32))
        self.truth_ids = dev(ids.astype(np.uint32).view(np.int32))
        self.truth_owner = dev(owner.astype(np.uint32).view(np.int32))
        self.particle_offsets = dev(np.asarray(gen.particle_offsets, np.uint32).view(np.int32))
        self.reconstructible = dev(recoble)
        self.matched = torch.zeros(max(self.n_particles, 1), dtype=torch.int32, device="cuda")
        self.counts = torch.zeros(5, dtype=torch.int64, device="cuda")


def evaluate_device(chain, truth: DeviceTruth) -> dict:
    """The counts of evaluate(), computed on the GPU from the chain's last run (no track copies)."""
    import ctypes as C
    from .chain import _check, _current_stream
    p = chain.device_outputs()
    lib = chain.lib
    lib.velo_validate_tracks.restype = C.c_int
    lib.velo_validate_tracks.argtypes = [C.c_uint] + [C.c_void_p] * 8 + [C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p]
    _check(lib, lib.velo_validate_tracks(
        truth.n_events, p["dev_offsets_all_velo_tracks"], p["dev_offsets_velo_track_hit_number"],
        p["dev_velo_track_hits"], truth.truth_offsets.data_ptr(), truth.truth_ids.data_ptr(),
        truth.truth_owner.data_ptr(), truth.particle_offsets.data_ptr(), truth.reconstructible.data_ptr(),
        truth.n_particles, truth.matched.data_ptr(), truth.counts.data_ptr(), _current_stream()))
    t, g, rb, r, c = (int(v) for v in truth.counts.cpu().numpy())
    return {"tracks": t, "ghosts": g, "ghost_rate": g / max(t, 1), "reconstructible": rb, "reconstructed": r,
            "efficiency": r / max(rb, 1), "clones": c, "clone_rate": c / max(r + c, 1)}
