"""The reference's contracts checked on the device (velo_check_contracts, through the C ABI).

The device checker counts the same violations as the host restatement in tests/contracts.py:
zero on the chain's own outputs, plain and learned mode, and the host checker's counts on the
oracle's outputs with mistakes planted into them on the CPU and uploaded as they are.
"""
import re

import numpy as np
import pytest

import contracts
import parity
from allen_b200 import generator
from allen_b200.chain import CONTRACTS, check_contracts, upload

pytestmark = pytest.mark.gpu

HOST_MESSAGES = {
    "cluster x or y outside": "cluster_outside",
    "module pair not sorted": "unsorted",
    "tracks above": "track_size",
    "tracks with a repeated hit": "repeated_hit",
    "zero LHCb ids": "zero_id",
    "LHCb ids without the VELO preamble": "id_type",
    "track or hit offsets decrease": "offsets",
}


def host_counts(out, n_events):
    counts = dict.fromkeys(CONTRACTS, 0)
    for message in contracts.check(out, n_events):
        key = next(v for k, v in HOST_MESSAGES.items() if message.startswith(k))
        m = re.search(r": (\d+)", message)
        counts[key] += int(m.group(1)) if m else 1
    return counts


def test_chain_outputs_hold_every_contract(chain):
    g = generator.generate(60, seed=71, pileup_min=1.0, pileup_max=15.0)
    chain.reserve_for(g.raw)
    chain.run(upload(g.raw))
    totals = chain.synchronize()
    got = check_contracts(chain.device_outputs(), totals)
    assert got == dict.fromkeys(CONTRACTS, 0), got
    assert contracts.check(chain.outputs_to_host(totals), g.raw.n_events) == []


def test_learned_mode_outputs_hold_every_contract(chain):
    from allen_b200 import seed_pruner as sp
    g = generator.generate(200, seed=72)
    saved = chain.get_config()
    chain.reserve_for(g.raw)
    try:
        sp.use_learned(chain)
        chain.run(upload(g.raw))
        totals = chain.synchronize()
        got = check_contracts(chain.device_outputs(), totals)
    finally:
        chain.set_seed_model(None)
        chain.configure(**saved)
    assert got == dict.fromkeys(CONTRACTS, 0), got


def _device_copy(out, keep):
    """Device copies of the oracle's output arrays, as Allen output name -> pointer."""
    import torch
    ptrs = {}
    for name, arr in out.items():
        raw = np.ascontiguousarray(arr).reshape(-1).view(np.uint8)
        t = torch.zeros(raw.size + 64, dtype=torch.uint8, device="cuda")
        if raw.size:
            t[:raw.size] = torch.from_numpy(raw.copy()).cuda()
        keep.append(t)
        ptrs[name] = t.data_ptr()
    return ptrs


def _totals(out, n_events):
    offs = np.asarray(out["dev_offsets_all_velo_tracks"])
    hit_off = np.asarray(out["dev_offsets_velo_track_hit_number"])
    n_tracks = int(offs[-1])
    return {"n_events": n_events,
            "host_total_number_of_velo_clusters": int(out["dev_offsets_estimated_input_size"][-1]),
            "host_number_of_reconstructed_velo_tracks": n_tracks,
            "host_accumulated_number_of_hits_in_velo_tracks": int(hit_off[n_tracks]),
            "track_container_size": parity._u8(out["dev_tracks"]).size // 54}


def test_planted_mistakes_are_counted_on_the_device(oracle, geometry):
    g = generator.generate(10, seed=4)
    n = g.raw.n_events
    out = {k: np.array(v, copy=True) for k, v in oracle.run(g.raw, geometry).items()}
    keep = []
    assert check_contracts(_device_copy(out, keep), _totals(out, n)) == dict.fromkeys(CONTRACTS, 0)

    # the mistakes of tests/test_contracts.py, planted in the oracle's outputs on the CPU
    off = out["dev_offsets_estimated_input_size"]
    num = out["dev_module_cluster_num"]
    T = int(off[-1])
    mp = int(np.argmax(num[:26]))
    s0 = int(off[mp])
    ids, xyz, phi = parity.container_fields(out["dev_sorted_velo_cluster_container"], T)
    for a in (ids, phi):
        a[[s0, s0 + 1]] = a[[s0 + 1, s0]]
    xyz[[s0, s0 + 1]] = xyz[[s0 + 1, s0]]
    xyz[s0 + 2, 1] = -150.0
    e = int(np.argmax(out["dev_number_of_velo_tracks"]))
    to = parity.track_offset(off, e)
    t = parity._u8(out["dev_tracks"]).reshape(-1, 54)
    hits = t[to, :52].view(np.uint16)
    hits[1] = hits[0]
    t[to + 1, 52] = 27
    lhcb = parity._u8(out["dev_velo_track_hits"]).view(np.uint32)
    lhcb[0] = 0
    lhcb[1] = (0x3 << 28) | (lhcb[1] & 0x0FFFFFFF)

    expected = host_counts(out, n)
    assert all(expected[k] > 0 for k in ("cluster_outside", "unsorted", "track_size", "repeated_hit", "zero_id",
                                         "id_type")), expected
    got = check_contracts(_device_copy(out, keep), _totals(out, n))
    assert got == expected, (got, expected)
