"""The contract checker (tests/contracts.py) on the oracle's outputs: they hold on real and
generated events, and each planted mistake (in a copy of the oracle's outputs, on the CPU)
is caught by the contract the reference wrote for it."""
import numpy as np
import pytest

import contracts
import golden_io
import parity
from allen_b200 import generator


@pytest.mark.parametrize("name", ["minbias_vp_10ev", "synthetic_seed7_20ev", "minbias_retina_10ev"])
def test_contracts_hold_on_fixtures(oracle, geometry, name):
    s, _ = golden_io.load(name)
    assert contracts.check(oracle.run(s, geometry), s.n_events) == []


def test_contracts_hold_on_stress_events(oracle, geometry):
    g = generator.generate(20, seed=8, mean_pileup=15.0, noise_rate=1e-4, hit_efficiency=0.95)
    assert contracts.check(oracle.run(g.raw, geometry), g.raw.n_events) == []


def _copy(out):
    return {k: np.array(v, copy=True) for k, v in out.items()}


def test_planted_mistakes_are_caught(oracle, geometry):
    g = generator.generate(10, seed=4)
    out = oracle.run(g.raw, geometry)
    n = g.raw.n_events
    assert contracts.check(out, n) == []
    off = out["dev_offsets_estimated_input_size"]
    num = out["dev_module_cluster_num"]
    T = int(off[-1])

    # two neighbours of a module pair swapped: not sorted
    bad = _copy(out)
    mp = int(np.argmax(num[:26]))
    s0 = int(off[mp])
    ids, xyz, phi = parity.container_fields(bad["dev_sorted_velo_cluster_container"], T)
    for a in (ids, phi):
        a[[s0, s0 + 1]] = a[[s0 + 1, s0]]
    xyz[[s0, s0 + 1]] = xyz[[s0 + 1, s0]]
    assert any("sorted" in b for b in contracts.cluster_container(bad))

    # a cluster far outside the detector
    bad = _copy(out)
    _, xyz, _ = parity.container_fields(bad["dev_sorted_velo_cluster_container"], T)
    xyz[s0, 0] = 150.0
    assert any("outside" in b for b in contracts.cluster_container(bad))

    # a track with one hit twice, and one above 26 hits
    bad = _copy(out)
    e = int(np.argmax(out["dev_number_of_velo_tracks"]))
    to = parity.track_offset(off, e)
    t = parity._u8(bad["dev_tracks"]).reshape(-1, 54)
    hits = t[to, :52].view(np.uint16)
    hits[1] = hits[0]
    t[to + 1, 52] = 27
    found = contracts.track_container(bad, n)
    assert any("repeated" in b for b in found) and any("above 26" in b for b in found)

    # consolidated ids: one zero, one of another detector
    bad = _copy(out)
    ids = parity._u8(bad["dev_velo_track_hits"]).view(np.uint32)
    ids[0] = 0
    ids[1] = (0x3 << 28) | (ids[1] & 0x0FFFFFFF)
    found = contracts.lhcb_ids(bad)
    assert any("zero" in b for b in found) and any("preamble" in b for b in found)
