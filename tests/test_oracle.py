"""The oracle (plain-C restatement) pinned against the reference's own outputs."""
import ctypes as C

import numpy as np
import pytest

import cpu_checkers
import golden_io
import parity
from allen_b200 import generator


@pytest.mark.parametrize("name", golden_io.FIXTURES)
def test_oracle_matches_committed_reference_outputs(oracle, geometry, name):
    s, ref = golden_io.load(name)
    out = oracle.run(s, geometry)
    for k, v in ref.items():
        assert np.array_equal(parity._u8(out[k]), parity._u8(v)), k


def test_prefix_sum_known_answer(oracle, geometry):
    """TestPrefixSum.cu:9-32: iota 1..1000 against std::partial_sum, here through the
    oracle's candidate offsets (a prefix sum over 2 x super pixels per event)."""
    s, ref = golden_io.load("synthetic_seed7_20ev")
    out = oracle.run(s, geometry)
    n = out["dev_number_of_candidates"]
    assert np.array_equal(out["dev_candidates_offsets"], np.concatenate([[0], np.cumsum(n)]).astype(np.uint32))
    iota = np.arange(1, 1001, dtype=np.uint64)
    assert int(np.cumsum(iota)[-1]) == 500500


@pytest.mark.skipif(not cpu_checkers.available("ref"), reason="reference CPU build not present")
@pytest.mark.parametrize("cfg", [dict(), dict(bank_version=4), dict(mean_pileup=15.0, noise_rate=1e-4)])
def test_oracle_matches_reference_build(oracle, geometry, cfg):
    ref = cpu_checkers.load("ref")
    g = generator.generate(30, seed=3, **cfg)
    a, b = oracle.run(g.raw, geometry), ref.run(g.raw, geometry)
    assert sorted(a) == sorted(b)
    for k in a:
        assert np.array_equal(parity._u8(a[k]), parity._u8(b[k])), k


def test_oracle_planted_mistake_is_caught(oracle, geometry):
    """A wrong property changes the tracks: the comparison must see it."""
    s, ref = golden_io.load("synthetic_seed7_20ev")
    out = oracle.run(s, geometry, max_scatter=0.05)
    assert not np.array_equal(out["dev_offsets_all_velo_tracks"], ref["dev_offsets_all_velo_tracks"])


def test_empty_banks_and_single_event(oracle, geometry):
    from allen_b200 import rawbanks
    # one event with all 208 banks empty, one with a single isolated super pixel
    empty = [(63, sid, np.array([0], np.uint32).tobytes()) for sid in range(208)]
    one = list(empty)
    word = (1 << 31) | (100 << 14) | (10 << 8) | 0x01
    one[17] = (63, 17, np.array([1, word], np.uint32).tobytes())
    s = rawbanks.build_slice([empty, one], bank_version=2)
    out = oracle.run(s, geometry)
    assert out["dev_module_cluster_num"].sum() == 1
    assert out["dev_offsets_all_velo_tracks"][-1] == 0


@pytest.mark.parametrize("version", [2, 4])
def test_sp_order_invariance(oracle, geometry, version):
    """The reference's decoding does not depend on the order of SPs inside a bank: the
    generator's column order and its shuffled readout order give the same clusters and tracks."""
    runs = [oracle.run(generator.generate(8, seed=12, bank_version=version, sp_order=o).raw, geometry)
            for o in (0, 1)]
    assert parity.same_clusters_and_tracks(runs[0], runs[1])


@pytest.mark.parametrize("beamline", [(0.0, 0.0), (0.35, -0.2)])
def test_kalman_filter_matches_reference_build(oracle, geometry, beamline):
    """velo_kalman_filter of the C restatement against the reference's own kernel compiled as
    CPU C++: dev_is_backward and the written fields of both state containers, bit for bit."""
    if not cpu_checkers.available("ref"):
        pytest.skip("oracle/_ref not built")
    ref = cpu_checkers.load("ref")
    g = generator.generate(25, seed=17, pileup_min=1.0, pileup_max=15.0)
    a = oracle.run(g.raw, geometry, beamline=beamline)
    b = ref.run(g.raw, geometry, beamline=beamline)
    reco = int(a["dev_offsets_all_velo_tracks"][-1])
    assert np.array_equal(a["dev_is_backward"], b["dev_is_backward"])
    written = parity.kalman_written_words(reco)
    for k in ("dev_velo_kalman_beamline_states", "dev_velo_kalman_endvelo_states"):
        assert np.array_equal(a[k].view(np.uint32)[written], b[k].view(np.uint32)[written]), k


@pytest.mark.parametrize("cfg", [dict(), dict(bank_version=4), dict(raw_format=1, bank_version=3)])
def test_mep_layout_in_reference_build(geometry, cfg):
    """The reference's own mep_layout kernels on our MEP transpose give its Allen-layout results:
    pins rawbanks.to_mep (the layout the GPU kernels read) against MEPTools.h."""
    if not cpu_checkers.available("ref"):
        pytest.skip("oracle/_ref not built")
    from allen_b200 import rawbanks
    ref = cpu_checkers.load("ref")
    g = generator.generate(10, seed=4, **cfg)
    assert parity.compare(ref.run(rawbanks.to_mep(g.raw), geometry), ref.run(g.raw, geometry), g.raw.n_events) == []
