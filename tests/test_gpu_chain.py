"""Parity of the B200 chain (through the C ABI) with the oracle, bit for bit."""
import numpy as np
import pytest

import golden_io
import parity
from allen_b200 import generator
from allen_b200.chain import VeloError, upload

pytestmark = pytest.mark.gpu


def run_chain(chain, s, use_graph=False):
    chain.reserve_for(s)
    d = upload(s)
    chain.run(d, use_graph=use_graph)
    totals = chain.synchronize()
    return totals, chain.outputs_to_host(totals)


@pytest.mark.parametrize("name", golden_io.FIXTURES)
def test_golden_fixture(chain, oracle, geometry, name):
    s, ref = golden_io.load(name)
    totals, out = run_chain(chain, s)
    assert totals["device_flags"] == 0
    # against the reference's own outputs committed with the fixture
    for k in parity.EXACT:
        if k in ref:
            assert np.array_equal(parity._u8(out[k]), parity._u8(ref[k])), k
    # against the oracle, every buffer
    assert parity.compare(out, oracle.run(s, geometry), s.n_events) == []


CONFIGS = {
    "nu7.6": dict(),
    "v3": dict(bank_version=3),
    "v4": dict(bank_version=4),
    "uneven": dict(pileup_min=1.0, pileup_max=15.0),
    "nu15_noise": dict(mean_pileup=15.0, noise_rate=1e-4, hit_efficiency=0.95),
}


@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_synthetic(chain, oracle, geometry, cfg):
    g = generator.generate(150, seed=100 + len(cfg), **CONFIGS[cfg])
    totals, out = run_chain(chain, g.raw)
    assert totals["device_flags"] == 0
    assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []


def test_graph_replay_and_host_path(chain, oracle, geometry):
    g = generator.generate(64, seed=5)
    t1, a = run_chain(chain, g.raw, use_graph=True)
    d = upload(g.raw)
    chain.run(d, use_graph=True)
    chain.run(d, use_graph=True)  # replay of the cached graph
    t2 = chain.synchronize()
    b = chain.outputs_to_host(t2)
    assert t1 == t2
    assert parity.compare(a, b, g.raw.n_events) == []
    t3, host_out, up, down = chain.run_host(g.raw)
    assert up >= g.raw.raw.nbytes and down > 0
    ref = oracle.run(g.raw, geometry)
    assert np.array_equal(host_out["dev_offsets_all_velo_tracks"], ref["dev_offsets_all_velo_tracks"])
    TH = int(ref["dev_offsets_velo_track_hit_number"][-1])
    assert np.array_equal(host_out["dev_velo_track_hits"][:16 * TH], parity._u8(ref["dev_velo_track_hits"])[:16 * TH])


def test_event_slice_offset(chain, oracle, geometry):
    """A slice that starts inside the arrays (RuntimeOptions::event_interval)."""
    g = generator.generate(40, seed=9)
    d = upload(g.raw).sub(10, 25)
    chain.reserve_for(g.raw)
    chain.run(d)
    totals = chain.synchronize()
    out = chain.outputs_to_host(totals)
    ref = oracle.run(g.raw, geometry, event_start=10, n_events=25)
    assert parity.compare(out, ref, 25) == []


def test_host_pipeline_matches_oracle(oracle, geometry):
    """End-to-end path (page-locked host slices, three chains and two copy streams overlapping,
    each chain taking several slices) against the oracle."""
    import torch
    from allen_b200.chain import HostPipeline
    from allen_b200.rawbanks import super_pixels_per_event
    import bench
    slices = [generator.generate(30, seed=40 + i).raw for i in range(8)]
    pinned = [bench.pin(s) for s in slices]
    pipe = HostPipeline()
    pipe.reserve(30, max(int(super_pixels_per_event(s).sum()) for s in slices) + 64,
                 max(s.raw.nbytes for s in slices), max(s.sizes.size for s in slices),
                 max(s.types.size for s in slices))
    totals, outs = pipe.run(pinned, keep_outputs=8)
    assert len(outs) == 8 and [t["n_events"] for t in totals] == [30] * 8
    pipe.close()
    for s, out in zip(slices, outs):
        ref = oracle.run(s, geometry)
        assert np.array_equal(out["dev_offsets_all_velo_tracks"], ref["dev_offsets_all_velo_tracks"])
        assert np.array_equal(out["dev_offsets_velo_track_hit_number"], ref["dev_offsets_velo_track_hit_number"])
        TH = int(ref["dev_offsets_velo_track_hit_number"][-1])
        assert np.array_equal(out["dev_velo_track_hits_id_xyz"], parity._u8(ref["dev_velo_track_hits"])[:16 * TH])


@pytest.mark.parametrize("threads,lanes", [(128, 1), (256, 2), (256, 4), (512, 4), (128, 0), (256, 0), (512, 0)])
def test_search_variants_identical(chain, oracle, geometry, threads, lanes):
    """Every compiled search configuration gives the same bit-exact result (one CTA per event,
    rings in shared memory; the tuned configuration's persistent launches with global rings are
    what every other test runs)."""
    g = generator.generate(40, seed=77, pileup_min=1.0, pileup_max=15.0)
    saved = chain.get_config()
    try:
        chain.configure(search_threads=threads, search_lanes_per_seed=lanes, search_hit_capacity=2048,
                        cluster_stage_capacity=2048, search_ring_global=0, persistent=0)
        totals, out = run_chain(chain, g.raw)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    finally:
        chain.configure(**saved)


@pytest.mark.parametrize("blob", [65536, 16384, 4096])
def test_decode_staging_paths(chain, oracle, geometry, blob):
    """Raw-event staging sizes that select each decoding path: the event and its sorted
    bank copies in shared memory (64 KiB), the event alone with the full neighbour scans
    (16 KiB, events of about 13 KB), and the event read from global memory (4 KiB)."""
    g = generator.generate(40, seed=31, pileup_min=1.0, pileup_max=15.0)
    saved = chain.get_config()
    try:
        chain.configure(estimate_blob_bytes=blob, cluster_blob_bytes=min(blob, 32768),
                        cluster_stage_capacity=1024 if blob < 65536 else 2560)
        totals, out = run_chain(chain, g.raw)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    finally:
        chain.configure(**saved)


@pytest.mark.parametrize("version", [2, 4])
def test_sp_order_does_not_change_results(chain, oracle, geometry, version):
    """Banks in column order and in shuffled readout order decode to the same sorted
    clusters and tracks (candidate indices differ, so those buffers are not compared)."""
    outs = []
    for order in (0, 1):
        g = generator.generate(30, seed=12, bank_version=version, sp_order=order)
        totals, out = run_chain(chain, g.raw)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
        outs.append(out)
    assert parity.same_clusters_and_tracks(outs[0], outs[1])


@pytest.mark.parametrize("claim", [1, 3])
def test_persistent_work_queue_identical(chain, oracle, geometry, claim):
    """Resident CTAs claiming events (largest first) from a work queue give the results of
    one CTA per event, bit for bit, on an uneven slice (nu uniform in 1..15)."""
    g = generator.generate(300, seed=78, pileup_min=1.0, pileup_max=15.0)
    saved = chain.get_config()
    try:
        chain.configure(persistent=1, events_per_claim=claim)
        totals, out = run_chain(chain, g.raw, use_graph=True)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    finally:
        chain.configure(**saved)


@pytest.mark.parametrize("threads,blob", [(128, 0), (128, 16384), (256, 0)])
def test_cluster_block_size_and_global_sorted_copies(chain, oracle, geometry, threads, blob):
    """The clustering kernel with 128 or 256 threads, its sorted bank copies in shared memory
    or (blob 0: nothing staged) in the global scratch: the same results, bit for bit."""
    g = generator.generate(200, seed=83, pileup_min=1.0, pileup_max=15.0)
    saved = chain.get_config()
    try:
        with pytest.raises(VeloError):
            chain.configure(cluster_threads=64)
        chain.configure(cluster_threads=threads, cluster_blob_bytes=blob)
        totals, out = run_chain(chain, g.raw, use_graph=True)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    finally:
        chain.configure(**saved)


@pytest.mark.parametrize("threads", [64, 96, 128, 256])
def test_search_ring_in_global_scratch(chain, oracle, geometry, threads):
    """The search's ring of tracks to follow in global scratch (one ring per resident CTA)
    instead of shared memory: the same results, bit for bit, on an uneven slice; the setting
    needs persistent launches."""
    g = generator.generate(300, seed=79, pileup_min=1.0, pileup_max=15.0)
    saved = chain.get_config()
    try:
        with pytest.raises(VeloError):
            chain.configure(search_threads=threads, search_lanes_per_seed=0, persistent=0, search_ring_global=1)
        chain.configure(search_threads=threads, search_lanes_per_seed=0, persistent=1, search_ring_global=1)
        totals, out = run_chain(chain, g.raw, use_graph=True)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    finally:
        chain.configure(**saved)


@pytest.mark.parametrize("version", [2, 3, 4])
def test_retina_front_end(chain, oracle, geometry, version):
    """Retina-cluster banks: decoding, search and consolidation against the oracle."""
    g = generator.generate(120, seed=90 + version, raw_format=1, bank_version=version, pileup_min=1.0,
                           pileup_max=15.0)
    assert g.raw.retina
    totals, out = run_chain(chain, g.raw, use_graph=True)
    assert totals["device_flags"] == 0
    ref = oracle.run(g.raw, geometry)
    assert parity.compare(out, ref, g.raw.n_events) == []
    for k in ("dev_each_sensor_pair_size", "dev_offsets_each_sensor_pair_size"):
        assert np.array_equal(out[k], ref[k]), k
    # back to super pixels on the same chain
    s = generator.generate(30, seed=3).raw
    totals, out = run_chain(chain, s)
    assert parity.compare(out, oracle.run(s, geometry), s.n_events) == []


@pytest.mark.parametrize("cfg", [dict(), dict(bank_version=4), dict(raw_format=1, bank_version=3)])
def test_mep_layout(chain, oracle, geometry, cfg):
    """The same events in the MEP layout (banks of one source together, MEPTools.h) give the
    Allen-layout results bit for bit, for super-pixel and retina banks."""
    from allen_b200 import rawbanks
    g = generator.generate(80, seed=66, pileup_min=1.0, pileup_max=15.0, **cfg)
    m = rawbanks.to_mep(g.raw)
    assert m.mep and m.n_events == g.raw.n_events
    totals, out = run_chain(chain, m, use_graph=True)
    assert totals["device_flags"] == 0
    assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []


def test_full_size_slice(chain, oracle, geometry):
    """A slice of the benchmark's size (16000 events at nu = 7.6) with the tuned configuration:
    bit for bit the oracle's, and the same as with one CTA per event, shared-memory rings and
    staging (the other code paths of every kernel)."""
    g = generator.generate(16000, seed=2024)
    saved = chain.get_config()
    try:
        totals, tuned = run_chain(chain, g.raw, use_graph=True)
        assert totals["device_flags"] == 0
        assert parity.compare(tuned, oracle.run(g.raw, geometry), g.raw.n_events) == []
        chain.configure(search_threads=256, search_lanes_per_seed=0, search_ring_global=0, persistent=0,
                        search_hit_capacity=3072, cluster_stage_capacity=2560, cluster_blob_bytes=32768,
                        estimate_blob_bytes=32768, cluster_threads=256)
        totals2, other = run_chain(chain, g.raw, use_graph=True)
        assert totals2 == totals
        assert parity.compare(other, tuned, g.raw.n_events) == []
    finally:
        chain.configure(**saved)
