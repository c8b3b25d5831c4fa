"""The learned seed pruner on the GPU: recording, features, gradients, learned search modes.

The oracle for the network is oracle/velo_seed_oracle.py (numpy, same rounding points);
the plain search it falls back to is checked bit for bit against the reference oracle.
"""
import os
import sys

import numpy as np
import pytest

import parity
from allen_b200 import generator
from allen_b200.chain import upload

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import velo_seed_oracle as so  # noqa: E402

pytestmark = pytest.mark.gpu


def _run(chain, s):
    chain.reserve_for(s)
    chain.run(upload(s))
    totals = chain.synchronize()
    return totals, chain.outputs_to_host(totals)


@pytest.fixture
def flat_chain(chain):
    saved = chain.get_config()
    chain.configure(search_threads=256, search_lanes_per_seed=0)
    yield chain
    chain.set_seed_model(None)
    chain.record_doublets(None, None)
    chain.configure(**saved)


def _records(chain, s, every=1, capacity=1 << 20):
    from allen_b200 import seed_pruner as sp
    chain.reserve_for(s)
    rec, n, total = sp.collect(chain, [upload(s)], capacity, every)
    assert n == total
    return rec, n


def test_recording_keeps_plain_results_and_features_match_oracle(flat_chain, oracle, geometry):
    from allen_b200 import seed_pruner as sp
    g = generator.generate(12, seed=61)
    rec, n = _records(flat_chain, g.raw, every=3)
    assert n > 1000
    totals, out = _run(flat_chain, g.raw)
    assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    # the recording run itself (learned kernel, no model) is the plain search
    r = sp.records_to_host(rec, n)
    T = int(out["dev_offsets_estimated_input_size"][-1])
    ids, xyz, phi = parity.container_fields(out["dev_sorted_velo_cluster_container"], T)
    xyz = xyz.reshape(-1, 3) if xyz.ndim == 1 else xyz
    f = so.doublet_features(xyz[r["h0"], 0], xyz[r["h0"], 1], xyz[r["h0"], 2], phi[r["h0"]], xyz[r["h1"], 0],
                            xyz[r["h1"], 1], xyz[r["h1"], 2], phi[r["h1"]], r["f"][:, 9], r["f"][:, 10])
    assert np.array_equal(f.view(np.uint32), r["f"].view(np.uint32))
    # one chosen doublet at most per recorded h1, ranks 0..found-1
    assert set(np.unique(r["label"])) <= {0.0, 1.0}
    key = r["h1"].astype(np.int64)
    for h1 in np.unique(key)[:200]:
        sel = r[key == h1]
        assert sel["label"].sum() <= 1
        assert sorted(sel["f"][:, 9]) == list(range(len(sel)))


def test_gradients_match_oracle(flat_chain):
    from allen_b200 import seed_pruner as sp
    g = generator.generate(6, seed=62)
    rec, n = _records(flat_chain, g.raw)
    model = sp.initial_model(rec, n, seed=3)
    tr = sp.Trainer(model, lr=1e-3, pos_weight=2.0)
    try:
        batch = min(n, 4000)
        loss, grads = tr.gradients(rec, 0, batch)
        r = sp.records_to_host(rec, batch)
        p = sp.model_params(model)
        ref_loss, ref = so.gradients(p, np.ctypeslib.as_array(model.mean), np.ctypeslib.as_array(model.inv_std),
                                     r["f"], r["label"], pos_weight=2.0)
        assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss) + 1e-6
        # fp32 tensor-core sums vs float64 sums: within 1e-2 of the largest component
        scale = np.abs(ref).max()
        assert np.abs(grads - ref).max() <= 1e-2 * scale, (np.abs(grads - ref).max(), scale)
        z = tr.score(rec, batch).cpu().numpy()
        zr, _ = so.forward(p, np.ctypeslib.as_array(model.mean), np.ctypeslib.as_array(model.inv_std), r["f"])
        assert np.abs(z - zr).max() <= 1e-3 * (1 + np.abs(zr).max())
        # training lowers the loss
        first = tr.step(rec, 0, batch, want_loss=True)
        for _ in range(60):
            last = tr.step(rec, 0, batch, want_loss=True)
        assert last < first
    finally:
        tr.close()


def _model_keep_all(rec, n, **kw):
    from allen_b200 import seed_pruner as sp
    m = sp.initial_model(rec, n)
    m.threshold_logit = float("-inf")
    for k, v in kw.items():
        setattr(m, k, v)
    return m


@pytest.mark.parametrize("threads,ring", [(256, 1), (128, 1), (256, 0)])
def test_learned_search_keeping_every_doublet_is_the_plain_search(flat_chain, oracle, geometry, threads, ring):
    """A model that keeps every doublet: the learned kernel (each block size, ring of tracks to
    follow in global scratch or shared memory) gives the plain search's results bit for bit."""
    g = generator.generate(40, seed=63, pileup_min=1.0, pileup_max=15.0)
    flat_chain.configure(search_threads=threads, search_ring_global=ring, persistent=1)
    rec, n = _records(flat_chain, g.raw, every=5)
    flat_chain.set_seed_model(_model_keep_all(rec, n))
    totals, out = _run(flat_chain, g.raw)
    assert totals["device_flags"] == 0
    assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    st = flat_chain.seed_stats(g.raw.n_events)
    assert (st[:, 2] == 1).all() and (st[:, 0] == st[:, 1]).all()


def test_anomalous_events_fall_back_to_the_plain_search(flat_chain, oracle, geometry):
    g = generator.generate(30, seed=64)
    rec, n = _records(flat_chain, g.raw, every=5)
    # a threshold that prunes every doublet, with bounds that call that anomalous
    m = _model_keep_all(rec, n, kept_lo=0.5, kept_hi=1.0)
    m.threshold_logit = float("inf")
    flat_chain.set_seed_model(m)
    totals, out = _run(flat_chain, g.raw)
    assert totals["device_flags"] == 0
    assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    st = flat_chain.seed_stats(g.raw.n_events)
    assert (st[:, 2] == 2).all() and (st[:, 1] == 0).all()


def test_trained_network_prunes_doublets_at_equal_efficiency(flat_chain):
    """What training buys: an untrained network at the same recall calibration keeps nearly
    every doublet; after a few hundred Adam steps on plain-search labels the learned search
    scans far fewer doublets with (almost) the same tracking efficiency."""
    from allen_b200 import seed_pruner as sp
    train, n, _ = sp.collect_generated(flat_chain, 8000, 8000, 901, 4, 8000 * 1200 + 4096)
    val, n_val, _ = sp.collect_generated(flat_chain, 2000, 2000, 902, 4, 2000 * 1200 + 4096)
    model = sp.initial_model(train, n, seed=1)
    tr = sp.Trainer(model, lr=1e-3)
    try:
        thr0, before = sp.calibrate_threshold(tr, val, n_val, 0.995)
        sp.train(tr, train, n, epochs=4, batch=16384, seed=2)
        thr1, after = sp.calibrate_threshold(tr, val, n_val, 0.995)
        trained = tr.model()
    finally:
        tr.close()
    assert after["kept_fraction"] < 0.8 * before["kept_fraction"]
    trained.threshold_logit = thr1
    trained.kept_lo, trained.kept_hi = 0.0, 1.0
    g = generator.generate(300, seed=903)
    flat_chain.reserve_for(g.raw)
    flat_chain.set_seed_model(None)
    plain = sp.quality(flat_chain, g)
    flat_chain.set_seed_model(trained)
    learned = sp.quality(flat_chain, g)
    assert learned["doublets_scanned"] < 0.8 * plain["doublets_scanned"]
    assert learned["efficiency"] >= plain["efficiency"] - 0.005
    assert learned["ghost_rate"] <= plain["ghost_rate"] + 0.005
