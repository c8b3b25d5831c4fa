"""The learned seed gate on the GPU: recording, features, gradients, the gated search modes.

The oracle for the network and its features is oracle/velo_seed_oracle.py (numpy, same
rounding points); the plain search the gate falls back to is checked bit for bit against the
reference oracle; learned-mode tracks (no bit-exact oracle) are checked against the
reference's contracts and, for quality, against generator truth within 0.2 % of the plain
search's efficiency and ghost rate.
"""
import os
import sys

import numpy as np
import pytest

import contracts
import parity
from allen_b200 import generator
from allen_b200.chain import upload

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import velo_seed_oracle as so  # noqa: E402

pytestmark = pytest.mark.gpu
TOLERANCE = 0.002  # largest efficiency loss and ghost-rate rise allowed to the learned mode


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
    chain.record_seeds(None, None)
    chain.configure(**saved)


def _records(chain, s, every=1, capacity=1 << 20):
    from allen_b200 import seed_pruner as sp
    chain.reserve_for(s)
    rec, n, total = sp.collect(chain, [upload(s)], capacity, every)
    assert n == total
    return rec, n


def _event_hits(out, e):
    off = out["dev_offsets_estimated_input_size"]
    num = out["dev_module_cluster_num"]
    T = int(off[-1])
    ids, xyz, phi = parity.container_fields(out["dev_sorted_velo_cluster_container"], T)
    start = off[26 * e:26 * e + 27].astype(np.int64) - int(off[26 * e])
    return xyz[int(off[26 * e]):], phi[int(off[26 * e]):], start, num[26 * e:26 * e + 26], int(off[26 * e])


def test_recording_keeps_plain_results_and_features_match_oracle(flat_chain, oracle, geometry):
    from allen_b200 import seed_pruner as sp
    g = generator.generate(12, seed=61)
    rec, n = _records(flat_chain, g.raw, every=3)
    assert n > 500
    totals, out = _run(flat_chain, g.raw)
    assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    r = sp.records_to_host(rec, n)
    assert (r["h0"] == 0xFFFFFFFF).all() and set(np.unique(r["label"])) <= {0.0, 1.0}
    assert 0.1 < r["label"].mean() < 0.6  # about one seed candidate in four makes a seed
    zs = so.module_zs(geometry)
    tol = so.phi_tolerance_i16()
    got = {}
    for k in range(0, n, max(1, n // 400)):  # a sample of the records, every event
        e = int(r["event"][k])
        xyz, phi, start, num, base = _event_hits(out, e)
        h1 = int(r["h1"][k]) - base
        m = int(np.searchsorted(start[1:], h1, side="right"))
        assert 1 <= m <= 24 and h1 - start[m] < num[m]
        f = so.seed_features(xyz, phi, start, num, zs, m, h1, tol)
        got[k] = f
        assert np.array_equal(f.view(np.uint32), r["f"][k].view(np.uint32)), (k, f, r["f"][k])


def test_gradients_match_oracle(flat_chain):
    from allen_b200 import seed_pruner as sp
    g = generator.generate(30, seed=62)
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


def _model(rec, n, **kw):
    from allen_b200 import seed_pruner as sp
    m = sp.initial_model(rec, n)
    m.threshold_logit = float("-inf")
    for k, v in kw.items():
        setattr(m, k, v)
    return m


def test_gate_decisions_match_oracle(flat_chain, geometry):
    """The gate kernel's keep decisions equal the oracle network's on the oracle's features
    (decisions within 1e-3 of the threshold are not compared: fp32 tensor-core sums)."""
    from allen_b200 import seed_pruner as sp
    g = generator.generate(10, seed=66)
    rec, n = _records(flat_chain, g.raw, every=1)
    m = _model(rec, n)
    r = sp.records_to_host(rec, n)
    p = sp.model_params(m)
    mean, inv_std = np.ctypeslib.as_array(m.mean), np.ctypeslib.as_array(m.inv_std)
    z, _ = so.forward(p, mean, inv_std, r["f"])
    m.threshold_logit = float(np.median(z))
    m.kept_lo, m.kept_hi = 0.0, 1.0
    flat_chain.set_seed_model(m)
    totals, out = _run(flat_chain, g.raw)
    gate = flat_chain._fetch(flat_chain.device_outputs()["dev_seed_gate"],
                             totals["host_total_number_of_velo_clusters"], np.uint8)
    clear = np.abs(z - m.threshold_logit) > 1e-3
    assert clear.mean() > 0.95
    assert np.array_equal(gate[r["h1"][clear]], (z[clear] > m.threshold_logit).astype(np.uint8))
    st = flat_chain.gate_stats(g.raw.n_events)
    assert (st[:, 1] <= st[:, 0]).all() and 0.2 < st[:, 1].sum() / st[:, 0].sum() < 0.8


@pytest.mark.parametrize("threads,ring", [(256, 1), (128, 1), (256, 0)])
def test_gate_keeping_every_candidate_is_the_plain_search(flat_chain, oracle, geometry, threads, ring):
    """A gate that keeps every candidate: the gated kernel (each block size, ring of tracks to
    follow in global scratch or shared memory) gives the plain search's results bit for bit."""
    g = generator.generate(40, seed=63, pileup_min=1.0, pileup_max=15.0)
    flat_chain.configure(search_threads=threads, search_ring_global=ring, persistent=1)
    rec, n = _records(flat_chain, g.raw, every=5)
    flat_chain.set_seed_model(_model(rec, n))
    totals, out = _run(flat_chain, g.raw)
    assert totals["device_flags"] == 0
    assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    st = flat_chain.seed_stats(g.raw.n_events)
    assert (st[:, 2] == 1).all() and (st[:, 0] == st[:, 1]).all()


def test_anomalous_events_fall_back_to_the_plain_search(flat_chain, oracle, geometry):
    g = generator.generate(30, seed=64)
    rec, n = _records(flat_chain, g.raw, every=5)
    # a threshold that gates every candidate off, with bounds that call that anomalous
    m = _model(rec, n, kept_lo=0.5, kept_hi=1.0)
    m.threshold_logit = float("inf")
    flat_chain.set_seed_model(m)
    totals, out = _run(flat_chain, g.raw)
    assert totals["device_flags"] == 0
    assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    st = flat_chain.seed_stats(g.raw.n_events)
    assert (st[:, 2] == 2).all() and (st[:, 0] == st[:, 1]).all()


def _trained(flat_chain, recall=0.99):
    from allen_b200 import seed_pruner as sp
    train, n, _ = sp.collect_generated(flat_chain, 8000, 8000, 901, 2, 8000 * 400 + 4096)
    val, n_val, _ = sp.collect_generated(flat_chain, 2000, 2000, 902, 2, 2000 * 400 + 4096)
    model = sp.initial_model(train, n, seed=1)
    tr = sp.Trainer(model, lr=1e-3)
    try:
        thr0, before = sp.calibrate_threshold(tr, val, n_val, recall)
        sp.train(tr, train, n, epochs=4, batch=16384, seed=2)
        thr1, after = sp.calibrate_threshold(tr, val, n_val, recall)
        trained = tr.model()
    finally:
        tr.close()
    trained.threshold_logit = thr1
    trained.kept_lo, trained.kept_hi = 0.0, 1.0
    return trained, before, after


def test_trained_gate_prunes_candidates_at_equal_efficiency(flat_chain):
    """What training buys: an untrained network at the same recall calibration keeps most
    candidates; after a few hundred Adam steps on plain-search labels the learned search
    searches far fewer candidates at the plain search's efficiency and ghost rate (within
    0.2 %), and its tracks keep every contract of the reference."""
    from allen_b200 import seed_pruner as sp
    trained, before, after = _trained(flat_chain)
    assert after["kept_fraction"] < 0.7 * before["kept_fraction"]
    for cfg in (dict(), dict(mean_pileup=15.0, noise_rate=1e-4, hit_efficiency=0.95)):
        g = generator.generate(400, seed=903, **cfg)
        flat_chain.reserve_for(g.raw)
        flat_chain.set_seed_model(None)
        plain = sp.quality(flat_chain, g)
        flat_chain.set_seed_model(trained)
        learned = sp.quality(flat_chain, g)
        totals = flat_chain.synchronize()
        out = flat_chain.outputs_to_host(totals)
        assert contracts.check(out, g.raw.n_events) == []
        assert learned["candidates_searched"] < 0.6 * plain["candidates_searched"]
        assert learned["efficiency"] >= plain["efficiency"] - TOLERANCE, (learned, plain)
        assert learned["ghost_rate"] <= plain["ghost_rate"] + TOLERANCE, (learned, plain)
