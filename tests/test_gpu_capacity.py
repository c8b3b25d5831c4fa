"""Capacity limits and the less-travelled code paths of the chain, through the C ABI.

Every input here is well formed: the slices are generated, and the paths they take are the
kernels' own bounds-checked ones (a workspace reserved too small makes each stage return
before writing, a dense event overflows the 2048-entry ring of tracks to follow, which the
kernel indexes modulo its size and flags).  Parity cases force the fallbacks that typical
events never reach: the retina decoder's full key comparison and the Kalman filter's
in-place hit reads.
"""
import numpy as np
import pytest

import parity
from allen_b200 import generator
from allen_b200.chain import VeloError, upload
from allen_b200.rawbanks import super_pixels_per_event

pytestmark = pytest.mark.gpu

VELO_ERR_CAPACITY = 3
VELO_ERR_DEVICE_FLAGS = 4
ERR_TTF_OVERFLOW = 1 << 2
ERR_INPUT_CAPACITY = 1 << 6


def run_chain(chain, s, use_graph=False):
    chain.reserve_for(s)
    chain.run(upload(s), use_graph=use_graph)
    totals = chain.synchronize()
    return totals, chain.outputs_to_host(totals)


@pytest.mark.parametrize("capacity", [0, 256])
def test_retina_full_comparison_rank(chain, oracle, geometry, capacity):
    """Retina clusters ranked by comparing every pair of keys (events above the bucket
    order's capacity take that path) give the oracle's sorted container, bit for bit."""
    g = generator.generate(60, seed=140 + capacity, raw_format=1, bank_version=3, pileup_min=1.0,
                           pileup_max=15.0)
    saved = chain.get_config()
    try:
        chain.configure(retina_order_capacity=capacity)
        totals, out = run_chain(chain, g.raw, use_graph=True)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []
    finally:
        chain.configure(**saved)


@pytest.mark.parametrize("warp_hits", [0, 64])
def test_kalman_hits_read_in_place(chain, oracle, geometry, warp_hits):
    """The Kalman filter with its per-warp staging capped (0: every span read in place; 64:
    most spans of 32 tracks exceed it) gives the oracle's states, bit for bit."""
    g = generator.generate(80, seed=57, pileup_min=5.0, pileup_max=15.0)
    saved = chain.get_config()
    chain.reserve_for(g.raw)
    chain.set_kalman(True, (0.1, -0.05))
    try:
        chain.configure(kalman_warp_hits=warp_hits)
        chain.run(upload(g.raw), use_graph=True)
        totals = chain.synchronize()
        got = chain.kalman_outputs(totals)
    finally:
        chain.set_kalman(False)
        chain.configure(**saved)
    ref = oracle.run(g.raw, geometry, beamline=(0.1, -0.05))
    reco = totals["host_number_of_reconstructed_velo_tracks"]
    assert reco == int(ref["dev_offsets_all_velo_tracks"][-1])
    assert np.array_equal(got["dev_is_backward"], ref["dev_is_backward"])
    w = parity.kalman_written_words(reco)
    for k in ("dev_velo_kalman_beamline_states", "dev_velo_kalman_endvelo_states"):
        assert np.array_equal(got[k].view(np.uint32)[w], ref[k].view(np.uint32)[w]), k
    with pytest.raises(VeloError):
        chain.configure(kalman_warp_hits=369)


def test_workspace_too_small(chain, oracle, geometry):
    """More events than reserved: VELO_ERR_CAPACITY before anything is queued.  More super
    pixels than reserved: the stages find the slice too large, write nothing, and the run
    ends in VELO_ERR_DEVICE_FLAGS with err_input_capacity; the chain then runs a slice that
    fits as before."""
    small = generator.generate(20, seed=61, mean_pileup=2.0).raw
    big = generator.generate(20, seed=62, mean_pileup=15.0, noise_rate=1e-4).raw
    # the reservation holds 2 estimated clusters per reserved super pixel: exceed that
    assert super_pixels_per_event(big).sum() > 3 * super_pixels_per_event(small).sum()
    chain.reserve_for(small)
    chain.set_kalman(True, (0.0, 0.0))
    try:
        more = generator.generate(21, seed=63).raw
        with pytest.raises(VeloError) as e:
            chain.run(upload(more))
        assert e.value.status == VELO_ERR_CAPACITY
        chain.run(upload(big))
        with pytest.raises(VeloError) as e:
            chain.synchronize()
        assert e.value.status == VELO_ERR_DEVICE_FLAGS
        assert e.value.flags & ERR_INPUT_CAPACITY
    finally:
        chain.set_kalman(False)
    totals, out = run_chain(chain, small)
    assert totals["device_flags"] == 0
    assert parity.compare(out, oracle.run(small, geometry), small.n_events) == []


def test_ring_overflow_is_flagged(chain):
    """Events dense enough to hold more than 2048 tracks to follow at once (the reference
    overwrites ring entries it has not read yet): the run reports err_ttf_overflow through
    VELO_ERR_DEVICE_FLAGS instead of returning silently different tracks."""
    g = generator.generate(2, seed=64, mean_pileup=150.0)
    chain.reserve_for(g.raw)
    chain.run(upload(g.raw))
    with pytest.raises(VeloError) as e:
        chain.synchronize()
    assert e.value.status == VELO_ERR_DEVICE_FLAGS
    assert e.value.flags & ERR_TTF_OVERFLOW
    # the chain stays usable
    s = generator.generate(10, seed=65).raw
    totals, _ = run_chain(chain, s)
    assert totals["device_flags"] == 0
