"""velo_kalman_filter on the GPU against the oracle, bit for bit (written state fields)."""
import ctypes as C

import numpy as np
import pytest

import parity
from allen_b200 import generator
from allen_b200.chain import upload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("beamline", [(0.0, 0.0), (0.35, -0.2)])
def test_chain_kalman_matches_oracle(chain, oracle, geometry, beamline):
    g = generator.generate(120, seed=55, pileup_min=1.0, pileup_max=15.0)
    chain.reserve_for(g.raw)
    chain.set_kalman(True, beamline)
    try:
        chain.run(upload(g.raw), use_graph=True)
        totals = chain.synchronize()
        got = chain.kalman_outputs(totals)
    finally:
        chain.set_kalman(False)
    ref = oracle.run(g.raw, geometry, beamline=beamline)
    reco = totals["host_number_of_reconstructed_velo_tracks"]
    assert reco == int(ref["dev_offsets_all_velo_tracks"][-1])
    assert np.array_equal(got["dev_is_backward"], ref["dev_is_backward"])
    w = parity.kalman_written_words(reco)
    for k in ("dev_velo_kalman_beamline_states", "dev_velo_kalman_endvelo_states"):
        assert np.array_equal(got[k].view(np.uint32)[w], ref[k].view(np.uint32)[w]), k


def test_standalone_kalman_entry_point(chain, oracle, geometry):
    """velo_run_kalman_filter() on the chain's consolidated outputs, into caller buffers."""
    import torch
    from allen_b200.chain import _current_stream
    g = generator.generate(60, seed=56)
    chain.reserve_for(g.raw)
    chain.run(upload(g.raw))
    totals = chain.synchronize()
    p = chain.device_outputs()
    reco = totals["host_number_of_reconstructed_velo_tracks"]
    back = torch.zeros(reco + 1, dtype=torch.uint8, device="cuda")
    beam = torch.zeros(56 * reco + 8, dtype=torch.uint8, device="cuda")
    end = torch.zeros(56 * reco + 8, dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = chain.lib.velo_run_kalman_filter(g.raw.n_events, p["dev_offsets_all_velo_tracks"],
                                      p["dev_offsets_velo_track_hit_number"], p["dev_velo_track_hits"], reco,
                                      0.0, 0.0, back.data_ptr(), beam.data_ptr(), end.data_ptr(), status.data_ptr(),
                                      _current_stream())
    assert st == 0
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref = oracle.run(g.raw, geometry)
    assert np.array_equal(back.cpu().numpy()[:reco], ref["dev_is_backward"])
    w = parity.kalman_written_words(reco)
    assert np.array_equal(beam.cpu().numpy()[:56 * reco].view(np.uint32)[w],
                          ref["dev_velo_kalman_beamline_states"].view(np.uint32)[w])
    assert np.array_equal(end.cpu().numpy()[:56 * reco].view(np.uint32)[w],
                          ref["dev_velo_kalman_endvelo_states"].view(np.uint32)[w])
    # too small a capacity is reported, nothing written
    status.zero_()
    st = chain.lib.velo_run_kalman_filter(g.raw.n_events, p["dev_offsets_all_velo_tracks"],
                                      p["dev_offsets_velo_track_hit_number"], p["dev_velo_track_hits"], reco - 1,
                                      0.0, 0.0, back.data_ptr(), beam.data_ptr(), end.data_ptr(), status.data_ptr(),
                                      _current_stream())
    torch.cuda.synchronize()
    assert st == 0 and int(status.item()) != 0
