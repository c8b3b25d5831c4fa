"""MDF input through the B200 chain: records indexed and transposed on the host
(libvelo_io.so), reconstructed on the GPU, checked bit for bit against the oracle."""
import numpy as np
import pytest

import mdf_streams
import parity
from allen_b200 import generator, mdf
from allen_b200.chain import upload

pytestmark = pytest.mark.gpu


def run_chain(chain, s, retina=None):
    chain.reserve_for(s)
    d = upload(s)
    if retina is not None:
        d.retina = retina
    chain.run(d)
    totals = chain.synchronize()
    return totals, chain.outputs_to_host(totals)


@pytest.mark.parametrize("by_source_id", [False, True])
def test_mdf_stream_through_chain(chain, oracle, geometry, by_source_id):
    g = generator.generate(200, seed=31, pileup_min=1.0, pileup_max=15.0)
    stream = mdf_streams.synthetic_stream(g.raw, seed=10, by_source_id=by_source_id)
    ev = mdf.scan(stream, check_checksum=True)
    s = mdf.transpose_vp(stream, ev)
    if by_source_id:
        # the VELO source IDs carry their subdetector bits; the decoders read the sensor from
        # the low bits only for bank version 4, so compare against the oracle on the same slice
        totals, out = run_chain(chain, s)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(s, geometry), s.n_events) == []
    else:
        assert np.array_equal(s.raw, g.raw.raw)
        totals, out = run_chain(chain, s)
        assert totals["device_flags"] == 0
        assert parity.compare(out, oracle.run(g.raw, geometry), g.raw.n_events) == []


def test_mdf_slices_through_the_host_pipeline(oracle, geometry):
    """MDF records in slices through the end-to-end pipeline (page-locked slices, three chains):
    the tracks the host receives are the oracle's, for super-pixel and retina-cluster banks."""
    from allen_b200.chain import HostPipeline, pin_slice
    from allen_b200.rawbanks import super_pixels_per_event
    for gen in (dict(), dict(raw_format=1, bank_version=3)):
        g = generator.generate(240, seed=35, pileup_min=1.0, pileup_max=15.0, **gen)
        stream = mdf_streams.synthetic_stream(g.raw, seed=12)
        parts = list(mdf.slices(stream, events_per_slice=60))
        assert len(parts) == 4 and sum(p.n_events for p in parts) == 240
        pipe = HostPipeline()
        pipe.reserve(60, max(int(super_pixels_per_event(p).sum()) for p in parts) + 64,
                     max(p.raw.nbytes for p in parts), max(p.sizes.size for p in parts),
                     max(p.types.size for p in parts))
        totals, outs = pipe.run([pin_slice(p) for p in parts], keep_outputs=4)
        pipe.close()
        for part, out, t in zip(parts, outs, totals):
            assert t["device_flags"] == 0
            ref = oracle.run(part, geometry)
            assert np.array_equal(out["dev_offsets_all_velo_tracks"], ref["dev_offsets_all_velo_tracks"])
            assert np.array_equal(out["dev_offsets_velo_track_hit_number"], ref["dev_offsets_velo_track_hit_number"])
            TH = int(ref["dev_offsets_velo_track_hit_number"][-1])
            assert np.array_equal(out["dev_velo_track_hits_id_xyz"], parity._u8(ref["dev_velo_track_hits"])[:16 * TH])
