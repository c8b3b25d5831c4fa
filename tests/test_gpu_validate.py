"""On-device validation (velo_validate_tracks) against the host TrackChecker-rule restatement."""
import pytest

from allen_b200 import generator
from allen_b200.chain import upload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg", [dict(), dict(raw_format=1, bank_version=3),
                                 dict(mean_pileup=15.0, noise_rate=1e-4, hit_efficiency=0.95)])
def test_device_counts_equal_host_counts(chain, cfg):
    from allen_b200.validation import DeviceTruth, evaluate, evaluate_device, tracks_from_outputs
    g = generator.generate(200, seed=81, **cfg)
    chain.reserve_for(g.raw)
    chain.run(upload(g.raw))
    totals = chain.synchronize()
    host = evaluate(g, tracks_from_outputs(chain.outputs_to_host(totals)))
    dev = evaluate_device(chain, DeviceTruth(g))
    for k in ("tracks", "ghosts", "reconstructible", "reconstructed", "clones"):
        assert dev[k] == host[k], (k, dev[k], host[k])
    assert host["efficiency"] > 0.9
