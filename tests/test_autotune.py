"""The autotuner's coordinate descent on a stand-in chain (no GPU): the best search kernel depends on
a staging capacity chosen after it, which one sweep misses and the repeated sweeps find; invalid
configurations (global rings without persistent launches) are skipped."""
from allen_b200 import autotune


class FakeChain:
    def __init__(self):
        self.cfg = {"search_threads": 256, "search_lanes_per_seed": 2, "search_hit_capacity": 3072,
                    "cluster_stage_capacity": 3072, "cluster_blob_bytes": 16384, "estimate_blob_bytes": 32768,
                    "persistent": 0, "events_per_claim": 1, "search_ring_global": 0, "cluster_threads": 256}

    def get_config(self):
        return dict(self.cfg)

    def configure(self, **cfg):
        if cfg.get("search_ring_global") and not cfg.get("persistent"):
            raise RuntimeError("global rings need persistent launches")
        self.cfg = dict(cfg)

    def rate(self):
        c = self.cfg
        r = 1.0
        # the 128-thread global-ring search only pays once the hits are staged in global scratch
        if (c["search_threads"], c["search_lanes_per_seed"], c["search_ring_global"]) == (128, 0, 1):
            r *= 1.5 if c["search_hit_capacity"] == 0 else 0.7
        elif c["search_lanes_per_seed"] == 0:
            r *= 1.2 if c["search_threads"] == 256 else 1.1
        r *= 1.1 if c["search_hit_capacity"] == 0 else 1.0
        r *= 1.05 if c["persistent"] else 1.0
        return r


def test_sweeps_repeat_until_nothing_changes(monkeypatch):
    chain = FakeChain()
    monkeypatch.setattr(autotune, "measure", lambda ch, dev, repeats=3: ch.rate())
    best, rate, trials = autotune.tune(chain, [], log=lambda *_: None)
    assert (best["search_threads"], best["search_lanes_per_seed"], best["search_ring_global"]) == (128, 0, 1)
    assert best["search_hit_capacity"] == 0 and best["persistent"] == 1
    assert rate == chain.rate() and chain.cfg == best
    # one sweep alone stops at the flat 256-thread kernel
    chain1 = FakeChain()
    best1, _, _ = autotune.tune(chain1, [], log=lambda *_: None, max_sweeps=1)
    assert best1["search_threads"] == 256 and best1["search_lanes_per_seed"] == 0
    # the ring variants were tried with persistent launches, never without
    assert all(t["config"]["persistent"] for t in trials if t["config"]["search_ring_global"])


class FakeLearnedChain(FakeChain):
    """Stand-in for the learned mode: rate rises as the gate keeps less and the window
    shrinks; quality falls with them (recall below 0.98 or window 2 out of tolerance)."""

    def __init__(self):
        super().__init__()
        self.cfg.update(search_threads=128, search_lanes_per_seed=0, search_ring_global=1, persistent=1,
                        seed_window=0)
        self.threshold = None

    def configure(self, **cfg):  # VeloChain.configure: the given fields, the others kept
        merged = dict(self.cfg)
        merged.update(cfg)
        super().configure(**merged)

    def set_seed_model(self, model):
        self.threshold = model.threshold_logit

    def rate(self):
        r = 1.0 + 0.1 * self.threshold  # higher threshold: fewer candidates searched
        r *= {0: 1.0, 3: 1.04, 2: 1.08}[self.cfg["seed_window"]]
        r *= 1.05 if self.cfg["search_threads"] == 128 else 1.0
        r *= 1.02 if self.cfg["events_per_claim"] == 2 else 1.0
        return r

    def quality(self):
        recall = {1.0: 0.995, 2.0: 0.99, 3.0: 0.98, 4.0: 0.97}[self.threshold]
        eff = 0.994 - (0.003 if recall < 0.98 else 0.0) - (0.004 if self.cfg["seed_window"] == 2 else 0.0)
        return {"efficiency": eff, "ghost_rate": 0.003}


class Model:
    threshold_logit = 0.0


def test_learned_tuning_respects_the_quality_tolerance(monkeypatch):
    chain = FakeLearnedChain()
    monkeypatch.setattr(autotune, "measure", lambda ch, dev, repeats=3: ch.rate())
    thresholds = {0.995: 1.0, 0.99: 2.0, 0.98: 3.0, 0.97: 4.0}
    best, rate, trials = autotune.tune_learned(chain, Model(), thresholds, [], lambda ch: ch.quality(),
                                               {"efficiency": 0.994, "ghost_rate": 0.003}, log=lambda *_: None)
    # the fastest admissible gate: recall 0.98 (0.97 loses too much), window 3 (2 loses too much)
    assert (best["recall"], best["seed_window"]) == (0.98, 3)
    assert best["search_threads"] == 128 and best["events_per_claim"] == 2
    assert [t for t in trials if "admissible" in t and not t["admissible"]]
    assert rate == chain.rate()
