"""Learned seed gate of the triplet search: training data, GPU training, calibration.

Workflow (all GPU work through the C ABI of libvelo_b200.so):

1. ``collect``: the chain runs the plain search over generated slices and records one seed
   candidate (a hit the seeding met unused as middle hit h1) in ``every``, with its 12
   features and, as label, whether the plain seeding made a seed with it
   (velo_chain_record_seeds).
2. ``initial_model``: feature standardisation from a sample of the records, He-initialised
   weights from a seeded generator.
3. ``train``: Adam steps of the tensor-core forward/backward kernels (velo_seed_trainer_step)
   over shuffled batches held in HBM.
4. ``calibrate_threshold``: the logit threshold that keeps ``recall`` of the positive
   candidates of held-out records; the per-event bounds on the kept fraction beyond which an
   event is searched by the plain search instead come from held-out events.

No counterpart in the reference (its seeding, SearchByTriplet.cu:298-446, searches every
unused hit as h1).
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from .chain import SEED_PARAMS, SeedModelC, VeloChain, _check, _current_stream, _lib

RECORD_BYTES = 64
N_FEATURES = 12
HIDDEN = 32


def model_from_params(params, mean, inv_std, threshold_logit=0.0, kept_lo=0.0, kept_hi=1.0) -> SeedModelC:
    p = np.asarray(params, np.float32)
    assert p.size == SEED_PARAMS
    m = SeedModelC()
    o = 0
    for name, size in (("w1", HIDDEN * N_FEATURES), ("b1", HIDDEN), ("w2", HIDDEN * HIDDEN), ("b2", HIDDEN),
                       ("w3", HIDDEN)):
        C.memmove(C.addressof(getattr(m, name)), p[o:o + size].ctypes.data, 4 * size)
        o += size
    m.b3 = float(p[o])
    C.memmove(C.addressof(m.mean), np.asarray(mean, np.float32).ctypes.data, 4 * N_FEATURES)
    C.memmove(C.addressof(m.inv_std), np.asarray(inv_std, np.float32).ctypes.data, 4 * N_FEATURES)
    m.threshold_logit = float(threshold_logit)
    m.kept_lo = float(kept_lo)
    m.kept_hi = float(kept_hi)
    return m


def model_params(m: SeedModelC) -> np.ndarray:
    parts = [np.ctypeslib.as_array(getattr(m, n)).astype(np.float32).ravel() for n in ("w1", "b1", "w2", "b2", "w3")]
    return np.concatenate(parts + [np.array([m.b3], np.float32)])


def model_dict(m: SeedModelC) -> dict:
    return {"params": model_params(m), "mean": np.ctypeslib.as_array(m.mean).copy(),
            "inv_std": np.ctypeslib.as_array(m.inv_std).copy(), "threshold_logit": np.float32(m.threshold_logit),
            "kept_lo": np.float32(m.kept_lo), "kept_hi": np.float32(m.kept_hi)}


def save(m: SeedModelC, path: str):
    np.savez(path, **model_dict(m))


def load(path: str) -> SeedModelC:
    z = np.load(path)
    return model_from_params(z["params"], z["mean"], z["inv_std"], float(z["threshold_logit"]), float(z["kept_lo"]),
                             float(z["kept_hi"]))


LEARNED_CONFIG = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "launch_config_learned.json")
DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "seed_pruner.npz")


def load_learned_config(path: str = LEARNED_CONFIG) -> dict:
    """The launch configuration tuned for the learned mode (seed window, gated search kernel,
    events per claim), for VeloChain.configure; empty when none was tuned."""
    try:
        with open(path) as f:
            return dict(json.load(f)["config"])
    except (OSError, KeyError, ValueError):
        return {}


def use_learned(chain: VeloChain, path: str = DEFAULT_MODEL, config_path: str = LEARNED_CONFIG):
    """Switches a chain to learned mode with the committed model and its tuned configuration."""
    chain.configure(**load_learned_config(config_path))
    chain.set_seed_model(load(path))


def he_params(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, np.sqrt(2.0 / N_FEATURES), (HIDDEN, N_FEATURES))
    w2 = rng.normal(0, np.sqrt(2.0 / HIDDEN), (HIDDEN, HIDDEN))
    w3 = rng.normal(0, np.sqrt(1.0 / HIDDEN), HIDDEN)
    return np.concatenate([w1.ravel(), np.zeros(HIDDEN), w2.ravel(), np.zeros(HIDDEN), w3, [0.0]]).astype(np.float32)


RECORD_DTYPE = np.dtype([("f", np.float32, (N_FEATURES,)), ("label", np.float32), ("event", np.uint32),
                         ("h0", np.uint32), ("h1", np.uint32)])


def records_to_host(records, n: int) -> np.ndarray:
    """First n records of a device uint8 tensor as a numpy structured array."""
    return records[:RECORD_BYTES * n].cpu().numpy().view(RECORD_DTYPE)


def collect(chain: VeloChain, dev_slices, capacity: int, every: int = 1):
    """Runs the plain search over the slices, recording training candidates.  Returns the
    device tensor of records (uint8, 64 bytes each), how many were written and how many counted."""
    import torch
    records = torch.empty(RECORD_BYTES * capacity, dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    chain.set_seed_model(None)
    chain.record_seeds(records, count, every)
    try:
        for d in dev_slices:
            chain.run(d, use_graph=False)
            chain.synchronize()
    finally:
        chain.record_seeds(None, None)
    n = int(count.item())
    return records, min(n, capacity), n


def feature_stats(records, n: int, sample: int = 262144, seed: int = 0):
    """Mean and 1 / std of each feature over a random sample of the records."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    idx = torch.randperm(n, generator=g)[:min(sample, n)].to("cuda")
    rows = records[:RECORD_BYTES * n].view(n, RECORD_BYTES).index_select(0, idx).cpu().numpy().view(RECORD_DTYPE)
    f = rows["f"].reshape(-1, N_FEATURES).astype(np.float64)
    mean = f.mean(0)
    std = f.std(0)
    return mean.astype(np.float32), (1.0 / np.maximum(std, 1e-6)).astype(np.float32)


def initial_model(records, n: int, seed: int = 0) -> SeedModelC:
    mean, inv_std = feature_stats(records, n, seed=seed)
    return model_from_params(he_params(seed), mean, inv_std)


class Trainer:
    """velo_seed_trainer_*: fp32 master weights and Adam state in HBM, bf16 tensor-core passes."""

    def __init__(self, model: SeedModelC, lr: float = 1e-3, pos_weight: float = 1.0):
        self.lib = _lib()
        self.handle = C.c_void_p()
        self.model_meta = model
        _check(self.lib, self.lib.velo_seed_trainer_create(C.byref(model), lr, pos_weight, C.byref(self.handle)))

    def step(self, records, first: int, batch: int, want_loss: bool = False):
        loss = C.c_float()
        _check(self.lib, self.lib.velo_seed_trainer_step(self.handle, records.data_ptr(), first, batch, _current_stream(),
                                                         C.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def gradients(self, records, first: int, batch: int):
        grads = np.zeros(SEED_PARAMS, np.float32)
        loss = C.c_float()
        _check(self.lib, self.lib.velo_seed_trainer_gradients(
            self.handle, records.data_ptr(), first, batch, _current_stream(),
            grads.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return loss.value, grads

    def score(self, records, n: int):
        import torch
        logits = torch.empty(max(n, 1), dtype=torch.float32, device="cuda")
        _check(self.lib, self.lib.velo_seed_trainer_score(self.handle, records.data_ptr(), n, logits.data_ptr(),
                                                          _current_stream()))
        return logits[:n]

    def model(self) -> SeedModelC:
        m = SeedModelC()
        _check(self.lib, self.lib.velo_seed_trainer_model(self.handle, C.byref(m)))
        return m

    def close(self):
        if self.handle:
            self.lib.velo_seed_trainer_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def shuffled(records, n: int, seed: int):
    """The first n records in a seeded random order (a device gather)."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    perm = torch.randperm(n, generator=g).to("cuda")
    return records[:RECORD_BYTES * n].view(n, RECORD_BYTES).index_select(0, perm).reshape(-1).contiguous()


def train(trainer: Trainer, records, n: int, epochs: int = 2, batch: int = 65536, seed: int = 0, log=None):
    """Adam over shuffled copies of the records (one per epoch); returns the mean loss of
    each epoch's last tenth of steps."""
    history = []
    for ep in range(epochs):
        data = shuffled(records, n, seed + ep)
        steps = max(1, n // batch)
        tail = []
        for k in range(steps):
            want = k >= steps - max(1, steps // 10)
            loss = trainer.step(data, k * batch, min(batch, n - k * batch), want_loss=want)
            if want:
                tail.append(loss)
        history.append(float(np.mean(tail)))
        if log:
            log(f"epoch {ep}: loss {history[-1]:.4f} ({steps} steps of {batch})")
        del data
    return history


def calibrate_threshold(trainer: Trainer, records, n: int, recall: float) -> tuple[float, dict]:
    """Logit threshold that keeps `recall` of the positive candidates among records [0, n)."""
    logits = trainer.score(records, n).cpu().numpy()
    labels = records_to_host(records, n)["label"]
    pos = np.sort(logits[labels > 0.5])
    if pos.size == 0:
        return float("-inf"), {}
    k = int(np.floor((1.0 - recall) * pos.size))
    thr = float(np.nextafter(pos[k], np.float32(-np.inf))) if k < pos.size else float(pos[-1])
    kept = logits > thr
    stats = {"positives": int(pos.size), "candidates": int(n), "recall": float(np.mean(pos > thr)),
             "kept_fraction": float(kept.mean()),
             "precision": float(np.mean(labels[kept] > 0.5)) if kept.any() else 0.0}
    return thr, stats


def collect_generated(chain: VeloChain, n_events: int, slice_events: int, seed: int, every: int, capacity: int, **gen):
    """Generates n_events events (stream `seed`) slice by slice and records their training
    candidates from the plain search.  Returns (records, n, n_total_counted)."""
    import torch
    from . import generator
    from .chain import upload
    from .rawbanks import super_pixels_per_event
    records = torch.empty(RECORD_BYTES * capacity, dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    chain.set_seed_model(None)
    chain.record_seeds(records, count, every)
    try:
        for first in range(0, n_events, slice_events):
            s = generator.generate(min(slice_events, n_events - first), seed=seed, first_event=first, **gen).raw
            chain.reserve(s.n_events, int(super_pixels_per_event(s).sum()) + 64)
            chain.run(upload(s), use_graph=False)
            chain.synchronize()
    finally:
        chain.record_seeds(None, None)
    n = int(count.item())
    return records, min(n, capacity), n


def measure(chain: VeloChain, dev_slices, repeats: int = 3) -> float:
    """events/s of the chain over the slices (CUDA graphs, CUDA-event timed)."""
    import torch
    for d in dev_slices:
        chain.run(d, use_graph=True)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(repeats):
        for d in dev_slices:
            chain.run(d, use_graph=True)
    end.record()
    torch.cuda.synchronize()
    return repeats * sum(d.n_events for d in dev_slices) / (start.elapsed_time(end) / 1e3)


def quality(chain: VeloChain, gen) -> dict:
    """Tracking efficiency, ghost and clone rates (TrackChecker rules) of one generated slice,
    counted on the device (velo_validate_tracks), with the seeding's candidate statistics."""
    from .chain import upload
    from .validation import DeviceTruth, evaluate_device
    chain.reserve_for(gen.raw)
    chain.run(upload(gen.raw), use_graph=False)
    chain.synchronize()
    res = evaluate_device(chain, DeviceTruth(gen))
    st = chain.seed_stats(gen.raw.n_events)
    res["candidates"] = int(st[:, 0].sum())
    res["candidates_searched"] = int(st[:, 1].sum())
    res["fallback_events"] = int((st[:, 2] == 2).sum())
    return res
