"""Autotuner of the chain's launch configuration.

Sweeps, on a generated workload of the target occupancy, the search kernel's block size and
lanes per seed candidate (the compiled pairs), the clustering kernel's block size, the
shared-memory staging capacities of the search, clustering and estimate kernels, the place of the search's ring of tracks to follow, and
persistent launches with a work queue (events claimed per CTA) against one CTA per event, by
coordinate descent: each parameter in turn takes the
value with the highest events/s (CUDA-event timed graph replays) while the others stay at
the current best.  The winner is written to allen_b200/data/launch_config.json, which
VeloChain loads by default.  tune_learned() does the same for the learned mode, with the seed
gate's threshold and the seed window as coordinates constrained by tracking quality (run by
allen_b200.train_seed_pruner).

    python -m allen_b200.autotune [--events 16000] [--pileup-min 1 --pileup-max 15]
"""
from __future__ import annotations

import argparse
import json
import os
import time

# (block size, lanes per seed candidate, ring of tracks to follow in global scratch)
SEARCH_VARIANTS = [(128, 1, 0), (128, 2, 0), (256, 1, 0), (256, 2, 0), (256, 4, 0), (512, 2, 0), (512, 4, 0),
                   (128, 0, 0), (256, 0, 0), (512, 0, 0), (64, 0, 1), (96, 0, 1), (128, 0, 1), (256, 0, 1)]
SEARCH_CAPACITIES = [0, 1024, 2048, 2560, 3072, 4096]
CLUSTER_CAPACITIES = [0, 1024, 2048, 2560, 3072]
CLUSTER_BLOBS = [0, 16 * 1024, 24 * 1024, 32 * 1024, 40 * 1024]
CLUSTER_THREADS = [256, 128]
ESTIMATE_BLOBS = [0, 16 * 1024, 24 * 1024, 32 * 1024, 48 * 1024]
# (persistent, events per claim): one CTA per event, or resident CTAs claiming events
QUEUES = [(0, 1), (1, 1), (1, 2), (1, 4)]


def measure(chain, dev_slices, repeats=3) -> float:
    """events/s over `repeats` passes of all slices, graphs captured beforehand."""
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
    events = repeats * sum(d.n_events for d in dev_slices)
    return events / (start.elapsed_time(end) / 1e3)


def tune(chain, dev_slices, log=print, max_sweeps: int = 3) -> tuple[dict, float, list]:
    trials = []
    best = chain.get_config()

    def try_config(**upd):
        cfg = dict(best)
        cfg.update(upd)
        try:
            chain.configure(**cfg)
        except Exception as exc:  # configuration the device cannot hold
            log(f"skip {upd}: {exc}")
            return None
        rate = measure(chain, dev_slices)
        trials.append({"config": cfg, "events_per_s": rate})
        log(f"{upd} -> {rate:,.0f} events/s")
        return rate

    best_rate = try_config()
    coordinates = (
        ("search", SEARCH_VARIANTS),
        ("search_hit_capacity", SEARCH_CAPACITIES),
        ("cluster_stage_capacity", CLUSTER_CAPACITIES),
        ("cluster_threads", CLUSTER_THREADS),
        ("cluster_blob_bytes", CLUSTER_BLOBS),
        ("estimate_blob_bytes", ESTIMATE_BLOBS),
        ("queue", QUEUES),
    )
    # sweeps repeat until one changes nothing: the best search kernel depends on the staging
    # capacities chosen after it (its CTAs per SM), so one greedy sweep can stop short
    for sweep in range(max_sweeps):
        before = dict(best)
        for name, values in coordinates:
            best_rate = sweep_coordinate(name, values, best, best_rate, try_config)
        if best == before:
            break
    chain.configure(**best)
    return best, best_rate, trials


def sweep_coordinate(name, values, best, best_rate, try_config):
    """One coordinate: each value in turn against the current best; returns the new best rate."""
    for v in values:
        if name == "search":
            upd = {"search_threads": v[0], "search_lanes_per_seed": v[1], "search_ring_global": v[2]}
            if v[2]:
                upd["persistent"] = 1  # one ring per resident CTA
        elif name == "queue":
            upd = {"persistent": v[0], "events_per_claim": v[1]}
            if best.get("search_ring_global") and not v[0]:
                continue  # the global rings need persistent launches
        else:
            upd = {name: v}
        rate = try_config(**upd)
        if rate is not None and rate > best_rate:
            best_rate = rate
            best.update(upd)
    return best_rate


# learned mode: the gate's recall targets (each a logit threshold from the calibration), the
# seed window (h0 candidates per seed candidate; 0 = the reference's 4), the gated search kernels
# and the events a persistent CTA claims
GATE_RECALLS = [0.97, 0.98, 0.99, 0.995]
SEED_WINDOWS = [0, 3, 2]
GATED_SEARCH = [(128, 1), (256, 1), (96, 1), (64, 1)]
CLAIMS = [1, 2, 4]


def tune_learned(chain, model, thresholds: dict, dev_slices, quality, plain_quality: dict, tolerance: float = 0.002,
                 log=print, max_sweeps: int = 3) -> tuple[dict, float, list]:
    """The learned mode's seed gate and window, jointly with its launch configuration.

    thresholds: recall target -> logit threshold; quality(chain) -> {"efficiency", "ghost_rate"}
    of the chain's current mode on held-out events; plain_quality: the plain search's on the
    same events.  A (threshold, window) pair is admissible when its efficiency is at most
    `tolerance` below the plain search's and its ghost rate at most `tolerance` above; among
    admissible pairs, gated search kernels and claims, coordinate descent on events/s picks the
    best.  Returns ({"recall", "threshold_logit", "seed_window", launch parameters}, events/s,
    trials); the chain is left configured with it."""
    trials = []
    admissible = []
    for recall, thr in sorted(thresholds.items()):
        for window in SEED_WINDOWS:
            model.threshold_logit = float(thr)
            chain.set_seed_model(model)
            chain.configure(seed_window=window)
            q = quality(chain)
            ok = (q["efficiency"] >= plain_quality["efficiency"] - tolerance and
                  q["ghost_rate"] <= plain_quality["ghost_rate"] + tolerance)
            trials.append({"recall": recall, "seed_window": window, "quality": q, "admissible": ok})
            log(f"recall {recall} window {window}: {q} {'ok' if ok else 'out of tolerance'}")
            if ok:
                admissible.append((recall, window))
    if not admissible:
        raise RuntimeError("no gate threshold keeps the learned mode within tolerance")
    best = {"gate": admissible[-1], "search": (chain.get_config()["search_threads"], 1),
            "events_per_claim": chain.get_config()["events_per_claim"]}

    def apply(b):
        recall, window = b["gate"]
        model.threshold_logit = float(thresholds[recall])
        chain.configure(search_threads=b["search"][0], search_lanes_per_seed=0, search_ring_global=b["search"][1],
                        persistent=1, events_per_claim=b["events_per_claim"], seed_window=window)
        chain.set_seed_model(model)

    def rate_of(b):
        try:
            apply(b)
        except Exception as exc:
            log(f"skip {b}: {exc}")
            return None
        r = measure(chain, dev_slices)
        trials.append({"learned": dict(b), "events_per_s": r})
        log(f"{b} -> {r:,.0f} events/s")
        return r

    best_rate = rate_of(best) or 0.0
    for _ in range(max_sweeps):
        before = dict(best)
        for name, values in (("gate", admissible), ("search", GATED_SEARCH), ("events_per_claim", CLAIMS)):
            for v in values:
                cand = dict(best)
                cand[name] = v
                if cand == best:
                    continue
                r = rate_of(cand)
                if r is not None and r > best_rate:
                    best, best_rate = cand, r
        if best == before:
            break
    apply(best)
    recall, window = best["gate"]
    result = {"recall": recall, "threshold_logit": float(thresholds[recall]), "seed_window": window,
              "search_threads": best["search"][0], "search_ring_global": best["search"][1],
              "events_per_claim": best["events_per_claim"]}
    return result, best_rate, trials


def main():
    import torch
    from allen_b200 import _native, generator
    from allen_b200.chain import VeloChain, upload
    from allen_b200.rawbanks import super_pixels_per_event

    p = argparse.ArgumentParser()
    p.add_argument("--events", type=int, default=16000)
    p.add_argument("--slice", type=int, default=16000)
    p.add_argument("--pileup", type=float, default=7.6)
    p.add_argument("--pileup-min", type=float, default=0.0)
    p.add_argument("--pileup-max", type=float, default=0.0)
    p.add_argument("--seed", type=int, default=99)
    p.add_argument("--out", default=_native.TUNED_CONFIG)
    args = p.parse_args()
    torch.cuda.set_device(0)
    slices = []
    for first in range(0, args.events, args.slice):
        slices.append(generator.generate(min(args.slice, args.events - first), seed=args.seed, first_event=first,
                                         mean_pileup=args.pileup, pileup_min=args.pileup_min,
                                         pileup_max=args.pileup_max).raw)
    dev = [upload(s) for s in slices]
    chain = VeloChain(use_tuned=False)
    chain.reserve(max(s.n_events for s in slices), max(int(super_pixels_per_event(s).sum()) for s in slices) + 64)
    t0 = time.time()
    best, rate, trials = tune(chain, dev)
    workload = {k: v for k, v in vars(args).items() if k != "out"}
    result = {"config": best, "events_per_s": rate, "workload": workload, "trials": trials,
              "device": torch.cuda.get_device_name(0), "seconds": round(time.time() - t0, 1)}
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump(result, f, indent=1)
    print(json.dumps({"best": best, "events_per_s": rate}))
    chain.close()


if __name__ == "__main__":
    main()
