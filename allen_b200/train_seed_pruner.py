"""Trains, tunes and evaluates the learned seed gate on one GPU.

    python -m allen_b200.train_seed_pruner [--train-events 300000] [--eval-events 100000]
    python -m allen_b200.train_seed_pruner --evaluate-only allen_b200/data/seed_pruner.npz \
        --pileup 15 --noise 1e-4 --efficiency 0.95 --slice 4000          # the stress workload

Training candidates come from the plain search on generated events at nu = 7.6 (label: the
plain seeding made a seed with the candidate as middle hit); the network is trained by the
library's own tensor-core forward/backward kernels with Adam (lr 1e-3, batch 65536).  Logit
thresholds for several recall targets come from held-out records; allen_b200.autotune's
tune_learned() then picks the threshold, the seed window and the learned launch configuration
that run fastest with efficiency and ghost rate within 0.2 % of the plain search on held-out
events; the per-event fallback bounds come from the gate's kept fractions on those events.  The
evaluation compares learned and plain modes on --eval-events held-out events: events/s of the
whole chain, and tracking efficiency, ghost and clone rates (TrackChecker rules against the
generator's truth, counted on the GPU over every evaluation event).  The model goes to
allen_b200/data/seed_pruner.npz, its launch configuration to
allen_b200/data/launch_config_learned.json, the report to --report.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import autotune
from . import seed_pruner as sp

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DEFAULT_MODEL = os.path.join(DATA, "seed_pruner.npz")
LEARNED_CONFIG = os.path.join(DATA, "launch_config_learned.json")
TOLERANCE = 0.002


def _portable(v):
    """A path inside the repository as a path relative to its root (the report names no machine
    path); other values unchanged."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if isinstance(v, str) and os.path.isabs(v) and os.path.commonpath([root, os.path.abspath(v)]) == root:
        return os.path.relpath(v, root)
    return v


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--train-events", type=int, default=300000)
    p.add_argument("--val-events", type=int, default=16000)
    p.add_argument("--eval-events", type=int, default=100000)
    p.add_argument("--slice", type=int, default=16000)
    p.add_argument("--every", type=int, default=4)
    p.add_argument("--epochs", type=int, default=3)
    p.add_argument("--batch", type=int, default=65536)
    p.add_argument("--lr", type=float, default=1e-3)
    p.add_argument("--pos-weight", type=float, default=1.0)
    p.add_argument("--pileup", type=float, default=7.6)
    p.add_argument("--noise", type=float, default=1e-5, help="noise pixels per pixel of the evaluation events")
    p.add_argument("--efficiency", type=float, default=0.98, help="hit efficiency of the evaluation events")
    p.add_argument("--evaluate-only", default="", help="skip training: evaluate this saved model")
    p.add_argument("--out", default=DEFAULT_MODEL)
    p.add_argument("--config-out", default=LEARNED_CONFIG)
    p.add_argument("--report", default="")
    return p.parse_args()


def generated(args, seed: int, n_events: int, training_like: bool = False):
    """Generated slices (Generated objects, with truth) and their device copies."""
    from . import generator
    from .chain import upload
    cfg = {} if training_like else {"noise_rate": args.noise, "hit_efficiency": args.efficiency}
    gens = [generator.generate(min(args.slice, n_events - f), seed=seed, first_event=f, mean_pileup=args.pileup, **cfg)
            for f in range(0, n_events, args.slice)]
    return gens, [upload(g.raw) for g in gens]


def reserve_for_all(chain, gens):
    from .rawbanks import super_pixels_per_event
    chain.reserve(max(g.raw.n_events for g in gens), max(int(super_pixels_per_event(g.raw).sum()) for g in gens) + 64)


def quality_over(chain, gens, dev, truths) -> dict:
    """Efficiency, ghost and clone rates of the chain's current mode over every slice (counted on
    the GPU), with the seeding's candidate statistics."""
    from .validation import evaluate_device
    tot = dict(tracks=0, ghosts=0, reconstructible=0, reconstructed=0, clones=0)
    cand = searched = fallback = 0
    for g, d, t in zip(gens, dev, truths):
        chain.run(d, use_graph=False)
        chain.synchronize()
        r = evaluate_device(chain, t)
        for k in tot:
            tot[k] += r[k]
        st = chain.seed_stats(g.raw.n_events)
        cand += int(st[:, 0].sum())
        searched += int(st[:, 1].sum())
        fallback += int((st[:, 2] == 2).sum())
    n = sum(g.raw.n_events for g in gens)
    return dict(tot, events=n, efficiency=tot["reconstructed"] / max(tot["reconstructible"], 1),
                ghost_rate=tot["ghosts"] / max(tot["tracks"], 1),
                clone_rate=tot["clones"] / max(tot["reconstructed"] + tot["clones"], 1),
                candidates_per_event=cand / n, searched_fraction=searched / max(cand, 1),
                fallback_fraction=fallback / n)


def kept_fraction_bounds(chain, model, dev, gens):
    """The gate's per-event kept fraction with the fallback off; bounds: half the 0.1 % quantile
    and 1 (keeping every candidate is the plain search's cost, not an accuracy risk)."""
    model.kept_lo, model.kept_hi = 0.0, 1.0
    chain.set_seed_model(model)
    fr = []
    for d, g in zip(dev, gens):
        chain.run(d, use_graph=False)
        chain.synchronize()
        st = chain.gate_stats(g.raw.n_events)
        ok = st[:, 0] > 0
        fr.append(st[ok, 1] / st[ok, 0])
    fr = np.concatenate(fr)
    q = float(np.quantile(fr, 0.001))
    return 0.5 * q, 1.0, {"kept_fraction_median": float(np.median(fr)), "kept_fraction_q001": q}


def main():
    import torch
    from .chain import VeloChain
    from .validation import DeviceTruth

    args = parse()
    torch.cuda.set_device(0)
    t0 = time.time()
    log = lambda m: print(f"[{time.time() - t0:7.1f} s] {m}", flush=True)  # noqa: E731
    report = {"args": {k: _portable(v) for k, v in vars(args).items() if k != "report"},
              "device": torch.cuda.get_device_name(0)}
    chain = VeloChain()
    plain_config = chain.get_config()

    if args.evaluate_only:
        model = sp.load(args.evaluate_only)
        learned_config = sp.load_learned_config()
        report["model"] = args.evaluate_only
    else:
        cap = lambda n: int(n * 900 // args.every) + 4096  # noqa: E731  (about 700 candidates per event)
        train, n_train, n_counted = sp.collect_generated(chain, args.train_events, args.slice, 101, args.every,
                                                         cap(args.train_events), mean_pileup=args.pileup)
        val, n_val, _ = sp.collect_generated(chain, args.val_events, args.slice, 202, args.every,
                                             cap(args.val_events), mean_pileup=args.pileup)
        log(f"records: {n_train} training ({n_counted} counted), {n_val} held out")
        report["records"] = {"train": n_train, "validation": n_val,
                             "positive_fraction": float(sp.records_to_host(val, n_val)["label"].mean())}
        model = sp.initial_model(train, n_train, seed=7)
        trainer = sp.Trainer(model, lr=args.lr, pos_weight=args.pos_weight)
        t_train = time.time()
        history = sp.train(trainer, train, n_train, epochs=args.epochs, batch=args.batch, seed=11, log=log)
        torch.cuda.synchronize()
        report["training"] = {"loss_per_epoch": history, "seconds": round(time.time() - t_train, 2),
                              "steps": args.epochs * max(1, n_train // args.batch)}
        thresholds, calib = {}, {}
        for recall in autotune.GATE_RECALLS:
            thr, stats = sp.calibrate_threshold(trainer, val, n_val, recall)
            thresholds[recall] = thr
            calib[str(recall)] = dict(stats, threshold_logit=thr)
        log(f"thresholds {calib}")
        report["calibration"] = calib
        model = trainer.model()
        trainer.close()
        del train
        torch.cuda.empty_cache()

        # tuning on held-out events of the training configuration (stream 303)
        gens, dev = generated(args, 303, args.val_events, training_like=True)
        truths = [DeviceTruth(g) for g in gens]
        reserve_for_all(chain, gens)
        chain.set_seed_model(None)
        plain_q = quality_over(chain, gens, dev, truths)
        model.kept_lo, model.kept_hi = 0.0, 1.0
        best, rate, trials = autotune.tune_learned(
            chain, model, thresholds, dev, lambda ch: quality_over(ch, gens, dev, truths), plain_q,
            tolerance=TOLERANCE, log=log)
        model.threshold_logit = best["threshold_logit"]
        lo, hi, fstats = kept_fraction_bounds(chain, model, dev, gens)
        model.kept_lo, model.kept_hi = lo, hi
        report["tuning"] = {"best": best, "events_per_s": rate, "plain_quality": plain_q, "trials": trials}
        report["fallback_bounds"] = dict(fstats, kept_lo=lo, kept_hi=hi)
        log(f"tuned {best} at {rate:,.0f} events/s; fallback bounds [{lo:.4f}, {hi:.4f}]")
        os.makedirs(os.path.dirname(args.out), exist_ok=True)
        sp.save(model, args.out)
        learned_config = {k: best[k] for k in ("seed_window", "search_threads", "search_ring_global",
                                               "events_per_claim")}
        with open(args.config_out, "w") as f:
            json.dump({"config": dict(learned_config, search_lanes_per_seed=0, persistent=1),
                       "recall": best["recall"], "threshold_logit": best["threshold_logit"],
                       "events_per_s": rate, "tolerance": TOLERANCE}, f, indent=1)
        learned_config = sp.load_learned_config(args.config_out)
        chain.set_seed_model(None)
        chain.configure(**plain_config)
        del dev, gens, truths

    # evaluation on held-out events (stream 404): events/s of the whole chain per mode and the
    # tracking quality over every evaluation event
    gens, dev = generated(args, 404, args.eval_events)
    truths = [DeviceTruth(g) for g in gens]
    reserve_for_all(chain, gens)
    ev = {}
    for mode in ("plain", "learned"):
        if mode == "learned":
            chain.configure(**learned_config)
            chain.set_seed_model(model)
        else:
            chain.set_seed_model(None)
            chain.configure(**plain_config)
        ev[mode] = {"events_per_s": sp.measure(chain, dev)}
        ev[mode]["quality"] = quality_over(chain, gens, dev, truths)
        log(f"{mode}: {ev[mode]}")
    chain.set_seed_model(None)
    report["evaluation"] = ev
    qp, ql = ev["plain"]["quality"], ev["learned"]["quality"]
    report["speedup_learned_over_plain"] = ev["learned"]["events_per_s"] / ev["plain"]["events_per_s"]
    report["efficiency_delta"] = ql["efficiency"] - qp["efficiency"]
    report["ghost_rate_delta"] = ql["ghost_rate"] - qp["ghost_rate"]
    report["clone_rate_delta"] = ql["clone_rate"] - qp["clone_rate"]
    report["within_tolerance"] = report["efficiency_delta"] >= -TOLERANCE and report["ghost_rate_delta"] <= TOLERANCE
    log(json.dumps({k: report[k] for k in ("speedup_learned_over_plain", "efficiency_delta", "ghost_rate_delta",
                                           "clone_rate_delta", "within_tolerance")}))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1, default=float)
    chain.close()


if __name__ == "__main__":
    main()
