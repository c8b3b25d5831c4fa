"""Trains, calibrates and evaluates the learned seed pruner on one GPU.

    python -m allen_b200.train_seed_pruner [--train-events 300000] [--eval-events 100000]

Training doublets come from the plain search on generated events at nu = 7.6 (labels: the
doublet the plain seeding chose); the network is trained by the library's own tensor-core
forward/backward kernels with Adam (lr 1e-3, batch 65536).  The logit threshold keeps
--recall of the positive doublets of held-out events; the per-event fallback bounds are
set from the kept fractions of held-out events.  The evaluation compares the learned and
plain searches on held-out events: events/s of the whole chain and tracking efficiency,
ghost and clone rates (TrackChecker rules against the generator's truth).  The model goes
to allen_b200/data/seed_pruner.npz and the report to --report.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import seed_pruner as sp

DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "seed_pruner.npz")


def kept_fraction_bounds(chain, model, dev_slices, n_events_list):
    """Per-event kept fraction of doublets in learned mode with the fallback switched off;
    returns (lo, hi) bounds: half the 0.1% quantile, and 1 (keeping every doublet is the
    plain search's cost, not an accuracy risk)."""
    model.kept_lo, model.kept_hi = 0.0, 1.0
    chain.set_seed_model(model)
    fr = []
    for d, n in zip(dev_slices, n_events_list):
        chain.run(d, use_graph=False)
        chain.synchronize()
        st = chain.seed_stats(n)
        ok = st[:, 0] > 0
        fr.append(st[ok, 1] / st[ok, 0])
    fr = np.concatenate(fr)
    return 0.5 * float(np.quantile(fr, 0.001)), 1.0, {"kept_fraction_median": float(np.median(fr)),
                                                     "kept_fraction_q001": float(np.quantile(fr, 0.001))}


def train_phase():
    import torch
    from .chain import VeloChain

    p = argparse.ArgumentParser()
    p.add_argument("--train-events", type=int, default=300000)
    p.add_argument("--val-events", type=int, default=20000)
    p.add_argument("--eval-events", type=int, default=100000)
    p.add_argument("--quality-events", type=int, default=2000)
    p.add_argument("--slice", type=int, default=16000)
    p.add_argument("--every", type=int, default=64)
    p.add_argument("--epochs", type=int, default=3)
    p.add_argument("--batch", type=int, default=65536)
    p.add_argument("--lr", type=float, default=1e-3)
    p.add_argument("--pos-weight", type=float, default=1.0)
    p.add_argument("--recall", type=float, default=0.995)
    p.add_argument("--pileup", type=float, default=7.6)
    p.add_argument("--noise", type=float, default=1e-5, help="noise pixels per pixel of the evaluation events")
    p.add_argument("--efficiency", type=float, default=0.98, help="hit efficiency of the evaluation events")
    p.add_argument("--evaluate-only", default="", help="skip training: evaluate this saved model")
    p.add_argument("--out", default=DEFAULT_MODEL)
    p.add_argument("--report", default="")
    args = p.parse_args()
    if args.evaluate_only:
        torch.cuda.set_device(0)
        t0 = time.time()
        log = lambda m: print(f"[{time.time() - t0:7.1f} s] {m}", flush=True)  # noqa: E731
        chain = VeloChain()
        chain.configure(search_lanes_per_seed=0)
        report = {"args": vars(args), "device": torch.cuda.get_device_name(0), "model": args.evaluate_only}
        return args, report, chain, sp.load(args.evaluate_only), log
    torch.cuda.set_device(0)
    t0 = time.time()
    log = lambda m: print(f"[{time.time() - t0:7.1f} s] {m}", flush=True)  # noqa: E731
    report = {"args": vars(args), "device": torch.cuda.get_device_name(0)}

    chain = VeloChain()
    chain.configure(search_lanes_per_seed=0)
    cap = lambda n: int(n * 12000 // args.every) + 4096  # noqa: E731  (about 10k doublets per event)
    train, n_train, n_counted = sp.collect_generated(chain, args.train_events, args.slice, 101, args.every,
                                                     cap(args.train_events), mean_pileup=args.pileup)
    val, n_val, _ = sp.collect_generated(chain, args.val_events, args.slice, 202, args.every, cap(args.val_events),
                                         mean_pileup=args.pileup)
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
    thr, stats = sp.calibrate_threshold(trainer, val, n_val, args.recall)
    log(f"threshold {thr:.4f}: {stats}")
    report["calibration"] = dict(stats, threshold_logit=thr)
    model = trainer.model()
    model.threshold_logit = thr
    del train
    torch.cuda.empty_cache()
    return args, report, chain, model, log


def eval_slices(args, seed: int, n_events: int, training_like: bool = False):
    """Generated slices of the evaluation configuration (or of the training one)."""
    from . import generator
    from .chain import upload
    cfg = {} if training_like else {"noise_rate": args.noise, "hit_efficiency": args.efficiency}
    gens = [generator.generate(min(args.slice, n_events - f), seed=seed, first_event=f, mean_pileup=args.pileup, **cfg)
            for f in range(0, n_events, args.slice)]
    return gens, [upload(g.raw) for g in gens]


def main():
    import torch
    from .rawbanks import super_pixels_per_event
    args, report, chain, model, log = train_phase()
    if not args.evaluate_only:
        calibrate_bounds(args, report, chain, model, log)
    evaluate(args, report, chain, model, log)


def calibrate_bounds(args, report, chain, model, log):
    from .rawbanks import super_pixels_per_event
    # fallback bounds from held-out events (stream 303)
    gens, dev = eval_slices(args, 303, min(args.val_events, args.slice), training_like=True)
    chain.reserve(max(g.raw.n_events for g in gens), max(int(super_pixels_per_event(g.raw).sum()) for g in gens) + 64)
    lo, hi, fstats = kept_fraction_bounds(chain, model, dev, [g.raw.n_events for g in gens])
    model.kept_lo, model.kept_hi = lo, hi
    report["fallback_bounds"] = dict(fstats, kept_lo=lo, kept_hi=hi)
    log(f"fallback bounds [{lo:.4f}, {hi:.4f}] {fstats}")
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    sp.save(model, args.out)


def evaluate(args, report, chain, model, log):
    from .rawbanks import super_pixels_per_event
    # evaluation on held-out events (stream 404): throughput of the whole chain per mode
    gens, dev = eval_slices(args, 404, args.eval_events)
    chain.reserve(max(g.raw.n_events for g in gens), max(int(super_pixels_per_event(g.raw).sum()) for g in gens) + 64)
    ev = {}
    for mode in ("plain", "learned"):
        chain.set_seed_model(model if mode == "learned" else None)
        rate = sp.measure(chain, dev)
        fallback = doublets = scanned = 0
        for d, g in zip(dev, gens):
            chain.run(d, use_graph=False)
            chain.synchronize()
            st = chain.seed_stats(g.raw.n_events)
            fallback += int((st[:, 2] == 2).sum())
            doublets += int(st[:, 0].sum())
            scanned += int(st[:, 1].sum())
        ev[mode] = {"events_per_s": rate, "fallback_fraction": fallback / args.eval_events,
                    "doublets_per_event": doublets / args.eval_events,
                    "scanned_fraction": scanned / max(doublets, 1)}
        log(f"{mode}: {rate:,.0f} events/s, {ev[mode]}")
    # quality on the first events of the held-out stream
    qg = _generate_quality(args)
    for mode in ("plain", "learned"):
        chain.set_seed_model(model if mode == "learned" else None)
        ev[mode]["quality"] = sp.quality(chain, qg)
        log(f"{mode} quality: {ev[mode]['quality']}")
    chain.set_seed_model(None)
    report["evaluation"] = ev
    report["speedup_learned_over_plain"] = ev["learned"]["events_per_s"] / ev["plain"]["events_per_s"]
    report["efficiency_delta"] = ev["learned"]["quality"]["efficiency"] - ev["plain"]["quality"]["efficiency"]
    report["ghost_rate_delta"] = ev["learned"]["quality"]["ghost_rate"] - ev["plain"]["quality"]["ghost_rate"]
    log(json.dumps({k: report[k] for k in ("speedup_learned_over_plain", "efficiency_delta", "ghost_rate_delta")}))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1, default=float)
    chain.close()


def _generate_quality(args):
    from . import generator
    return generator.generate(args.quality_events, seed=505, mean_pileup=args.pileup, noise_rate=args.noise,
                              hit_efficiency=args.efficiency)


if __name__ == "__main__":
    main()
