#!/usr/bin/env python
"""VELO events/s on B200: the plain chain (SP decoding + clustering, phi sort,
search_by_triplet, three-hit filter, consolidation) over synthetic events.

Workload (one step): 100k generated events at nu = 7.6 (Poisson PVs, beam spot
sigma 0.04/45 mm, Poisson(25) tracks per PV, eta in [2, 5], 98% hit efficiency,
0.01 mm smear, 1-4 pixel clusters, 1e-5 noise), processed in slices of 16000 events,
the raw banks resident in HBM (1.3 GB per step, larger than L2).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  Under torchrun (N > 1) every rank processes its own events
(replicas, weak scaling) and the time is the max over ranks.  `--impl reference` times
the reference's own VELO kernels built as CPU C++ (oracle/_ref; the plain-C oracle if
that build is absent) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "VELO events/s on 1 B200, learned+batched vs plain at equal eff & ghost rate"
UNIT = "events/s"
N_MP = 26


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--events", type=int, default=100_000)
    p.add_argument("--slice", type=int, default=16_000)
    p.add_argument("--seed", type=int, default=2024)
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-learned", action="store_true", help="skip the learned-mode measurement")
    p.add_argument("--no-kalman", action="store_true", help="skip the velo_kalman_filter measurement")
    p.add_argument("--no-retina", action="store_true", help="skip the retina-cluster front-end measurement")
    p.add_argument("--no-mdf", action="store_true", help="skip the host MDF transpose measurement")
    p.add_argument("--no-workloads", action="store_true",
                   help="skip the small-slice, uneven-pileup and stress (nu 15, noise, inefficiency) measurements")
    p.add_argument("--e2e-slice", type=int, default=4000,
                   help="events per slice of the end-to-end pipeline (smaller slices overlap the copies better)")
    p.add_argument("--e2e-chains", type=int, default=3, help="chains (streams) of the end-to-end pipeline")
    return p.parse_args()


# ----------------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------------
from allen_b200.replicas import aggregate_rate, dist_env, max_over_ranks, rank_seed  # noqa: E402


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def generate_events(n_events, slice_size, seed, **gen):
    """Generated slices with their Monte Carlo truth (allen_b200.generator.Generated)."""
    from allen_b200 import generator
    return [generator.generate(min(slice_size, n_events - first), seed=seed, first_event=first, **gen)
            for first in range(0, n_events, slice_size)]


def generate_slices(n_events, slice_size, seed, pinned=False, **gen):
    return [g.raw for g in generate_events(n_events, slice_size, seed, **gen)]


def pin(s):
    from allen_b200.chain import pin_slice
    return pin_slice(s)


def kernel_bytes(n, raw_bytes, T, H, n4, n3_all, n3_out, TH, tracks_all):
    """Algorithmic bytes per launch of each kernel for one slice (no re-reads counted)."""
    return {
        "estimate_kernel": raw_bytes + 4 * (N_MP * n + 3 * n),
        "cluster_sort_kernel": raw_bytes + 4 * N_MP * n + 18 * H + 4 * (2 * N_MP * n + 1),
        "search_by_triplet_kernel": 18 * H + 8 * N_MP * n + T + 54 * n4 + 6 * (n3_all + n3_out) + 24 * n,
        "consolidate_kernel": 54 * n4 + 6 * n3_out + 16 * TH + 16 * TH + 4 * (2 * tracks_all + 1) + tracks_all
                              + 4 * 4 * (n + 1),
    }


def chain_bytes(n, raw_bytes, H, TH, tracks_all):
    """Algorithmic bytes of the chain per slice: raw in, sorted hits out, consolidated tracks out."""
    return raw_bytes + 18 * H + 2 * 4 * N_MP * n + 18 * TH + 4 * tracks_all + 4 * (tracks_all + 1) + tracks_all


def cpu_baseline(slices, geometry, target_s):
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import cpu_checkers
    kind = "reference" if cpu_checkers.available("ref") else "port"
    chk = cpu_checkers.load("ref" if kind == "reference" else "oracle")
    threads = os.cpu_count() or 1
    s = slices[0]
    cal_n = min(100, s.n_events)
    t1 = chk.time(s, geometry, cal_n, 1, 1)
    rate1 = cal_n / max(t1, 1e-6)
    slice_size = 500
    n_slices = max(threads, int(rate1 * threads * target_s / slice_size))
    wall = chk.time(s, geometry, slice_size, n_slices, threads)
    value = n_slices * slice_size / wall
    cpu_model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                cpu_model = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{n_slices * slice_size} events (slices of {slice_size} cycling over the first "
                      f"{s.n_events} events of the workload, one slice per thread at a time), {wall:.1f} s wall; "
                      f"single-thread {rate1:.0f} events/s; CPU: {cpu_model}"}


def mdf_measurement(seed: int, n_unique: int = 250, copies: int = 16, repeats: int = 3) -> dict:
    """Host raw-input path: MDF records to the VELO slice (allen_b200.mdf, all host threads)
    next to the reference's own transpose (its main/src/Transpose.cpp compiled as CPU C++,
    one slice on one thread as its MDF provider runs it), on the same stream.  Each record holds
    a generated event's VELO banks plus 822 banks of other subdetectors (16-300 payload bytes,
    about 130 KB), the bank count of the 2018 minbias sample beside its VELO banks."""
    from allen_b200 import generator, mdf, rawbanks
    rng = np.random.default_rng(seed)
    g = generator.generate(n_unique, seed=seed + 7).raw
    events = []
    for e in range(g.n_events):
        banks = [(t, g.bank_version, src, p) for (t, src, p) in rawbanks.banks_of_event(g, e)]
        sizes = rng.integers(16, 301, 822)
        blob = rng.bytes(int(sizes.sum()))
        types = rng.choice([9, 13, 21, 22, 32, 33, 64, 66], 822)
        srcs = rng.integers(0, 2048, 822)
        at = 0
        for t, sz, src in zip(types.tolist(), sizes.tolist(), srcs.tolist()):
            banks.append((t, 0, src, blob[at:at + sz]))
            at += sz
        banks.append((16, 7, 0, rng.bytes(40)))
        order = rng.permutation(len(banks))
        events.append([banks[i] for i in order])
    stream = mdf.write_records(events, checksum=False) * copies
    n = n_unique * copies
    ev = mdf.scan(stream)
    threads = os.cpu_count() or 1
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        mdf.transpose_vp(stream, ev, by_source_id=False, n_threads=threads)
        times.append(time.perf_counter() - t0)
    ours = n / statistics.median(times)
    out = {"value": round(ours, 1), "unit": UNIT, "threads": threads,
           "sample": f"{n} MDF records ({len(stream) / n / 1e3:.0f} KB each: {n_unique} generated events x {copies}), "
                     f"median of {repeats} transposes into the VELO slice"}
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import cpu_checkers
    if cpu_checkers.available("ref"):
        r = cpu_checkers.ref_transpose_vp(stream, n)
        if r["status"] == 0:
            out["reference"] = {"value": round(n / r["transpose_seconds"], 1), "unit": UNIT, "threads": 1,
                                "what": "transpose_events() on one slice, as one thread of its MDF provider"}
    return out


# ----------------------------------------------------------------------------------
# reference arm: the reference's CPU build on the host cores
# ----------------------------------------------------------------------------------
def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from allen_b200 import _native
    geometry = _native.default_geometry()
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import cpu_checkers
    kind = "reference" if cpu_checkers.available("ref") else "port"
    chk = cpu_checkers.load("ref" if kind == "reference" else "oracle")
    # bounded sample per step, sized from a single-thread calibration
    cal = generate_slices(200, 200, args.seed)[0]
    t1 = chk.time(cal, geometry, 100, 1, 1)
    rate1 = 100 / max(t1, 1e-6)
    slice_size = 500
    per_step = max(threads * slice_size, int(rate1 * threads * 8.0 / slice_size) * slice_size)
    per_step = min(per_step, args.events)
    s = generate_slices(per_step, per_step, args.seed)[0]
    for _ in range(args.warmup):
        chk.time(s, geometry, slice_size, per_step // slice_size, threads)
    times = [chk.time(s, geometry, slice_size, per_step // slice_size, threads) for _ in range(args.steps)]
    total = sum(times)
    value = args.steps * per_step / total
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"VELO plain chain, synthetic events nu=7.6, CPU sample of {per_step} events per step "
                               f"(slices of {slice_size}) of the 100k-event workload", "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{per_step} events per step, slices of {slice_size}, one slice per thread"},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------------
def run_ours(args):
    import torch
    from allen_b200 import replicas
    world, rank, local = replicas.init("nccl")
    if world == 1:
        torch.cuda.set_device(0)
    from allen_b200 import _native
    from allen_b200.chain import VeloChain, upload
    from allen_b200.rawbanks import super_pixels_per_event

    geometry = _native.default_geometry()
    seed = rank_seed(args.seed, rank)
    gens = generate_events(args.events, args.slice, seed)
    slices = [g.raw for g in gens]
    dev = [upload(s) for s in slices]
    sp_max = max(int(super_pixels_per_event(s).sum()) for s in slices)
    chain = VeloChain(geometry)
    chain.reserve(max(s.n_events for s in slices), sp_max + 64, max(s.raw.nbytes for s in slices) + 64)
    chain.set_timing(True)
    stream = torch.cuda.current_stream()

    # per-slice counts for the byte model (one untimed pass)
    counts = []
    for s, d in zip(slices, dev):
        chain.run(d, use_graph=True)
        t = chain.synchronize()
        out = chain.device_outputs()
        n = s.n_events
        cn = chain._fetch(out["dev_module_cluster_num"], 4 * N_MP * n, np.uint32)
        at = chain._fetch(out["dev_atomics_velo"], 4 * 3 * n, np.uint32).reshape(-1, 3)
        raw_bytes = s.raw.nbytes + s.offsets.nbytes + s.sizes.nbytes + s.types.nbytes
        counts.append(dict(n=n, raw_bytes=raw_bytes, T=t["host_total_number_of_velo_clusters"], H=int(cn.sum()),
                           n4=t["host_number_of_velo_tracks_at_least_four_hits"], n3_all=int(at[:, 0].sum()),
                           n3_out=t["host_number_of_three_hit_tracks_filtered"],
                           TH=t["host_accumulated_number_of_hits_in_velo_tracks"],
                           tracks_all=t["host_number_of_reconstructed_velo_tracks"]))

    def step():
        for d in dev:
            chain.run(d, use_graph=True)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    totals_last = chain.synchronize(check=False)
    ms = max_over_ranks(ms)
    replicas.barrier()
    events_step = sum(c["n"] for c in counts)
    value = aggregate_rate(world, events_step, args.steps, ms)

    # per-kernel durations of the last step (CUDA events captured inside the graphs)
    try:
        ktimes, runs = chain.kernel_times()
    except Exception as exc:  # keep the throughput line even without per-kernel timing
        print(f"kernel timing unavailable: {exc}", file=sys.stderr)
        ktimes, runs = {}, 0
    kb = [kernel_bytes(**c) for c in counts]
    per_kernel = {}
    for name, total_ms in ktimes.items():
        if name == "kalman_filter_kernel":
            continue  # not launched in the plain chain (its timing slot spans no kernel)
        avg = total_ms / max(runs, 1)
        entry = {"ms_per_launch": round(avg, 4), "share": None}
        if name in kb[0]:
            b = sum(k[name] for k in kb) / len(kb)
            entry["bytes_per_launch"] = int(b)
            entry["gbs"] = round(b / (avg / 1e3) / 1e9, 1) if avg > 0 else None
        per_kernel[name] = entry
    tot = sum(v["ms_per_launch"] for v in per_kernel.values())
    for v in per_kernel.values():
        v["share"] = round(v["ms_per_launch"] / tot, 4) if tot else None
    timed = [k for k in per_kernel if "bytes_per_launch" in per_kernel[k]]
    dominant = max(timed, key=lambda k: per_kernel[k]["ms_per_launch"]) if timed else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    ach = per_kernel[dominant]["gbs"] if dominant else None
    traffic = None
    instructions = None
    try:  # ncu DRAM bytes and warp instructions per event of the dominant kernel, scaled to one launch
        for line in open(os.path.join(REPO, "profiles", "dram_traffic.md")):
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if len(cells) >= 2 and cells[0] == dominant:
                traffic = int(float(cells[1]) * events_step / len(counts))
                if len(cells) >= 4:
                    instructions = float(cells[3]) * events_step / len(counts)
    except Exception:
        pass
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4) if ach else None, "traffic": traffic,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    # What bounds the dominant kernel instead: instruction issue.  One warp instruction per
    # scheduler per cycle, four schedulers per SM, at the SM clock sampled during the timed region.
    sm_mhz = clocks.summary().get("sm_mhz")
    if instructions and sm_mhz and dominant:
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        issue_peak = 4 * sms * sm_mhz * 1e6
        issue_ach = instructions / (per_kernel[dominant]["ms_per_launch"] / 1e3)
        roofline["issue"] = {"achieved": round(issue_ach / 1e9, 1), "peak": round(issue_peak / 1e9, 1),
                             "unit": "G warp instructions/s", "frac": round(issue_ach / issue_peak, 4),
                             "instructions_per_launch": int(instructions)}
    chain_gbs = sum(chain_bytes(c["n"], c["raw_bytes"], c["H"], c["TH"], c["tracks_all"]) for c in counts) \
        * args.steps / (ms / 1e3) / 1e9

    def timed(dev_list, use_graph=True):
        def once():
            for d in dev_list:
                chain.run(d, use_graph=use_graph)
        for _ in range(max(3, args.warmup)):
            once()
        torch.cuda.synchronize()
        replicas.barrier()
        t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for _ in range(args.steps):
            once()
        t_end.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(t_start.elapsed_time(t_end))

    def stage_ms():
        kt, kruns = chain.kernel_times()
        return {k: v / max(kruns, 1) for k, v in kt.items()}

    # The metric's comparison: learned + batched (the seed gate, persistent launches, CUDA graphs)
    # against the plain search, both batched and as per-stage launches (one CTA per event, no
    # graph), on the same events and timing rules; tracking quality of both modes over every
    # event of the step, counted on the GPU against the generator's truth.
    learned = None
    if not args.no_learned:
        from allen_b200 import seed_pruner
        from allen_b200.chain import check_contracts
        from allen_b200.validation import DeviceTruth, evaluate_device
        plain_cfg = chain.get_config()
        plain_stages = {k: v["ms_per_launch"] for k, v in per_kernel.items()}
        truths = [DeviceTruth(g) for g in gens]

        def quality():
            tot = dict(tracks=0, ghosts=0, reconstructible=0, reconstructed=0, clones=0)
            cand = searched = fallback = 0
            violations = 0  # the reference's output contracts, counted on the device
            for s_, d, t in zip(slices, dev, truths):
                chain.run(d, use_graph=True)
                slice_totals = chain.synchronize(check=False)
                violations += sum(check_contracts(chain.device_outputs(), slice_totals).values())
                r = evaluate_device(chain, t)
                for k in tot:
                    tot[k] += r[k]
                st = chain.seed_stats(s_.n_events)
                cand += int(st[:, 0].sum())
                searched += int(st[:, 1].sum())
                fallback += int((st[:, 2] == 2).sum())
            return {"efficiency": round(tot["reconstructed"] / max(tot["reconstructible"], 1), 6),
                    "ghost_rate": round(tot["ghosts"] / max(tot["tracks"], 1), 6),
                    "clone_rate": round(tot["clones"] / max(tot["reconstructed"] + tot["clones"], 1), 6),
                    "tracks": tot["tracks"], "reconstructible": tot["reconstructible"],
                    "candidates_searched_fraction": round(searched / max(cand, 1), 4),
                    "fallback_event_fraction": round(fallback / max(events_step, 1), 6),
                    "contract_violations": violations}

        q_plain = quality()
        seed_pruner.use_learned(chain)
        l_ms = timed(dev)
        l_stages = stage_ms()
        q_learned = quality()
        l_value = aggregate_rate(world, events_step, args.steps, l_ms)
        # the plain search as per-stage launches (the reference's way: one CTA per event, one
        # kernel after the other, no graph)
        chain.set_seed_model(None)
        chain.configure(search_threads=256, search_lanes_per_seed=0, search_ring_global=0, persistent=0,
                        search_hit_capacity=2560, cluster_stage_capacity=2560, cluster_blob_bytes=32768,
                        estimate_blob_bytes=24576, seed_window=0)
        p_ms = timed(dev, use_graph=False)
        chain.configure(**plain_cfg)
        p_value = aggregate_rate(world, events_step, args.steps, p_ms)
        plain_chain_ms = ms / args.steps / len(slices)
        search_plain = plain_stages.get("search_by_triplet_kernel", 0.0)
        learned = {
            "value": round(l_value, 1), "unit": UNIT,
            "ratio_vs_plain": round(l_value / value, 4),
            "ratio_vs_per_stage_plain": round(l_value / p_value, 4),
            "per_stage_plain": {"value": round(p_value, 1), "unit": UNIT,
                                "how": "one CTA per event (rings and staging in shared memory), kernels launched one "
                                       "by one without a CUDA graph, plain search"},
            "quality": {"events": events_step, "plain": q_plain, "learned": q_learned,
                        "efficiency_delta": round(q_learned["efficiency"] - q_plain["efficiency"], 6),
                        "ghost_rate_delta": round(q_learned["ghost_rate"] - q_plain["ghost_rate"], 6),
                        "clone_rate_delta": round(q_learned["clone_rate"] - q_plain["clone_rate"], 6),
                        "tolerance": 0.002,
                        "within_tolerance": bool(q_learned["efficiency"] - q_plain["efficiency"] >= -0.002 and
                                                 q_learned["ghost_rate"] - q_plain["ghost_rate"] <= 0.002)},
            "phase_split_ms_per_slice": {
                "plain": {"search": round(search_plain, 4), "chain": round(plain_chain_ms, 4)},
                "learned": {"seed_gate": round(l_stages.get("seed_gate_kernel", 0.0), 4),
                            "search": round(l_stages.get("search_by_triplet_kernel", 0.0), 4),
                            "chain": round(l_ms / args.steps / len(slices), 4)}},
            "amdahl": {"search_share_plain": round(search_plain / plain_chain_ms, 4) if plain_chain_ms else None,
                       "ceiling_if_the_search_were_free": round(plain_chain_ms / (plain_chain_ms - search_plain), 3)
                       if plain_chain_ms > search_plain else None},
            "model": "allen_b200/data/seed_pruner.npz", "config": seed_pruner.load_learned_config(),
        }
        del truths

    # velo_kalman_filter appended to the chain (the next stage of the reference sequence)
    kalman = None
    if not args.no_kalman:
        chain.set_kalman(True)
        for _ in range(max(3, args.warmup)):
            step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        k_start, k_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k_start.record(stream)
        for _ in range(args.steps):
            step()
        k_end.record(stream)
        torch.cuda.synchronize()
        k_ms = k_start.elapsed_time(k_end)
        k_ms = max_over_ranks(k_ms)
        try:
            kt, kruns = chain.kernel_times()
            kf_ms = kt.get("kalman_filter_kernel", 0.0) / max(kruns, 1)
        except Exception:
            kf_ms = None
        chain.set_kalman(False)
        # bytes of one launch: track and hit offsets, x y z of every track hit in, is_backward and
        # two 56-byte states per track out
        kf_bytes = sum(4 * (c["n"] + 1) + 4 * (c["tracks_all"] + 1) + 12 * c["TH"] + 113 * c["tracks_all"]
                       for c in counts) / len(counts)
        kf_gbs = kf_bytes / (kf_ms / 1e3) / 1e9 if kf_ms else None
        kalman = {"value": round(world * events_step * args.steps / (k_ms / 1e3), 1), "unit": UNIT,
                  "kernel": "kalman_filter_kernel", "ms_per_launch": round(kf_ms, 4) if kf_ms else None,
                  "bytes_per_launch": int(kf_bytes),
                  "roofline": {"bound": "hbm", "achieved": round(kf_gbs, 1) if kf_gbs else None, "peak": peak,
                               "unit": "GB/s", "frac": round(kf_gbs / peak, 4) if kf_gbs else None,
                               "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
                  "workload": "chain + velo_kalman_filter (beamline 0, 0) on the same events"}

    # the retina-cluster front end (Allen's default decoding) on the same generated events,
    # written as VPRetinaCluster banks (version 3, as the 2018 sample)
    retina = None
    if not args.no_retina:
        r_slices = generate_slices(args.events, args.slice, seed, raw_format=1, bank_version=3)
        r_dev = [upload(x) for x in r_slices]
        chain.reserve(max(x.n_events for x in r_slices), max(int(super_pixels_per_event(x).sum()) for x in r_slices) + 64,
                      max(x.raw.nbytes for x in r_slices) + 64)

        def r_step():
            for d in r_dev:
                chain.run(d, use_graph=True)

        for _ in range(max(3, args.warmup)):
            r_step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        r_start, r_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r_start.record(stream)
        for _ in range(args.steps):
            r_step()
        r_end.record(stream)
        torch.cuda.synchronize()
        r_ms = r_start.elapsed_time(r_end)
        r_ms = max_over_ranks(r_ms)
        try:
            rt, rruns = chain.kernel_times()
            r_kernels = {"retina_count_kernel": round(rt["estimate_kernel"] / max(rruns, 1), 4),
                         "retina_decode_kernel": round(rt["cluster_sort_kernel"] / max(rruns, 1), 4),
                         "search_by_triplet_kernel": round(rt["search_by_triplet_kernel"] / max(rruns, 1), 4)}
        except Exception:
            r_kernels = None
        r_events = sum(x.n_events for x in r_slices)
        retina = {"value": round(world * r_events * args.steps / (r_ms / 1e3), 1), "unit": UNIT,
                  "ms_per_launch": r_kernels,
                  "workload": f"the same {args.events} events per GPU as VPRetinaCluster banks (version 3) "
                              f"through the retina-cluster front end, slices of {args.slice}"}
        chain.set_front_end(False)
        del r_dev, r_slices

    # end to end through the public API from page-locked host buffers: HostPipeline copies each
    # slice in, runs the chain and copies the consolidated tracks out, two chains overlapping
    e2e = None
    if not args.no_e2e:
        from allen_b200.chain import HostPipeline
        # the same events, cut into the pipeline's slices
        e_slices = slices if args.e2e_slice == args.slice else generate_slices(args.events, args.e2e_slice, seed)
        pinned = [pin(s) for s in e_slices]
        e_sp_max = max(int(super_pixels_per_event(s).sum()) for s in e_slices)
        pipe = HostPipeline(geometry, n_chains=args.e2e_chains)
        pipe.reserve(max(s.n_events for s in e_slices), e_sp_max + 64, max(s.raw.nbytes for s in e_slices),
                     max(s.sizes.size for s in e_slices), max(s.types.size for s in e_slices))
        pipe.run(pinned)  # warm-up: graph capture per chain
        torch.cuda.synchronize()
        pipe.h2d_bytes = pipe.d2h_bytes = 0
        e_steps = max(1, min(args.steps, 3))
        t0 = time.perf_counter()
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_start.record(stream)
        # the steps stream through the pipeline back to back (a server's steady state): every
        # step's slices are copied in, reconstructed and their tracks copied out
        pipe.run(pinned * e_steps)
        torch.cuda.synchronize()
        e_end.record(stream)
        torch.cuda.synchronize()
        wall_ms = (time.perf_counter() - t0) * 1e3
        e_ms = max(e_start.elapsed_time(e_end), wall_ms)
        e_ms = max_over_ranks(e_ms)
        # the copy rates the pipeline is up against: one 256 MiB page-locked copy each way
        link = {}
        n_b = 1 << 28
        h_buf = torch.empty(n_b, dtype=torch.uint8, pin_memory=True)
        d_buf = torch.empty(n_b, dtype=torch.uint8, device="cuda")
        for direction, copy in (("h2d_gbs", lambda: d_buf.copy_(h_buf, non_blocking=True)),
                                ("d2h_gbs", lambda: h_buf.copy_(d_buf, non_blocking=True))):
            copy()
            torch.cuda.synchronize()
            b_start, b_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            b_start.record()
            for _ in range(4):
                copy()
            b_end.record()
            torch.cuda.synchronize()
            link[direction] = round(4 * n_b / (b_start.elapsed_time(b_end) / 1e3) / 1e9, 1)
        del h_buf, d_buf
        e2e = {"value": round(world * events_step * e_steps / (e_ms / 1e3), 1), "unit": UNIT,
               "h2d_bytes_per_step": int(pipe.h2d_bytes / e_steps), "d2h_bytes_per_step": int(pipe.d2h_bytes / e_steps),
               "steps": e_steps, "slice": args.e2e_slice, "chains": args.e2e_chains, "pinned_copy": link,
               "api": "allen_b200.chain.HostPipeline (chains on their own streams, one copy stream per direction, page-locked buffers; the steps' slices streamed back to back)"}
        pipe.close()

    # more workloads, same timing rules: the same events in slices of 4000 and 1000; uneven pileup
    # (nu uniform in 1..15, twice the events), also run as per-stage launches (one CTA per event,
    # rings in shared memory, no CUDA graph) for comparison; a stress workload (nu = 15, noise 1e-4
    # per pixel, 95 % hit efficiency; slices of 4000, since 16000 such events overflow the 32-bit
    # container offsets), also in learned mode
    workloads = None
    if not args.no_workloads:
        workloads = {}
        for name, gen, n_ev, slice_ in (("slice4000", dict(), args.events, 4000),
                                        ("slice1000", dict(), args.events, 1000),
                                        ("uneven_nu1-15", dict(pileup_min=1.0, pileup_max=15.0), 2 * args.events,
                                         args.slice),
                                        ("stress_nu15_noise1e-4_eff0.95",
                                         dict(mean_pileup=15.0, noise_rate=1e-4, hit_efficiency=0.95), args.events,
                                         4000)):
            # the slice lines re-slice the main line's events; the others have events of their own
            c_slices = generate_slices(n_ev, slice_, seed if name.startswith("slice") else seed + 17, **gen)
            c_dev = [upload(x) for x in c_slices]
            chain.reserve(max(x.n_events for x in c_slices), max(int(super_pixels_per_event(x).sum()) for x in c_slices) + 64,
                          max(x.raw.nbytes for x in c_slices) + 64)
            c_events = sum(x.n_events for x in c_slices)
            c_ms = timed(c_dev)
            c_flags = chain.synchronize(check=False)["device_flags"]
            entry = {"value": round(aggregate_rate(world, c_events, args.steps, c_ms), 1), "unit": UNIT,
                     "slice": slice_, "events_per_step": c_events * world,
                     "super_pixels_per_event": round(sum(int(super_pixels_per_event(x).sum()) for x in c_slices)
                                                     / c_events, 1),
                     "device_flags": c_flags}
            if name.startswith("uneven"):
                tuned = chain.get_config()
                chain.configure(search_threads=256, search_lanes_per_seed=0, search_ring_global=0, persistent=0,
                                search_hit_capacity=2560, cluster_stage_capacity=2560, cluster_blob_bytes=32768,
                                estimate_blob_bytes=24576)
                p_ms = timed(c_dev, use_graph=False)
                chain.configure(**tuned)
                entry["per_stage_launches"] = {
                    "value": round(aggregate_rate(world, c_events, args.steps, p_ms), 1), "unit": UNIT,
                    "how": "one CTA per event (rings and staging in shared memory), kernels launched one by one "
                           "without a CUDA graph"}
            if name.startswith("stress") and not args.no_learned:
                from allen_b200 import seed_pruner
                tuned = chain.get_config()
                seed_pruner.use_learned(chain)
                l_ms = timed(c_dev)
                fb = sc = db = 0
                for x, d in zip(c_slices, c_dev):
                    chain.run(d, use_graph=True)
                    chain.synchronize(check=False)
                    st = chain.seed_stats(x.n_events)
                    db += int(st[:, 0].sum())
                    sc += int(st[:, 1].sum())
                    fb += int((st[:, 2] == 2).sum())
                chain.set_seed_model(None)
                chain.configure(**tuned)
                l_val = aggregate_rate(world, c_events, args.steps, l_ms)
                entry["learned"] = {"value": round(l_val, 1), "unit": UNIT,
                                    "ratio_vs_plain": round(l_val / entry["value"], 4),
                                    "candidates_searched_fraction": round(sc / max(db, 1), 4),
                                    "fallback_event_fraction": round(fb / max(c_events, 1), 6)}
            workloads[name] = entry
            del c_dev, c_slices

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(slices, geometry, args.cpu_seconds)
    mdf_in = None
    if rank == 0 and not args.no_mdf:
        mdf_in = mdf_measurement(args.seed)

    if rank == 0:
        c0 = counts[0]
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {
                "workload": f"VELO plain chain (SP decode + masked clustering, phi sort, search_by_triplet, "
                            f"three-hit filter, consolidation), {args.events} synthetic events per GPU at nu=7.6 "
                            f"in slices of {args.slice}, raw banks resident in HBM",
                "events_per_step": events_step * world, "slice": args.slice,
                "l2": "inputs larger than L2 (raw banks of a step: %.2f GB)" % (sum(c['raw_bytes'] for c in counts) / 1e9),
                "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                "mode": "plain", "cuda_graph": True,
                "per_event": {"super_pixels": round(sp_max / max(s.n_events for s in slices), 1),
                              "clusters": round(c0["H"] / c0["n"], 1),
                              "tracks": round(c0["tracks_all"] / c0["n"], 1)},
            },
            "roofline": roofline,
            "chain_hbm_gbs": round(chain_gbs, 1),
            "kernels": per_kernel,
            # per slice: estimate, scan, clustering, search, scan, consolidation, totals
            # (+ the event order of persistent launches)
            "gpu_launches": sum(1 for v in per_kernel.values() if v["ms_per_launch"] > 0) * len(dev) * args.steps
                            + (len(dev) * args.steps if args.events and chain.get_config().get("persistent") else 0),
            "clocks": clocks.summary(),
            "learned": learned,
            "kalman": kalman,
            "retina": retina,
            "mdf": mdf_in,
            "workloads": workloads,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "device_flags": totals_last["device_flags"],
        }
        print(json.dumps(line), flush=True)
    chain.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
