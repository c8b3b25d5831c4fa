"""The multi-GPU path on the host: replicas (every rank its own events, no exchange step),
run as two gloo ranks on CPU.  Each rank generates its event stream, reconstructs it with the
oracle, and the job combines the ranks' times the way bench.py does (max over ranks)."""
import os
import socket
import time

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import cpu_checkers
    from allen_b200 import _native, generator, replicas
    w, r, local = replicas.init("gloo", timeout_s=60)
    assert (w, r, local) == (world, rank, rank)
    seed = replicas.rank_seed(7, r)
    g = generator.generate(6, seed=seed, n_threads=1)
    t0 = time.perf_counter()
    out = cpu_checkers.load("oracle").run(g.raw, _native.default_geometry())
    ms = (time.perf_counter() - t0) * 1e3 + 100.0 * r  # rank 1 made the slower one on purpose
    job_ms = replicas.max_over_ranks(ms, device="cpu")
    replicas.barrier()
    np.savez(os.path.join(out_dir, f"rank{r}.npz"), seed=seed, ms=ms, job_ms=job_ms,
             raw=g.raw.raw, tracks=out["dev_offsets_all_velo_tracks"],
             rate=replicas.aggregate_rate(w, g.raw.n_events, 1, job_ms))
    replicas.finish()


def test_two_gloo_ranks_reconstruct_their_own_events_and_take_the_slowest_time(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"rank{r}.npz") for r in range(world))
    assert int(r0["seed"]) != int(r1["seed"])
    assert not np.array_equal(r0["raw"], r1["raw"])  # disjoint event streams
    assert r0["tracks"][-1] > 0 and r1["tracks"][-1] > 0
    slowest = max(float(r0["ms"]), float(r1["ms"]))
    assert float(r0["job_ms"]) == pytest.approx(slowest) and float(r1["job_ms"]) == pytest.approx(slowest)
    assert float(r0["rate"]) == pytest.approx(2 * 6 / (slowest / 1e3))


def test_single_process_needs_no_process_group():
    from allen_b200 import replicas
    assert replicas.max_over_ranks(3.5, device="cpu") == 3.5
    assert replicas.aggregate_rate(1, 100, 2, 1000.0) == 200.0
    assert replicas.rank_seed(5, 0) == 5 and replicas.rank_seed(5, 1) != replicas.rank_seed(5, 2)
