"""The replica plumbing of bench.py on CPU: two gloo ranks agree on the max of
their device times and the sum of their samples, the timed region reduces that
way through bench.main, the reference arm prints from rank 0 only (the other
ranks do no work), and --gpus N never renders on one process: without torchrun
it starts N replicas, and a replica count that disagrees with WORLD_SIZE stops."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)


def _rank(rank: int, world: int, port: int, out):
    _env(rank, world, port)
    import bench

    d = bench.Dist(world)
    try:
        d.barrier()
        out.put((rank, d.max(10.0 + rank), d.sum(100.0 * (rank + 1)), d.rank, d.world))
        d.barrier()
    finally:
        d.close()


def _reference_rank(rank: int, world: int, port: int, out):
    _env(rank, world, port)
    import bench

    calls, printed = [], []
    # The CPU renderer is stood in for by a counter: only who runs it is under test.
    bench.cpu_sample = lambda scenes, budget_s: (calls.append(1) or (1e6, 0.5, "port", 1, [0]))
    bench.print = lambda *a, **k: printed.append(a[0])
    d = bench.Dist(world)

    class A:
        steps, warmup = 2, 1

    try:
        bench.run_reference(A, d, [], "test")
    finally:
        d.barrier()
        d.close()
    out.put((rank, len(calls), len(printed)))


def _main_rank(rank: int, world: int, port: int, out):
    """bench.main on a gloo rank, with the GPU renderer stood in for by a step
    that reports fixed stats: rank r takes 10 * (r + 1) ms per step."""
    _env(rank, world, port)
    import bench

    printed = []

    def fake_run_rtg(a, dist, scenes, desc):
        def step():
            return {"device_ms": 10.0 * (dist.rank + 1), "camera_samples": 1000.0, "rays": 10.0,
                    "shadow_rays": 5.0, "kernel_launches": 4}

        for _ in range(a.warmup):
            step()
        t = bench.timed_steps(dist, None, step, a.steps)
        if dist.rank == 0:
            printed.append((dist.world, t["t_max_ms"], t["samples"], t["rays"]))

    bench.run_rtg = fake_run_rtg
    bench.workload_scenes = lambda name: ([], name)
    rc = bench.main(["--gpus", str(world), "--steps", "3", "--warmup", "3"])
    out.put((rank, rc, printed))


def _run(target, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return sorted(q.get(timeout=10) for _ in range(world))


def test_two_gloo_ranks_reduce_time_by_max_and_samples_by_sum():
    for rank, mx, total, r, w in _run(_rank):
        assert (mx, total, w) == (11.0, 300.0, 2) and r == rank


def test_reference_arm_runs_on_rank_zero_only():
    assert _run(_reference_rank) == [(0, 3, 1), (1, 0, 0)]


def test_bench_main_on_two_ranks_reports_max_time_and_total_samples():
    assert _run(_main_rank) == [(0, 0, [(2, 60.0, 6000.0, 90.0)]), (1, 0, [])]


def test_gpus_n_without_torchrun_starts_n_replicas(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.delenv("WORLD_SIZE", raising=False)
    seen = []
    monkeypatch.setattr(bench.subprocess, "call", lambda cmd: seen.append(cmd) or 0)
    assert bench.main(["--gpus", "4", "--steps", "2"]) == 0
    cmd = seen[0]
    assert cmd[1:3] == ["-m", "torch.distributed.run"] and "--nproc-per-node=4" in cmd
    assert "127.0.0.1" in cmd and cmd[-4:] == ["--gpus", "4", "--steps", "2"]


def test_replica_count_must_match_world_size(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.delenv("WORLD_SIZE", raising=False)
    with pytest.raises(SystemExit):
        bench.Dist(8)
