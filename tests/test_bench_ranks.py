"""The multi-rank path of bench.py on CPU: two processes on the gloo backend
run the same rank plumbing (bench.Ranks) that the GPU bench runs on NCCL under
torchrun -- process group, barrier, maximum over ranks -- plus the per-rank
replica seeding and the reference arm's rank-0-only rule."""
import io
import multiprocessing as mp
import os
import socket
import sys
from contextlib import redirect_stdout

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    r = bench.Ranks("gloo", timeout_s=60)
    try:
        r.barrier()
        # Each rank's own "device time"; the bench reports the slowest rank.
        t = r.max_over_ranks(1.5 + rank)
        r.barrier()
        t2 = r.max_over_ranks(10.0 - rank)
        q.put((rank, r.world, t, t2, bench.box_seed("small", rank)))
    finally:
        r.close()


def test_two_gloo_ranks_reduce_max_and_seed_replicas():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == world for g in got)
    assert all(g[2] == 2.5 and g[3] == 10.0 for g in got)
    # Replicas: every rank integrates a differently seeded box.
    seeds = [g[4] for g in got]
    assert len(set(seeds)) == world
    from tholedipoleplugin_b200 import systems as S
    a, b = (S.config_small(seed=sd).positions for sd in seeds)
    assert not np.allclose(a, b)


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    r = bench.Ranks("gloo")
    assert (r.rank, r.world) == (0, 1)
    r.barrier()
    assert r.max_over_ranks(3.25) == 3.25
    r.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    # Under torchrun every rank launches --impl reference; ranks > 0 exit
    # without work or output.
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = bench.parse(["--impl", "reference", "--steps", "1", "--warmup", "0"])
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    assert buf.getvalue() == ""
