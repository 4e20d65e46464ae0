"""The multi-process path of bench.py on the CPU: two ranks over gloo
(127.0.0.1 rendezvous) set up the group from the launcher's environment,
agree on the maximum of their timings, and the reference arm runs on rank 0
only (the other ranks return at once without work)."""

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank: int, world: int, port: int, q) -> None:
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, str(ROOT))
    import bench

    w, r, dist = bench.dist_setup("gloo", rank)
    # each rank's own step time; the job's time is the slowest rank's
    t = bench.max_over_ranks(10.0 + 3.0 * rank, dist, "cpu")
    dist.barrier()

    class Args:
        molecules, skin, steps, warmup = 64, 1.0, 1, 1

    # the reference arm: rank 0 alone works; here only the others call it
    ref = bench.run_reference(Args()) if rank != 0 else None
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, w, r, t, ref))


def test_two_gloo_ranks_agree_on_the_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2, 2] and [o[2] for o in out] == [0, 1]
    assert [o[3] for o in out] == [13.0, 13.0]
    assert out[1][4] == 0  # rank 1 of the reference arm: no work, success


def test_single_process_needs_no_group(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench

    for k in ("WORLD_SIZE", "RANK"):
        monkeypatch.delenv(k, raising=False)
    w, r, dist = bench.dist_setup("gloo")
    assert (w, r, dist) == (1, 0, None)
    assert bench.max_over_ranks(4.5, None, "cpu") == pytest.approx(4.5)
