"""The replica path of the benchmark on CPU (gloo, world size 2): the timed
region's max over ranks, the whole-job rate, and a rank that leaves before the
collective being reported on the host as an error within the process group's
timeout (no GPU involved)."""
from __future__ import annotations

import datetime
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, mode: str, q) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    try:
        if mode == "leave" and rank == 1:
            q.put((rank, "left", None))
            return
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        q.put((rank, ms, bench.job_rate(world, 1, ms)))
    except Exception as e:  # the peer left: the collective fails on the host
        q.put((rank, "error", type(e).__name__))
    finally:
        dist.destroy_process_group()


def _run(mode: str):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, a, b = q.get(timeout=120)
        out[rank] = (a, b)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_max_over_ranks_and_job_rate():
    out = _run("both")
    for rank in (0, 1):
        ms, rate = out[rank]
        assert ms == 15.0  # the slower rank's time, on every rank
        assert rate == pytest.approx(2 * 1e3 / 15.0)


def test_rank_that_leaves_is_reported_as_an_error():
    out = _run("leave")
    assert out[1][0] == "left"
    assert out[0][0] == "error"


def test_single_process_path():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.job_rate(1, 64, 100.0) == pytest.approx(640.0)
