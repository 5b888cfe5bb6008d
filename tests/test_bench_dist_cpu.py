"""bench.py's multi-rank timing on CPU ranks (gloo, world size 2): every rank
reports the slowest rank's step time, and the whole-job value counts the
units all ranks processed."""
import importlib.util
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, times, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = _bench()
    ms = b.max_over_ranks(times[rank], dist, device="cpu")
    q.put((rank, ms, b.whole_job_rows_per_s(world, 1000, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world, times = 2, [3.0, 5.5]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, value in got:
        assert ms == 5.5
        assert value == pytest.approx(2 * 1000 / 5.5e-3)


def test_single_rank_is_identity():
    b = _bench()
    assert b.max_over_ranks(4.0, None) == 4.0
