"""The multi-process side of bench.py on CPU: two gloo ranks on 127.0.0.1.

The solve does not shard (replicas only), so the only cross-rank steps are
the barriers and the max of the per-rank step time; rank 0 alone prints.
"""
import importlib.util
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = _bench()
        # each rank reports a different step time; every rank must see the largest
        got = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        dist.barrier()
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert got == [(0, 2.5), (1, 2.5)]


def test_max_over_ranks_single_process():
    assert _bench().max_over_ranks(3.25) == 3.25


def test_reference_arm_other_ranks_print_nothing(monkeypatch):
    bench = _bench()
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1"])
    out = io.StringIO()
    with redirect_stdout(out):
        rc = bench.run_reference_arm(bench.parse())
    assert rc == 0
    assert out.getvalue() == ""


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
