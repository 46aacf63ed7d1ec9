"""The host side of bench.py on CPU: two gloo ranks on 127.0.0.1, the clock
record, and the reference arm's line.

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


def test_reference_arm_line_on_rank_zero():
    """`bench.py --impl reference` as launched for one GPU: the reference's
    own CPU path on the full cube200 workload (one warm-up and one timed LOD
    step here), one JSON line carrying the same metric, unit and workload as
    the CUDA arm, the cpu_baseline it describes and an e2e with no copies."""
    import json
    import subprocess

    bench = _bench()
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    proc = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, proc.stdout[-2000:]
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["config"]["workload"] == bench.WORKLOAD and line["dtype"] == "f64"
    assert line["steps"] == 1 and line["warmup"] == 1 and line["n_gpus"] == 1 and line["higher_is_better"]
    assert line["value"] > 0 and line["ms_per_step"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}



def test_clock_sampler_summary():
    """The clock record bench.py attaches to its line: median SM clock under
    load, the maximum clock, and which slowdown reasons were active in any
    sample, from nvidia-smi's CSV rows (malformed and N/A rows skipped)."""
    bench = _bench()
    cs = bench.ClockSampler(0)
    cs.lines = [
        "0, 1965, 1965, 701.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 980.2, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "garbage",
        "0, [N/A], 1965, 10.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    s = cs.summary()
    assert s == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    cs.lines = ["0, 1200, 1965, 500.0, 0x0, Active, Not Active, Active, Not Active"]
    assert cs.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    cs.lines = []
    assert cs.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
