#!/usr/bin/env python3
"""Benchmark of the BioFVM 3-D diffusion-decay LOD step with cell sources.

Metric: voxel*substrate updates per second per LOD step (N*S*steps / time).
Workload (one GPU): cube200 -- 200^3 voxels, dx=10 um, 4 substrates with
log-uniform D in [1e2,1e5] and decay in [1e-3,1] (substrate 0 Dirichlet 38
on all faces), 100,000 agents with uptake in [0,10] and secretion in [0,1],
FP64, dt=0.01 min.  One bench step = one LOD step: the standalone agent
source kernel, then the x, y and z sweeps (four kernels), with the
reference's arithmetic (bit-identical results).

  value  whole-job updates/s with the field resident in HBM (CUDA events on
         the solve's stream around one call of K steps, which replays the
         library's captured 16-step graph; max over ranks).  The field is
         256 MB, larger than the 126 MB L2, so no flush is needed between
         steps.
  e2e    the same metric through the C ABI with host buffers, as a
         PhysiCell loop drives it: every step sends the constants of the 1%
         of agents whose volume changed (bfvm_update_agents), every 10th
         step the whole moved agent list (bfvm_set_agents: voxels and
         constants, re-binned on the device), runs the LOD step and reads
         the densities at every agent's voxel back to the host.
  fp64_short_chain  the same resident step with the opt-in short FP64
         forward chain (bfvm_set_fp64_chain), which is within 1e-12 of the
         reference per voxel rather than bit-identical.
  roofline  of the slowest kernel of the step (the x sweep), from CUDA
         events around each kernel of up to 100 more steps called one at a
         time (launch gaps included): its algorithmic bytes (the field read
         and written once, its coefficients) over its time, against the
         measured HBM copy bandwidth; per_kernel lists the source kernel and
         the three sweeps, x_interval the source kernel and the x sweep
         together, step_frac the whole step (six field passes, coefficients
         and agents) over the step time.

Multi-GPU: one process per GPU, each advancing its own replica of the
workload (the solve does not shard; replicas only), value summed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "physicell-x_b200"))

METRIC = "voxel·substrate updates/s per LOD step"
UNIT = "voxel·substrate updates/s"
WORKLOAD = ("cube200: 200x200x200 voxels (dx=10 um), 4 substrates, 100000 agents, FP64, dt=0.01 min; "
            "one LOD step = agent sources (standalone kernel, timed with the x sweep) + x/y/z Thomas "
            "sweeps with Dirichlet pins, the reference's arithmetic (bit-identical)")

# DRAM bytes per launch of each timed kernel (dram__bytes_read.sum +
# dram__bytes_write.sum) from one-kernel ncu captures of this workload at the
# current kernels; profiles/sweeps_cube200_fp64.txt gives the commands and
# the raw figures.  Keys: (precision, kernel index 0=sources 1=x 2=y 3=z).
NCU_TRAFFIC = {
    ("fp64", 0): 56553472 + 1718528,
    ("fp64", 1): 273038080 + 199272448,
    ("fp64", 2): 271641856 + 199482880,
    ("fp64", 3): 271166208 + 195453184,
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--substrate-streams", type=int, choices=[1, 2], default=1,
                    help="bfvm_set_substrate_streams of the timed solve: 1 (default) one sequence of launches, 2 "
                         "the two halves of the substrates on two streams")
    ap.add_argument("--fp64-chain", type=int, choices=[0, 1, 2], default=0,
                    help="arithmetic of the timed solve (bfvm_set_fp64_chain): 0 the reference's (default)")
    ap.add_argument("--workload", choices=["cube200", "uneven_batch", "serve", "accuracy"], default="cube200",
                    help="cube200 (default): the single-solve benchmark line; the others run the batched, "
                         "serving and FP32-accuracy suites and print one JSON line each")
    ap.add_argument("--requests", type=int, default=24, help="serve: requests in the stream")
    ap.add_argument("--rate", type=float, default=1.0, help="serve: Poisson arrival rate (requests/s)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x, dist=None, device="cpu"):
    """Largest value of x over all ranks (the job's time is its slowest
    rank's); x itself when there is one process."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            pk = json.load(fh)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        self.lines = []
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            # nvidia-smi takes a moment to start: wait for its first sample so the
            # samples cover the whole timed region (at most 10 s).
            import select

            ready, _, _ = select.select([self.proc.stdout], [], [], 10.0)
            if ready:
                first = self.proc.stdout.readline()
                if first.strip():
                    self.lines.append(first)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines += [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline_sample(wl, budget_s=10.0):
    """Time the reference's own CPU path (oracle/_ref, all host threads) on a
    bounded sample of the workload -- as many LOD steps as fit in about
    budget_s seconds after one timed probe step; the C restatement if the
    reference build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    threads = pyoracle.max_threads()
    if pyoracle.Reference.available():
        ref = pyoracle.Reference(wl, threads=threads)
        t0 = time.perf_counter()
        ref.run(1, solver=0, threads=threads, sources_threads=threads, fetch=False)  # also does the factorization
        probe = time.perf_counter() - t0
        steps = int(max(2, min(200, budget_s / max(probe, 1e-3))))
        t0 = time.perf_counter()
        ref.run(steps, solver=0, threads=threads, sources_threads=threads, fetch=False)
        dt = time.perf_counter() - t0
        ref.close()
        kind = "reference"
    else:
        field = wl.field0.copy()
        c1, c2, e2 = pyoracle.Port.workload_constants(wl)
        dv = wl.dirichlet_values
        steps = 2
        t0 = time.perf_counter()
        for _ in range(steps):
            pyoracle.Port.sources(field, wl.S, wl.agent_voxel, c1, c2, e2)
            pyoracle.Port.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv, threads)
        dt = time.perf_counter() - t0
        kind = "port"
    out = {"value": wl.n_values * steps / dt, "unit": UNIT, "cores": threads, "kind": kind,
           "sample": f"{steps} LOD steps of cube200 (sources + _BLOCKING sweeps, OpenMP {threads} threads), "
                     f"{dt:.2f} s"}
    out.update(host_cpu())
    return out


def run_reference_arm(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    from bfvm import workloads as W

    wl = W.cube200()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    threads = pyoracle.max_threads()
    kind = "reference" if pyoracle.Reference.available() else "port"
    if kind == "reference":
        ref = pyoracle.Reference(wl, threads=threads)
        step = lambda: ref.run(1, solver=0, threads=threads, sources_threads=threads, fetch=False)  # noqa: E731
    else:
        field = wl.field0.copy()
        c1, c2, e2 = pyoracle.Port.workload_constants(wl)
        dv = wl.dirichlet_values

        def step():
            pyoracle.Port.sources(field, wl.S, wl.agent_voxel, c1, c2, e2)
            pyoracle.Port.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv, threads)
    for _ in range(max(1, args.warmup)):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = wl.n_values * args.steps / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": f"replicas x{args.gpus}",
                       "l2": "inputs larger than L2 (256 MB field per GPU), no flush",
                       "voxels": wl.n_voxels, "substrates": wl.S, "agents": wl.n_agents,
                       "solver": "diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING",
                       "sources": f"simulate_cell_sources_and_sinks, OpenMP {threads} threads"},
            "cpu_baseline": dict({"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                                  "sample": f"{args.steps} timed LOD steps of cube200 after "
                                            f"{max(1, args.warmup)} warm-up"}, **host_cpu()),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_suite(args):
    """The batched, serving and accuracy suites (one GPU, rank 0 only)."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA GPU")
    torch.cuda.set_device(local)
    from bfvm import suites

    if args.workload == "uneven_batch":
        r = suites.uneven_batch(device=local)
        line = {"metric": METRIC, "value": r["fp32_batch"]["updates_per_s"], "unit": UNIT, "n_gpus": 1,
                "higher_is_better": True, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "uneven_batch: 256 solves, edges 24-128, 1-6 substrates, 0-20k agents, "
                                       "200 LOD steps with sources; FP32 batch vs plain FP64 one solve at a time"},
                "suite": r}
    elif args.workload == "serve":
        r = suites.serve(n_requests=args.requests, rate=args.rate, device=local)
        line = {"metric": "serve p50/p99 time-to-completion (s) and voxel·substrate updates/s",
                "value": r["fp32_server"]["updates_per_s"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
                "dtype": "f32", "data": "synthetic",
                "p50_s": r["fp32_server"]["p50_s"], "p99_s": r["fp32_server"]["p99_s"],
                "config": {"workload": f"serve: {args.requests} requests, Poisson {args.rate}/s, edges 32-256, "
                                       "1-8 substrates, 100-10000 steps, 0-200k agents; FP32 continuous batching "
                                       "vs plain FP64 one request at a time"},
                "suite": r}
    else:
        r = suites.accuracy(device=local)
        line = {"metric": "FP32 relative error vs FP64 (per substrate, normwise L-infinity and L2)",
                "value": max(max(x["linf_rel"]) for x in r), "unit": "relative", "n_gpus": 1,
                "higher_is_better": False, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "cube50 1000 steps, cube200 500 steps, cube640 1000 steps, with sources"},
                "suite": r}
    print(json.dumps(line), flush=True)
    return 0


def host_cpu():
    """The host CPU: model name and physical cores (distinct core ids per
    socket in /proc/cpuinfo), for the CPU baseline's record."""
    model, cores = None, set()
    try:
        phys = core = None
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                k, _, v = ln.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name" and model is None:
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif not k and phys is not None and core is not None:
                    cores.add((phys, core))
                    phys = core = None
        if phys is not None and core is not None:
            cores.add((phys, core))
    except OSError:
        pass
    return {"cpu_model": model, "physical_cores": len(cores) or None, "logical_cpus": os.cpu_count()}


def time_resident(me, steps, stream):
    """Time `steps` resident LOD steps with sources on the solve's stream
    (CUDA events) as one call, as a caller runs many steps (the library
    replays its captured 16-step graph); then, on min(steps, 100) more steps
    called one at a time with the per-kernel timing records on, the split by
    kernel.  Returns (ms per step, per-kernel ms [4]: sources, x, y, z,
    kernel launches in the timed call)."""
    import torch

    from bfvm import kernel_launches

    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = kernel_launches()
    ev0.record(stream)
    me.simulate_diffusion_decay(steps, sources=True)
    ev1.record(stream)
    me.synchronize()
    torch.cuda.synchronize()
    launches = kernel_launches() - launches0
    ms_step = ev0.elapsed_time(ev1) / steps
    me.timing_enable(True)
    k_steps = min(steps, 100)
    for _ in range(k_steps):
        me.simulate_diffusion_decay(1, sources=True)
    me.synchronize()
    me.timing_enable(False)
    ms_sxyz, nrec = me.timing_read_kernels()
    return ms_step, ms_sxyz / max(1, nrec), launches


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload != "cube200":
        return run_suite(args)

    rank, world, local = dist_env()
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA GPU")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from bfvm import Microenvironment
    from bfvm import workloads as W

    wl = W.cube200()
    me = Microenvironment.from_workload(wl, precision=args.precision, device=local)
    me.set_fp64_chain(args.fp64_chain)
    me.set_substrate_streams(args.substrate_streams)
    stream = torch.cuda.ExternalStream(me.stream, device=torch.device("cuda", local))
    N, S, A = wl.n_voxels, wl.S, wl.n_agents

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- warm-up: at least W steps, and one call long enough (17) for the
    # library to capture its 16-step graph, so no capture falls in the timing
    me.simulate_diffusion_decay(max(3, args.warmup, 17), sources=True)
    me.synchronize()

    # ---- timed region (resident field) -------------------------------------
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms_step, per_kernel_ms, launches = time_resident(me, args.steps, stream)
    barrier()
    if dist is not None:
        ms_step = max_over_ranks(ms_step, dist, "cuda")
    value = world * N * S / (ms_step * 1e-3)

    # ---- roofline of the dominant kernel -------------------------------------
    # per kernel of the step: the standalone source kernel, then the sweeps;
    # algorithmic bytes: a sweep reads and writes the field once and reads its
    # axis' coefficients; the source kernel reads the agents (voxel id and
    # three constants per substrate) and the x-line offsets, and reads and
    # writes each agent's voxel values
    eb = 8 if args.precision == "fp64" else 4
    names = ["agent_sources", "sweep_x (+pins)", "sweep_y (+pins)", "sweep_z (+pins)"]
    field_bytes = 2 * N * S * eb
    coef_bytes = [3 * wl.nx * S * 8, 3 * wl.ny * S * 8, 3 * wl.nz * S * 8]
    agent_bytes = A * (4 + 3 * S * 8) + (wl.ny * wl.nz + 1) * 4
    alg = [agent_bytes + A * S * 2 * eb] + [field_bytes + coef_bytes[a] for a in range(3)]
    peak, peak_kind = load_peaks()
    step_bytes = 3 * field_bytes + sum(coef_bytes) + agent_bytes  # six field passes + coefficients + agents

    def roofline_of(kernel_ms, step_ms):
        dom = 1 + int(np.argmax(kernel_ms[1:]))  # the slowest sweep (the source kernel is a few % of the step)
        achieved = alg[dom] / (kernel_ms[dom] * 1e-3) / 1e9
        x_int = kernel_ms[0] + kernel_ms[1]
        return {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": NCU_TRAFFIC.get((args.precision, dom)),
                "algorithmic_bytes_per_launch": alg[dom],
                "per_kernel": [{"kernel": names[k], "ms": kernel_ms[k],
                                "GB/s": alg[k] / (kernel_ms[k] * 1e-3) / 1e9} for k in range(4)],
                # the source kernel and the x sweep together, as one interval
                "x_interval": {"ms": x_int, "GB/s": (alg[0] + alg[1]) / (x_int * 1e-3) / 1e9,
                               "frac": (alg[0] + alg[1]) / (x_int * 1e-3) / 1e9 / peak},
                "step_frac": (step_bytes / (step_ms * 1e-3) / 1e9) / peak}

    roofline = roofline_of(per_kernel_ms, ms_step)

    # ---- the opt-in short FP64 chain, same resident step ----------------------
    short = None
    if args.precision == "fp64" and args.fp64_chain == 0:
        me.set_fp64_chain(1)
        me.simulate_diffusion_decay(17, sources=True)  # recaptures the graph for the new chain
        me.synchronize()
        torch.cuda.synchronize()
        ms_short, kms_short, _ = time_resident(me, args.steps, stream)
        if dist is not None:
            ms_short = max_over_ranks(ms_short, dist, "cuda")
        me.set_fp64_chain(args.fp64_chain)
        short = {"value": world * N * S / (ms_short * 1e-3), "unit": UNIT, "ms_per_step": ms_short,
                 "roofline": roofline_of(kms_short, ms_short),
                 "arithmetic": "forward y = fma(RN(c1/d), y, v*RN(1/d)); within 1e-12 relative per voxel of the "
                               "reference (tests/test_fp64_chain_gpu.py), not bit-identical"}

    # ---- gradients of the field (compute_all_gradient_vectors), resident -----
    g_out = torch.empty(N * S * 3, dtype=torch.float64, device=torch.device("cuda", local))
    for _ in range(2):
        me.compute_all_gradient_vectors_device(g_out.data_ptr())
    ge0, ge1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g_reps = 20
    ge0.record(stream)
    for _ in range(g_reps):
        me.compute_all_gradient_vectors_device(g_out.data_ptr())
    ge1.record(stream)
    me.synchronize()
    g_ms = ge0.elapsed_time(ge1) / g_reps
    g_bytes = N * S * (eb + 3 * 8)
    gradients = {"ms": g_ms, "algorithmic_bytes": g_bytes, "GB/s": g_bytes / (g_ms * 1e-3) / 1e9,
                 "frac": g_bytes / (g_ms * 1e-3) / 1e9 / peak, "peak_source": peak_kind,
                 "what": "bfvm_compute_gradients_device: the field read once, [voxel][S][3] FP64 written"}
    del g_out

    # ---- e2e through the C ABI with host buffers -----------------------------
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    c1, c2, e2 = _agent_constants(wl)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    rng = np.random.Generator(np.random.PCG64(17))
    # two agent layouts: the workload's, and every agent moved to a neighbouring voxel
    moved = wl.agent_voxel.astype(np.int64) + rng.choice([-1, 1], A) * rng.choice([1, wl.nz, wl.ny * wl.nz], A)
    moved = np.where((moved >= 0) & (moved < N), moved, wl.agent_voxel).astype(np.int32)
    h_vox = [pin(wl.agent_voxel), pin(moved)]
    h_c1, h_c2, h_e2 = pin(c1), pin(c2), pin(e2)
    # eight rotating sets of the 1% of agents whose volume changed this step, with their new constants
    n_delta = max(1, A // 100)
    deltas = []
    for _ in range(8):
        idx = np.sort(rng.choice(A, n_delta, replace=False)).astype(np.int32)
        g = 1.0 + 0.01 * rng.random((n_delta, 1))
        deltas.append(tuple(pin(x) for x in (idx, c1[idx] * g, 1.0 + (c2[idx] - 1.0) * g, e2[idx])))
    h_out = pin(np.zeros((A, S)))
    from bfvm import _lib
    import ctypes as C

    L = me.L
    vp = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    move_every = 10

    def e2e_step(k):
        if k % move_every == 0:
            _lib.check(L.bfvm_set_agents(me.h, A, vp(h_vox[(k // move_every) % 2]), None, vp(h_c1), vp(h_c2),
                                         vp(h_e2)), "bfvm_set_agents")
        else:
            d = deltas[k % len(deltas)]
            _lib.check(L.bfvm_update_agents(me.h, n_delta, *[vp(x) for x in d]), "bfvm_update_agents")
        _lib.check(L.bfvm_step(me.h, 1, _lib.BFVM_STEP_SOURCES), "bfvm_step")
        _lib.check(L.bfvm_sample_agents(me.h, vp(h_out)), "bfvm_sample_agents")

    e2e_steps = max(move_every, args.e2e_steps or args.steps)
    e2e_steps -= e2e_steps % move_every
    for k in range(move_every):
        e2e_step(k)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        e2e_step(k)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if dist is not None:
        e2e_s = max_over_ranks(e2e_s, dist, "cuda")
    full_h2d = A * 4 + 3 * A * S * 8
    delta_h2d = n_delta * 4 + 3 * n_delta * S * 8
    h2d = (full_h2d + (move_every - 1) * delta_h2d) / move_every
    d2h = A * S * 8
    e2e = {"value": world * N * S / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "ms_per_step": e2e_s * 1e3,
           "path": f"bfvm_update_agents ({n_delta} agents, pinned host) on 9 of 10 steps, bfvm_set_agents (all "
                   f"{A} moved agents) on every 10th, + bfvm_step + bfvm_sample_agents (to pinned host), "
                   "wall clock"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_sample(wl)
        except Exception as exc:  # report, do not fail the GPU measurement
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "unavailable", "sample": repr(exc)}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD if args.fp64_chain == 0 and args.precision == "fp64"
                           else WORKLOAD.replace("FP64", args.precision.upper()).replace(
                               "the reference's arithmetic (bit-identical)", f"arithmetic chain {args.fp64_chain}"),
                           "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2 (256 MB field per GPU), no flush",
                           "voxels": N, "substrates": S, "agents": A,
                           "substrate_streams": args.substrate_streams},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "fp64_short_chain": short,
                "gradients": gradients,
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    return 0


def _agent_constants(wl):
    """The agents' (c1, c2, e2) for the e2e upload, computed by the library on
    the device with the arithmetic of Basic_Agent::set_internal_uptake_constants."""
    import ctypes as C

    import torch
    from bfvm import _lib

    n, S = wl.n_agents, wl.S
    dev = torch.device("cuda", torch.cuda.current_device())
    t_vol = torch.from_numpy(np.ascontiguousarray(wl.agent_volume, np.float64)).to(dev)
    t_r = [torch.from_numpy(np.ascontiguousarray(r, np.float64)).to(dev)
           for r in (wl.secretion, wl.uptake, wl.saturation, wl.net_export)]
    t_out = torch.empty((3, n, S), dtype=torch.float64, device=dev)
    rc = _lib.lib().bfvm_agent_constants_device(n, S, wl.dt, wl.dx ** 3, C.c_void_p(t_vol.data_ptr()),
                                                *[C.c_void_p(t.data_ptr()) for t in t_r],
                                                *[C.c_void_p(t_out[k].data_ptr()) for k in range(3)], None)
    _lib.check(rc, "bfvm_agent_constants_device")
    torch.cuda.synchronize()
    o = t_out.cpu().numpy()
    return o[0].copy(), o[1].copy(), o[2].copy()


if __name__ == "__main__":
    sys.exit(main())
