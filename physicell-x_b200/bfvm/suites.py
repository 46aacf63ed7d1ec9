"""Measurement suites beyond the single-solve benchmark: the batched uneven
workload, the serving stream, and the FP32-against-FP64 accuracy report.

The FP64 reference results here come from the library's FP64 path, which the
parity tests show to be bit-identical to the reference solver, so the FP32
errors reported are errors against the reference's own FP64 results.
"""
from __future__ import annotations

import time

import numpy as np

from . import workloads as W
from .batch import Batch
from .serve import Server, SolveRequest, poisson_arrivals, run_one_at_a_time
from .solver import Microenvironment


def _device_field(me, device):
    """The solve's densities as a float64 CUDA tensor [voxels, S] (reference layout)."""
    import torch

    nx, ny, nz, S = me.shape
    out = torch.empty((nx * ny * nz, S), dtype=torch.float64, device=torch.device("cuda", device))
    me.download_field_device(out.data_ptr())
    me.synchronize()
    return out


def field_errors(approx, ref):
    """Per-substrate errors of `approx` against `ref` (tensors [voxels, S]):
    normwise relative L-infinity max|a-r| / max|r| and relative L2."""
    d = (approx - ref).abs()
    r = ref.abs()
    linf = (d.amax(dim=0) / r.amax(dim=0).clamp_min(1e-300)).tolist()
    l2 = ((approx - ref).pow(2).sum(dim=0).sqrt() / ref.pow(2).sum(dim=0).sqrt().clamp_min(1e-300)).tolist()
    return {"linf_rel": linf, "l2_rel": l2}


def _timed_steps(me, steps, sources=True):
    import torch

    st = torch.cuda.ExternalStream(me.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    me.simulate_diffusion_decay(steps, sources=sources)
    e1.record(st)
    me.synchronize()
    return e0.elapsed_time(e1) * 1e-3


def uneven_batch(n_envs=256, steps=200, trial_steps=5, device=0, chain=0):
    """The uneven batch (n_envs solves, edges 24-128, 1-6 substrates, 0-20k
    agents): plain FP64 and plain FP32 one solve at a time, the FP64 batch and
    the FP32 batch (autotuned), each for `steps` LOD steps with sources; FP32
    errors against FP64 per solve and substrate.  `chain` is the FP32 form's
    recurrence (bfvm_set_fp64_chain); the FP64 runs keep the reference's
    arithmetic.  The FP32-batch over FP64-plain ratio is split into its
    precision factor (plain FP64 over plain FP32: half the bytes) and its
    batching factor (plain FP32 over the FP32 batch: launches and idle gaps
    of one-at-a-time solves removed)."""
    import torch

    wls = W.uneven_batch(n_envs, steps=steps)
    tot = sum(wl.n_values for wl in wls)
    out = {"envs": n_envs, "steps": steps, "values_per_step": tot, "fp32_chain": chain}
    # plain, one solve at a time (each synchronised before the next starts)
    ref = []
    for prec in ("fp64", "fp32"):
        t_plain = 0.0
        for wl in wls:
            me = Microenvironment.from_workload(wl, prec, device)
            if prec == "fp32":
                me.set_fp64_chain(chain)
            t_plain += _timed_steps(me, steps)
            if prec == "fp64":
                ref.append(_device_field(me, device))
            me.close()
        out[f"{prec}_plain"] = {"s": t_plain, "updates_per_s": tot * steps / t_plain}
    for prec in ("fp64", "fp32"):
        b = Batch(prec, device)
        mes = [Microenvironment.from_workload(wl, prec, device) for wl in wls]
        for me in mes:
            if prec == "fp32":
                me.set_fp64_chain(chain)
            b.add(me)
        tuned_ms = b.autotune(sources=True, trial_steps=trial_steps)
        bs = torch.cuda.ExternalStream(b.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(bs)
        b.step(steps, sources=True)
        e1.record(bs)
        b.synchronize()
        t = e0.elapsed_time(e1) * 1e-3
        res = {"s": t, "updates_per_s": tot * steps / t, "schedule": b.get_schedule(),
               "direct_threshold": b.get_direct_threshold(), "autotune_ms_per_step": tuned_ms}
        if prec == "fp64":
            res["bitwise_equal_to_plain"] = all(bool(torch.equal(_device_field(me, device), r))
                                                for me, r in zip(mes, ref))
        else:
            worst_inf, worst_l2 = 0.0, 0.0
            for me, r in zip(mes, ref):
                e = field_errors(_device_field(me, device), r)
                worst_inf = max(worst_inf, max(e["linf_rel"]))
                worst_l2 = max(worst_l2, max(e["l2_rel"]))
            res["max_linf_rel_vs_fp64"] = worst_inf
            res["max_l2_rel_vs_fp64"] = worst_l2
        b.close()
        for me in mes:
            me.close()
        out[f"{prec}_batch"] = res
    out["fp32_batch_over_fp64_plain"] = out["fp32_batch"]["updates_per_s"] / out["fp64_plain"]["updates_per_s"]
    out["decomposition"] = {
        "precision_fp64_plain_over_fp32_plain": out["fp64_plain"]["s"] / out["fp32_plain"]["s"],
        "batching_fp32_plain_over_fp32_batch": out["fp32_plain"]["s"] / out["fp32_batch"]["s"],
        "batching_fp64_plain_over_fp64_batch": out["fp64_plain"]["s"] / out["fp64_batch"]["s"],
        "bytes_ratio": 2.0,
    }
    return out


def single_accuracy(wl, device=0, mass_every=None):
    """One workload run to its full step count in FP64 and in FP32, with
    agent sources; per-substrate FP32 errors and both times, and the
    periodic FP64 mass-balance check: every `mass_every` steps (default a
    tenth of the run) both forms record their per-substrate field sums in
    FP64, and the FP32 records are compared with the FP64 ones."""
    out = {"workload": wl.name, "shape": list(wl.shape), "agents": wl.n_agents, "steps": wl.steps}
    every = mass_every or max(1, wl.steps // 10)
    fields, masses = {}, {}
    for prec in ("fp64", "fp32"):
        # one-time setup (module load, kernel attributes, occupancy queries)
        # on a throwaway solve of the same shape, so the timed run is warm
        # and still runs exactly wl.steps steps
        warm = Microenvironment.from_workload(wl, prec, device)
        _timed_steps(warm, 3)
        warm.close()
        me = Microenvironment.from_workload(wl, prec, device)
        me.set_mass_log(every, capacity=wl.steps // every + 1)
        t = _timed_steps(me, wl.steps)
        out[f"{prec}_s"] = t
        out[f"{prec}_updates_per_s"] = wl.n_values * wl.steps / t
        fields[prec] = _device_field(me, device)
        masses[prec] = me.mass_log()
        me.close()
    out.update(field_errors(fields["fp32"], fields["fp64"]))
    m32, m64 = masses["fp32"], masses["fp64"]
    out["mass_check"] = {"every_steps": every, "records": int(m64.shape[0]),
                         "max_rel_vs_fp64": (np.abs(m32 - m64) / np.maximum(np.abs(m64), 1e-300)).max(axis=0).tolist()}
    return out


def accuracy(names=("cube50", "cube200", "cube640"), device=0):
    gens = {"cube50": W.cube50, "cube200": W.cube200, "cube640": W.cube640}
    return [single_accuracy(gens[n](), device) for n in names]


def serve(n_requests=24, rate=1.0, seed=5, quantum=64, device=0, mode=2, direct_min=None, **request_kw):
    """A Poisson stream of requests (serving workload distribution unless
    overridden) through the FP32 server (batch schedule `mode`, and for mode
    2 the direct threshold), then the same stream through the plain FP64 path
    one request at a time."""
    arr = poisson_arrivals(n_requests, rate=rate, seed=seed)
    reqs = [SolveRequest(i, W.serve_request(i, seed=seed, **request_kw), float(arr[i])) for i in range(n_requests)]
    srv = Server("fp32", quantum=quantum, device=device, mode=mode, direct_min=direct_min)
    st = srv.run(reqs)
    srv.close()
    base = run_one_at_a_time(reqs, "fp64", device)
    s32, s64 = st.summary(), base.summary()
    return {"requests": n_requests, "rate_per_s": rate, "seed": seed, "quantum": quantum,
            "fp32_server": s32, "fp64_one_at_a_time": s64,
            "throughput_ratio": (s32["updates_per_s"] / s64["updates_per_s"]) if s64["updates_per_s"] else None,
            "request_sizes": [[r.workload.nx, r.workload.ny, r.workload.nz, r.workload.S, r.workload.steps,
                               r.workload.n_agents] for r in reqs]}


def timed(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0
