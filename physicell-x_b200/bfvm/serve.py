"""Serving loop: microenvironment solves arriving over time, admitted by a
device-memory budget and advanced together by the batched engine.

The reference has no server: PhysiCell parameter sweeps and dosing scenarios
run one process per solve.  Here a request is one BioFVM solve (grid, Thomas
coefficients, Dirichlet data, initial densities, agents, step count).  The loop
is continuous batching:

* a request that has arrived waits in a FIFO queue until its device memory
  (``bfvm_estimate_bytes``) fits in the budget next to the solves already
  resident, then it is created on the GPU, its densities and agents are
  uploaded and it joins the batch;
* each iteration advances every resident solve by a quantum of LOD steps
  (never past the end of any of them) with one ``bfvm_batch_step`` call --
  by default (batch mode 2) one launch per sweep over the members under
  2,097,152 voxel-substrate values and the larger ones stepped with their own
  tensor-memory kernels, all replayed from a CUDA graph;
* solves that finish in that quantum leave the batch at once and their
  densities are read back while the next quantum already runs, then their
  memory is freed, which admits the next requests;
* a request can be cancelled (``Server.cancel``, from any thread) while it
  waits or runs: between two quanta it is dropped from the queue, or leaves
  the batch and is freed, and is reported as cancelled.

A solve's result does not depend on what else is in the batch: members run the
same per-tile code as a solve stepped alone (tests check this bit for bit).
"""
from __future__ import annotations

import collections
import ctypes as C
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .batch import Batch
from .solver import Microenvironment
from .workloads import Workload


@dataclass
class SolveRequest:
    rid: int
    workload: Workload
    arrival: float = 0.0          # seconds after the stream starts
    keep_result: bool = False     # read the final densities back to the host


@dataclass
class SolveResult:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    n_values: int
    field: np.ndarray | None = None

    @property
    def latency(self):
        return self.finished - self.arrival

    @property
    def updates(self):
        return self.n_values * self.steps


def estimate_bytes(wl: Workload, precision: str) -> int:
    """Device bytes a request needs while resident (from the library's own
    allocation sizes, including a reference-layout transfer buffer)."""
    D = np.ascontiguousarray(wl.D, np.float64)
    lam = np.ascontiguousarray(wl.decay, np.float64)
    cfg = _lib.bfvm_config(wl.nx, wl.ny, wl.nz, wl.S, wl.dx, wl.dt, D.ctypes.data_as(C.POINTER(C.c_double)),
                           lam.ctypes.data_as(C.POINTER(C.c_double)),
                           _lib.BFVM_FP64 if precision == "fp64" else _lib.BFVM_FP32, 0)
    return int(_lib.lib().bfvm_estimate_bytes(C.byref(cfg), wl.n_agents))


def initial_field_device(wl: Workload, device: int = 0):
    """The request's initial densities, drawn on the device from the
    workload's per-substrate description with a generator seeded by the
    workload seed (same bits on every call), as a float64 tensor in the
    reference layout [x][y][z][S]."""
    import torch

    dev = torch.device("cuda", device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(wl.seed) * 7919 + 17)
    out = torch.empty((wl.n_voxels, wl.S), dtype=torch.float64, device=dev)
    for s, kind in enumerate(wl.init_kind):
        if kind[0] == "const":
            out[:, s] = float(kind[1])
        else:
            lo, hi = float(kind[1]), float(kind[2])
            out[:, s] = torch.rand(wl.n_voxels, generator=g, dtype=torch.float64, device=dev) * (hi - lo) + lo
    return out


def create_solve(wl: Workload, precision: str, device: int = 0) -> Microenvironment:
    """A resident solve for the request: coefficients, Dirichlet data, the
    device-drawn initial field and the agents (constants from their rates)."""
    import torch

    me = Microenvironment.from_workload(wl, precision=precision, device=device, upload=False)
    f0 = initial_field_device(wl, device)
    torch.cuda.synchronize(device)
    me.upload_field_device(f0.data_ptr())
    me.synchronize()
    del f0
    return me


@dataclass
class _Active:
    req: SolveRequest
    me: Microenvironment
    remaining: int
    admitted: float
    nbytes: int


@dataclass
class ServeStats:
    results: list = field(default_factory=list)
    wall: float = 0.0
    rejected: list = field(default_factory=list)
    cancelled: list = field(default_factory=list)  # (rid, steps done) of cancelled requests
    peak_bytes: int = 0
    quanta: int = 0

    def latencies(self):
        return np.array([r.latency for r in self.results])

    def summary(self):
        lat = self.latencies()
        upd = sum(r.updates for r in self.results)
        return {"requests": len(self.results), "rejected": len(self.rejected), "cancelled": len(self.cancelled),
                "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
                "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
                "wall_s": self.wall, "updates": upd, "updates_per_s": upd / self.wall if self.wall > 0 else None,
                "peak_bytes": self.peak_bytes, "quanta": self.quanta}


class Server:
    """Continuous-batching loop over one GPU (see the module docstring)."""

    def __init__(self, precision="fp32", budget_bytes=None, device=0, quantum=64, sources=True, mode=2,
                 yz_chunk=32, graph_steps=16, direct_min=None):
        import torch

        self.precision = precision
        self.device = device
        self.quantum = int(quantum)
        self.sources = sources
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(device)
            budget_bytes = int(free * 0.8)
        self.budget = int(budget_bytes)
        self.batch = Batch(precision, device)
        self.batch.set_schedule(mode=mode, yz_chunk=yz_chunk, graph_steps=graph_steps)
        if direct_min is not None:
            self.batch.set_direct_threshold(direct_min)
        self._cancel_lock = threading.Lock()
        self._cancelled = set()

    def close(self):
        self.batch.close()

    def cancel(self, rid):
        """Cancel request `rid` (safe from any thread).  It takes effect
        between two quanta: a waiting request is dropped, a running one leaves
        the batch, its solve is freed and its steps so far are reported in
        ``ServeStats.cancelled``.  The other solves' results do not change."""
        with self._cancel_lock:
            self._cancelled.add(rid)

    def _take_cancellations(self):
        with self._cancel_lock:
            out = set(self._cancelled)
            self._cancelled.clear()
        return out

    def run(self, requests, clock=time.perf_counter, poll=0.0005, on_quantum=None):
        """Serve the requests (arrival times relative to the start) and return
        the statistics; blocks until every admissible request has finished or
        was cancelled.  on_quantum(server, quanta) is called after each
        quantum is enqueued (a client can cancel requests from it)."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue = collections.deque()
        active: list[_Active] = []
        retiring: list[_Active] = []
        used = 0
        st = ServeStats()
        t0 = clock()
        cancelled = set()
        while pending or queue or active or retiring:
            cancelled |= self._take_cancellations()
            if cancelled:
                for dq in (pending, queue):
                    for req in [r for r in dq if r.rid in cancelled]:
                        dq.remove(req)
                        st.cancelled.append((req.rid, 0))
                        cancelled.discard(req.rid)
                for a in [a for a in active if a.req.rid in cancelled]:
                    # leaves between quanta: the batch orders the solve's
                    # later work (its release) after the steps already queued
                    self.batch.remove(a.me)
                    a.me.close()
                    used -= a.nbytes
                    active.remove(a)
                    st.cancelled.append((a.req.rid, int(a.req.workload.steps) - a.remaining))
                    cancelled.discard(a.req.rid)
                if not (pending or queue or active or retiring):
                    break
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            # admission: FIFO, as long as the head of the queue fits
            while queue:
                req = queue[0]
                need = estimate_bytes(req.workload, self.precision)
                if need > self.budget:
                    st.rejected.append(queue.popleft().rid)
                    continue
                if used + need > self.budget:
                    break
                queue.popleft()
                me = create_solve(req.workload, self.precision, self.device)
                self.batch.add(me)
                active.append(_Active(req, me, int(req.workload.steps), clock() - t0, need))
                used += need
                st.peak_bytes = max(st.peak_bytes, used)
            # one quantum for every resident solve; the ones that end in it leave
            # the batch now and are read back while the next quantum runs
            finished = []
            if active:
                k = min(self.quantum, min(a.remaining for a in active))
                self.batch.step(k, sources=self.sources)
                st.quanta += 1
                if on_quantum is not None:
                    on_quantum(self, st.quanta)
                for a in active:
                    a.remaining -= k
                finished = [a for a in active if a.remaining == 0]
                for a in finished:
                    self.batch.remove(a.me)
                active = [a for a in active if a.remaining > 0]
            for a in retiring:
                fld = a.me.download_field() if a.req.keep_result else None
                a.me.synchronize()
                st.results.append(SolveResult(a.req.rid, a.req.arrival, a.admitted, clock() - t0,
                                              int(a.req.workload.steps), a.req.workload.n_values, fld))
                a.me.close()
                used -= a.nbytes
            retiring = finished
            if not active and not retiring and not queue and pending:
                # idle until the next arrival
                while pending and pending[0].arrival > clock() - t0:
                    time.sleep(poll)
        self.batch.synchronize()
        st.wall = clock() - t0
        return st


def run_one_at_a_time(requests, precision="fp64", device=0, sources=True, clock=time.perf_counter):
    """The plain path the server is measured against: requests in arrival
    order, each solve created, stepped alone (``bfvm_step``) to its end, read
    back and freed before the next starts."""
    st = ServeStats()
    t0 = clock()
    for req in sorted(requests, key=lambda r: r.arrival):
        while clock() - t0 < req.arrival:
            time.sleep(0.0005)
        admitted = clock() - t0
        me = create_solve(req.workload, precision, device)
        me.simulate_diffusion_decay(int(req.workload.steps), sources=sources)
        fld = me.download_field() if req.keep_result else None
        me.synchronize()
        st.results.append(SolveResult(req.rid, req.arrival, admitted, clock() - t0, int(req.workload.steps),
                                      req.workload.n_values, fld))
        me.close()
    st.wall = clock() - t0
    return st


def poisson_arrivals(n, rate, seed):
    """n arrival times (seconds) of a Poisson process with the given rate."""
    rng = np.random.Generator(np.random.PCG64([seed, 77]))
    return np.cumsum(rng.exponential(1.0 / rate, n))
