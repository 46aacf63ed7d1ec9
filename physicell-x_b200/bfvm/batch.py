"""Batched engine: many resident solves advanced together, either by one fused
persistent launch per LOD step or by one launch per sweep over every member,
replayed from a CUDA graph (C ABI ``bfvm_batch_*``)."""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import BFVM_FP32, BFVM_FP64, BFVM_STEP_SOURCES, check


class Batch:
    """A set of :class:`bfvm.Microenvironment` solves stepped together.

    Members keep their own state and methods; a member gives the same result,
    bit for bit, as when it is stepped alone.
    """

    def __init__(self, precision="fp64", device=0):
        self.L = _lib.lib()
        h = C.c_void_p()
        check(self.L.bfvm_batch_create(BFVM_FP64 if precision == "fp64" else BFVM_FP32, int(device), C.byref(h)),
              "bfvm_batch_create")
        self.h = h
        self.precision = precision
        self.members = []

    def close(self):
        if getattr(self, "h", None):
            self.L.bfvm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return int(self.L.bfvm_batch_size(self.h))

    def add(self, me):
        check(self.L.bfvm_batch_add(self.h, me.h), "bfvm_batch_add")
        self.members.append(me)

    def remove(self, me):
        check(self.L.bfvm_batch_remove(self.h, me.h), "bfvm_batch_remove")
        self.members.remove(me)

    def step(self, nsteps=1, sources=False):
        check(self.L.bfvm_batch_step(self.h, int(nsteps), BFVM_STEP_SOURCES if sources else 0), "bfvm_batch_step")

    def synchronize(self):
        check(self.L.bfvm_batch_synchronize(self.h), "bfvm_batch_synchronize")

    @property
    def stream(self):
        return int(self.L.bfvm_batch_stream(self.h) or 0)

    def set_schedule(self, mode=0, yz_chunk=32, order=0, ctas_per_sm=0, graph_steps=16):
        """mode 0: one fused persistent launch per step; mode 1: one launch per
        sweep over every member; mode 2: mode 1 for the members under the
        direct threshold, the others stepped with their own kernels."""
        check(self.L.bfvm_batch_set_schedule(self.h, int(mode), int(yz_chunk), int(order), int(ctas_per_sm),
                                             int(graph_steps)), "bfvm_batch_set_schedule")

    def set_direct_threshold(self, values):
        """Mode 2: members of at least `values` voxel-substrate values step
        with their own kernels."""
        check(self.L.bfvm_batch_set_direct_threshold(self.h, C.c_longlong(int(values))),
              "bfvm_batch_set_direct_threshold")

    def get_direct_threshold(self):
        v = C.c_longlong()
        check(self.L.bfvm_batch_get_direct_threshold(self.h, C.byref(v)), "bfvm_batch_get_direct_threshold")
        return int(v.value)

    def get_schedule(self):
        v = [C.c_int() for _ in range(5)]
        check(self.L.bfvm_batch_get_schedule(self.h, *[C.byref(x) for x in v]), "bfvm_batch_get_schedule")
        return dict(zip(("mode", "yz_chunk", "order", "ctas_per_sm", "graph_steps"), (x.value for x in v)))

    def autotune(self, sources=False, trial_steps=5):
        """Pick the fastest schedule; returns its ms per step."""
        best = C.c_double()
        check(self.L.bfvm_batch_autotune(self.h, BFVM_STEP_SOURCES if sources else 0, int(trial_steps),
                                         C.byref(best)), "bfvm_batch_autotune")
        return best.value
