"""bfvm_apply_sources_noalloc against the allocating path
(bfvm_set_agents + bfvm_apply_sources) on the same field and agents.

This file is collected last on purpose: the no-allocation entry point keeps
its sort scratch in one fixed device array of the library, so it is checked
both in a fresh process (run this file alone) and after every other test has
used the library in the same process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bfvm import Microenvironment  # noqa: E402
from bfvm._lib import BFVM_ERR_ARG, BFVM_OK  # noqa: E402

MAX_AGENTS = 262144  # the entry point's documented limit


def _agents(rng, nvox, n, S):
    voxel = rng.integers(-1, nvox, n).astype(np.int32)
    # A third of the agents share a handful of voxels, so runs of several
    # agents per voxel (applied in list order) are exercised.
    hot = rng.integers(0, nvox, 8)
    m = n // 3
    voxel[:m] = hot[rng.integers(0, 8, m)]
    rng.shuffle(voxel)
    active = (rng.random(n) < 0.9).astype(np.uint8)
    c1 = rng.random((n, S)) * 1e-3
    c2 = 1.0 + rng.random((n, S)) * 1e-2
    e2 = rng.random((n, S)) * 1e-4
    return voxel, active, c1, c2, e2


def _solve(shape, precision, field):
    nx, ny, nz, S = shape
    me = Microenvironment(nx, ny, nz, 20.0, 0.01, np.linspace(1e3, 1e5, S), np.linspace(0.01, 1.0, S),
                          precision=precision)
    me.upload_field(field)
    return me


def _noalloc(me, dev):
    voxel, active, c1, c2, e2 = dev
    st = me.L.bfvm_apply_sources_noalloc(me.h, int(voxel.numel()), C.c_void_p(voxel.data_ptr()),
                                         C.c_void_p(active.data_ptr()), C.c_void_p(c1.data_ptr()),
                                         C.c_void_p(c2.data_ptr()), C.c_void_p(e2.data_ptr()))
    assert st == BFVM_OK, st


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_apply_sources_two_calls(precision):
    """Two calls in a row on each path; the fields agree bit for bit after
    each call, in both precisions: both paths apply every voxel's agents in
    list order with the same FP64 operations and round once when storing."""
    shape = (48, 40, 36, 3)
    nx, ny, nz, S = shape
    rng = np.random.default_rng(20261203)
    field = rng.random(nx * ny * nz * S) * 10.0
    n = 60000
    voxel, active, c1, c2, e2 = _agents(rng, nx * ny * nz, n, S)

    ref = _solve(shape, precision, field)
    ref.set_agents(voxel, c1, c2, e2, active=active)
    new = _solve(shape, precision, field)
    dev = tuple(torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0") for a in (voxel, active, c1, c2, e2))
    torch.cuda.synchronize()
    for _ in range(2):
        ref.simulate_cell_sources_and_sinks()
        _noalloc(new, dev)
        a = ref.download_field()
        b = new.download_field()
        assert not np.array_equal(a, field)
        np.testing.assert_array_equal(b, a)
    ref.close()
    new.close()


def test_noalloc_limits():
    """Empty lists are a no-op; lists above the limit are rejected before any
    work is queued; the limit itself is accepted."""
    shape = (64, 64, 64, 1)
    rng = np.random.default_rng(7)
    field = rng.random(int(np.prod(shape)))
    me = _solve(shape, "fp64", field)
    L = me.L
    assert L.bfvm_apply_sources_noalloc(me.h, 0, None, None, None, None, None) == BFVM_OK
    assert L.bfvm_apply_sources_noalloc(me.h, MAX_AGENTS + 1, C.c_void_p(1), None, C.c_void_p(1),
                                        C.c_void_p(1), C.c_void_p(1)) == BFVM_ERR_ARG
    np.testing.assert_array_equal(me.download_field(), field)
    # Exactly the limit, compared with the allocating path.
    n = MAX_AGENTS
    voxel, active, c1, c2, e2 = _agents(rng, 64 ** 3, n, 1)
    ref = _solve(shape, "fp64", field)
    ref.set_agents(voxel, c1, c2, e2, active=active)
    ref.simulate_cell_sources_and_sinks()
    dev = tuple(torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0") for a in (voxel, active, c1, c2, e2))
    torch.cuda.synchronize()
    _noalloc(me, dev)
    np.testing.assert_array_equal(me.download_field(), ref.download_field())
    me.close()
    ref.close()


def test_noalloc_allocates_nothing_after_setup():
    """After one call with n = 0 (the set-up call, which loads the library's
    scratch array on the device), further calls leave the device's free
    memory unchanged: no allocation, however many agents."""
    shape = (40, 40, 40, 2)
    rng = np.random.default_rng(11)
    field = rng.random(int(np.prod(shape)))
    me = _solve(shape, "fp64", field)
    n = 100000
    voxel, active, c1, c2, e2 = _agents(rng, 40 ** 3, n, 2)
    dev = tuple(torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0") for a in (voxel, active, c1, c2, e2))
    assert me.L.bfvm_apply_sources_noalloc(me.h, 0, None, None, None, None, None) == BFVM_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        _noalloc(me, dev)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    me.close()
