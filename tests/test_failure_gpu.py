"""The timeout path of the bounded device waits, driven without faulting the
GPU: a short wait limit (bfvm_set_wait_limit_ns) and a batch member whose
y sweep waits on an x-tile count that the host started far below zero
(bfvm_batch_inject_stall).  The waits run out, the kernel records the
timeout and finishes; bfvm_batch_synchronize returns BFVM_ERR_TIMEOUT once;
the other members of that step and every later step are bit-exact."""
import numpy as np
import pytest

from bfvm import Batch, Microenvironment
from bfvm import workloads as W
from bfvm._lib import BFVM_ERR_STATE, BFVM_ERR_TIMEOUT, BFVM_OK
from pyoracle import Port

pytestmark = pytest.mark.gpu

LIMIT_TEST_NS = 1_000_000       # 1 ms
LIMIT_DEFAULT_NS = 2_000_000_000


def _wls():
    return [W.small_random(7100 + i, nx=24 + 4 * i, ny=20 + 3 * i, nz=18 + 2 * i, S=2, n_agents=200, steps=1,
                           stack=True) for i in range(3)]


def test_stalled_member_times_out_and_the_batch_recovers():
    wls = _wls()
    b = Batch("fp64")
    b.set_schedule(mode=0, graph_steps=16)
    mes = [Microenvironment.from_workload(wl) for wl in wls]
    for me in mes:
        b.add(me)
    L = b.L
    assert L.bfvm_set_wait_limit_ns(0, LIMIT_TEST_NS) == BFVM_OK
    try:
        assert L.bfvm_batch_inject_stall(b.h, mes[1].h) == BFVM_OK
        b.step(1, sources=True)
        assert L.bfvm_batch_synchronize(b.h) == BFVM_ERR_TIMEOUT
        assert L.bfvm_batch_synchronize(b.h) == BFVM_OK  # the status was cleared
    finally:
        assert L.bfvm_set_wait_limit_ns(0, LIMIT_DEFAULT_NS) == BFVM_OK
    # members that were not stalled computed their step exactly
    for q in (0, 2):
        np.testing.assert_array_equal(mes[q].download_field(), Port.run(wls[q], nsteps=1))
    # every member, restarted from its initial field, steps bit-exactly again
    for wl, me in zip(wls, mes):
        me.upload_field(wl.field0)
    b.step(4, sources=True)
    b.synchronize()
    for wl, me in zip(wls, mes):
        np.testing.assert_array_equal(me.download_field(), Port.run(wl, nsteps=4))
    b.close()


def test_stall_needs_a_member_and_the_fused_schedule():
    wls = _wls()[:1]
    b = Batch("fp64")
    me = Microenvironment.from_workload(wls[0])
    other = Microenvironment.from_workload(wls[0])
    b.add(me)
    assert b.L.bfvm_batch_inject_stall(b.h, other.h) == BFVM_ERR_STATE
    b.set_schedule(mode=1)
    assert b.L.bfvm_batch_inject_stall(b.h, me.h) == BFVM_ERR_STATE
    b.close()
