"""bfvm_step's CUDA-graph replay and the agent-delta upload
(bfvm_update_agents), each against the plain launches / a full re-upload."""
import numpy as np
import pytest

from bfvm import Microenvironment, kernel_launches
from bfvm import workloads as W
from pyoracle import Port

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("fused", [0, 1])
def test_graph_replay_equals_single_steps(precision, fused):
    """40 steps in one call (a 16-step graph replayed twice, after one
    uncaptured step, plus the rest launched directly) give the bits of 40
    one-step calls; the launch counter counts the replayed kernels."""
    wl = W.small_random(611, nx=40, ny=36, nz=30, S=2, n_agents=800, steps=40, stack=True)
    a = Microenvironment.from_workload(wl, precision=precision)
    b = Microenvironment.from_workload(wl, precision=precision)
    for me in (a, b):
        me.L.bfvm_set_fused_sources(me.h, fused)
    for _ in range(wl.steps):
        a.simulate_diffusion_decay(1, sources=True)
    before = kernel_launches()
    b.simulate_diffusion_decay(wl.steps, sources=True)
    b.synchronize()
    # sources and three sweeps per substrate group (two groups by default)
    per_step = (3 if fused else 4) * b.substrate_streams()
    assert kernel_launches() - before == wl.steps * per_step
    np.testing.assert_array_equal(b.download_field(), a.download_field())
    if precision == "fp64":
        np.testing.assert_array_equal(b.download_field(), Port.run(wl))


def test_graph_follows_agent_and_schedule_changes():
    """A new agent list, new constants and another sweep schedule between
    runs of steps each take effect (the graph is recaptured)."""
    wl = W.small_random(612, nx=48, ny=40, nz=36, S=3, n_agents=1500, steps=20, stack=True)
    expect = Port.run(wl, nsteps=20)
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(20, sources=True)
    np.testing.assert_array_equal(me.download_field(), expect)
    # second list: half the agents, another schedule
    c1, c2, e2 = Port.workload_constants(wl)
    half = wl.n_agents // 2
    me.set_agents(wl.agent_voxel[:half], c1[:half], c2[:half], e2[:half])
    me.set_sweep_schedule(2)
    me.simulate_diffusion_decay(20, sources=True)
    f = expect.copy()
    dv = wl.dirichlet_values
    for _ in range(20):
        Port.sources(f, wl.S, wl.agent_voxel[:half], c1[:half], c2[:half], e2[:half])
        Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv)
    np.testing.assert_array_equal(me.download_field(), f)
    me.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_update_agents_equals_full_reupload(precision):
    """Constants changed for a subset of the agents (the ones whose volume
    changed) through bfvm_update_agents give the bits of a full re-upload of
    the list with those constants."""
    wl = W.small_random(613, nx=36, ny=30, nz=28, S=3, n_agents=3000, steps=6, stack=True)
    c1, c2, e2 = Port.workload_constants(wl)
    rng = np.random.default_rng(5)
    idx = rng.choice(wl.n_agents, 300, replace=False).astype(np.int32)
    n1, n2, n3 = c1.copy(), c2.copy(), e2.copy()
    n1[idx] *= 1.5
    n2[idx] = 1.0 + (n2[idx] - 1.0) * 0.5
    n3[idx] += 1e-3
    a = Microenvironment.from_workload(wl, precision=precision)
    b = Microenvironment.from_workload(wl, precision=precision)
    a.simulate_diffusion_decay(3, sources=True)
    b.simulate_diffusion_decay(3, sources=True)
    a.set_agents(wl.agent_voxel, n1, n2, n3)
    b.update_agents(idx, n1[idx], n2[idx], n3[idx])
    a.simulate_diffusion_decay(3, sources=True)
    b.simulate_diffusion_decay(3, sources=True)
    np.testing.assert_array_equal(b.download_field(), a.download_field())
    np.testing.assert_array_equal(b.sample_agents(), a.sample_agents())
    if precision == "fp64":
        f = wl.field0.copy()
        dv = wl.dirichlet_values
        for step in range(6):
            k = (c1, c2, e2) if step < 3 else (n1, n2, n3)
            Port.sources(f, wl.S, wl.agent_voxel, *k)
            Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv)
        np.testing.assert_array_equal(b.download_field(), f)


def test_update_agents_rejects_bad_indices():
    wl = W.small_random(614, nx=10, ny=10, nz=10, S=1, n_agents=50, steps=1)
    me = Microenvironment.from_workload(wl)
    before = me.download_field()
    one = np.ones((1, 1))
    for bad in ([50], [-1], [3, 3]):
        with pytest.raises(Exception):
            me.update_agents(np.array(bad), np.ones((len(bad), 1)), np.ones((len(bad), 1)), np.ones((len(bad), 1)))
    me.update_agents(np.zeros(0, np.int32), one[:0], one[:0], one[:0])
    np.testing.assert_array_equal(me.download_field(), before)
    me.close()


def test_mass_log_records_every_k_steps_and_checks_fp32():
    """The periodic FP64 mass-balance record: one record per `every` steps,
    the same bits with graph replay and with single steps, equal to the
    oracle's per-substrate sums to rounding, and the FP32 form's records
    within 1e-6 of the FP64 form's."""
    wl = W.small_random(615, nx=44, ny=38, nz=30, S=3, n_agents=1200, steps=60, stack=True)
    logs = {}
    for prec, single in (("fp64", False), ("fp64", True), ("fp32", False)):
        me = Microenvironment.from_workload(wl, precision=prec)
        me.set_mass_log(every=20, capacity=8)
        if single:
            for _ in range(wl.steps):
                me.simulate_diffusion_decay(1, sources=True)
        else:
            me.simulate_diffusion_decay(25, sources=True)
            me.simulate_diffusion_decay(35, sources=True)
        logs[(prec, single)] = me.mass_log()
        me.close()
    a = logs[("fp64", False)]
    assert a.shape == (3, wl.S)
    np.testing.assert_array_equal(a, logs[("fp64", True)])
    f = wl.field0.copy()
    c1, c2, e2 = Port.workload_constants(wl)
    dv = wl.dirichlet_values
    for step in range(1, wl.steps + 1):
        Port.sources(f, wl.S, wl.agent_voxel, c1, c2, e2)
        Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv)
        if step % 20 == 0:
            np.testing.assert_allclose(a[step // 20 - 1], f.reshape(-1, wl.S).sum(axis=0), rtol=1e-12)
    np.testing.assert_allclose(logs[("fp32", False)], a, rtol=1e-6)


def test_per_kernel_timing_records():
    """bfvm_timing_read_kernels splits each recorded step into the source
    kernel and the three sweeps; bfvm_timing_read reports the source kernel
    with the x sweep; both clear the records; the results are unchanged."""
    wl = W.small_random(613, nx=40, ny=36, nz=30, S=2, n_agents=800, steps=4, stack=True)
    me = Microenvironment.from_workload(wl)
    me.timing_enable(True)
    for _ in range(2):
        me.simulate_diffusion_decay(1, sources=True)
    ms, n = me.timing_read_kernels()
    assert n == 2 and np.all(ms > 0.0)
    for _ in range(2):
        me.simulate_diffusion_decay(1, sources=True)
    xyz, n = me.timing_read()
    assert n == 2 and np.all(xyz > 0.0)
    assert me.timing_read_kernels()[1] == 0 and me.timing_read()[1] == 0
    me.timing_enable(False)
    np.testing.assert_array_equal(me.download_field(), Port.run(wl))
    me.close()
