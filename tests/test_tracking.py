"""Internalized-substrate tracking (Microenvironment_Options::
track_internalized_substrates_in_each_agent, BioFVM/BioFVM_microenvironment.h:477;
Basic_Agent::simulate_secretion_and_uptake, BioFVM/BioFVM_basic_agent.cpp:
520-532, 553-556; Basic_Agent::release_internalized_substrates, :310-333).

CPU: the oracle against the reference build (field and every agent's
amounts, bit for bit) and a mass-balance property of the oracle.  GPU: the
fused and the standalone source/sink stage, list changes, release and the
batched engine against the oracle, bit for bit in FP64."""
import numpy as np
import pytest

import pyoracle
from pyoracle import Port
from bfvm import workloads as W


def _vvox(wl):
    return wl.dx * wl.dx * wl.dx


def _e1(wl):
    return wl.net_export * wl.dt


def _oracle_run(wl, steps, internal=None):
    """steps x [tracked sources; LOD step] on the oracle; returns (field, internal)."""
    f = wl.field0.copy()
    c1, c2, e2 = Port.workload_constants(wl)
    internal = np.zeros((wl.n_agents, wl.S)) if internal is None else internal
    for _ in range(steps):
        Port.sources_tracked(f, wl.S, wl.agent_voxel, c1, c2, e2, _e1(wl), _vvox(wl), internal)
        Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    return f, internal


# --------------------------------------------------------------------- CPU --

@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
@pytest.mark.parametrize("seed,stack", [(1, False), (2, True), (3, True)])
def test_oracle_tracking_matches_reference_build(seed, stack):
    wl = W.small_random(800 + seed, n_agents=50, steps=3, stack=stack)
    assert np.any(wl.net_export != 0)
    ref = pyoracle.Reference(wl, threads=1)
    try:
        ref.set_tracking(True)
        assert np.array_equal(ref.agent_voxels(), wl.agent_voxel)
        for _ in range(wl.steps):
            ref.sources()
            ref.diffusion()
        want_f, want_in = ref.field(), ref.internalized()
    finally:
        ref.set_tracking(False)
        ref.close()
    f, internal = _oracle_run(wl, wl.steps)
    assert np.any(internal != 0)
    assert np.array_equal(f, want_f)
    assert np.array_equal(internal, want_in)


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
def test_oracle_release_matches_reference_build():
    wl = W.small_random(811, n_agents=40, steps=1, stack=True)
    rng = np.random.default_rng(5)
    amounts = rng.uniform(-3e4, 3e4, (wl.n_agents, wl.S))
    agents = rng.permutation(wl.n_agents)[:25]
    fraction = rng.uniform(0.0, 1.0, (agents.size, wl.S))
    ref = pyoracle.Reference(wl, threads=1)
    try:
        ref.set_internalized(amounts)
        ref.release(agents, fraction)
        want_f, want_in = ref.field(), ref.internalized()
    finally:
        ref.close()
    f = wl.field0.copy()
    internal = amounts.copy()
    Port.release_internalized(f, wl.S, agents, wl.agent_voxel, fraction, _vvox(wl), internal)
    assert np.array_equal(f, want_f)
    assert np.array_equal(internal, want_in)
    assert np.all(internal[agents] == 0)


def test_oracle_tracking_balances_mass():
    """Over source/sink stages alone, what leaves the field is what the agents
    internalize: sum(field) * V_voxel + sum(internal) is unchanged (to rounding)."""
    wl = W.small_random(820, nx=9, ny=8, nz=7, S=3, n_agents=59, steps=1, stack=True)
    f = wl.field0.copy()
    c1, c2, e2 = Port.workload_constants(wl)
    internal = np.zeros((wl.n_agents, wl.S))
    V = _vvox(wl)
    before = f.reshape(-1, wl.S).sum(0) * V
    for _ in range(4):
        Port.sources_tracked(f, wl.S, wl.agent_voxel, c1, c2, e2, _e1(wl), V, internal)
    after = f.reshape(-1, wl.S).sum(0) * V + internal.sum(0)
    np.testing.assert_allclose(after, before, rtol=1e-11)
    assert np.abs(internal).max() > 0


# --------------------------------------------------------------------- GPU --

@pytest.mark.gpu
@pytest.mark.parametrize("seed,stack", [(31, False), (32, True)])
def test_gpu_tracking_fused_and_standalone_bitwise(seed, stack):
    from bfvm import Microenvironment

    wl = W.small_random(seed, nx=21, ny=14, nz=9, S=3, n_agents=55, steps=4, stack=stack)
    want_f, want_in = _oracle_run(wl, wl.steps)
    # fused: the agents are applied inside the x sweep
    me = Microenvironment.from_workload(wl)
    me.set_track_internalized_substrates(True)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    assert np.array_equal(me.download_field(), want_f)
    assert np.array_equal(me.internalized_substrates(), want_in)
    me.close()
    # standalone stage, tracking switched on before the agent list exists
    me = Microenvironment.from_workload(wl, agents="none")
    me.set_track_internalized_substrates(True)
    me.set_agents_from_rates(wl.agent_voxel, wl.agent_volume, wl.secretion, wl.uptake, wl.saturation,
                             wl.net_export)
    for _ in range(wl.steps):
        me.simulate_cell_sources_and_sinks()
        me.simulate_diffusion_decay(1)
    assert np.array_equal(me.download_field(), want_f)
    assert np.array_equal(me.internalized_substrates(), want_in)
    me.close()


@pytest.mark.gpu
def test_gpu_tracking_constants_list_changes_and_release():
    """A list given as constants plus exports; a longer list keeps the amounts
    of the positions it shares and starts the new ones at zero; release and
    switching off and on again."""
    from bfvm import BfvmError, Microenvironment

    wl = W.small_random(41, nx=17, ny=12, nz=10, S=2, n_agents=45, steps=2, stack=True)
    c1, c2, e2 = Port.workload_constants(wl)
    e1 = _e1(wl)
    V = _vvox(wl)
    me = Microenvironment.from_workload(wl, agents="none")
    with pytest.raises(BfvmError):
        me.internalized_substrates()  # tracking off
    me.set_track_internalized_substrates(True)
    m = 30
    me.set_agents(wl.agent_voxel[:m], c1[:m], c2[:m], e2[:m])
    me.set_agent_exports(e1[:m])
    f = wl.field0.copy()
    internal = np.zeros((wl.n_agents, wl.S))
    for _ in range(2):
        me.simulate_diffusion_decay(1, sources=True)
        Port.sources_tracked(f, wl.S, wl.agent_voxel[:m], c1[:m], c2[:m], e2[:m], e1[:m], V, internal[:m])
        Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    assert np.array_equal(me.internalized_substrates(), internal[:m])
    # the whole list: positions < m keep their amounts, the rest start at zero
    me.set_agents(wl.agent_voxel, c1, c2, e2)
    got = me.internalized_substrates()
    assert np.array_equal(got[:m], internal[:m]) and np.all(got[m:] == 0)
    me.set_agent_exports(e1)
    for _ in range(2):
        me.simulate_cell_sources_and_sinks()
        me.simulate_diffusion_decay(1)
        Port.sources_tracked(f, wl.S, wl.agent_voxel, c1, c2, e2, e1, V, internal)
        Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    assert np.array_equal(me.download_field(), f)
    assert np.array_equal(me.internalized_substrates(), internal)
    # release a few agents, in an order that revisits stacked voxels
    rng = np.random.default_rng(3)
    agents = rng.permutation(wl.n_agents)[:20]
    fraction = rng.uniform(0.0, 1.0, (agents.size, wl.S))
    me.release_internalized_substrates(agents, fraction)
    Port.release_internalized(f, wl.S, agents, wl.agent_voxel, fraction, V, internal)
    assert np.array_equal(me.download_field(), f)
    assert np.array_equal(me.internalized_substrates(), internal)
    # written amounts are used; off and on again starts from zero
    me.set_internalized_substrates(internal * 2.0)
    assert np.array_equal(me.internalized_substrates(), internal * 2.0)
    me.set_track_internalized_substrates(False)
    me.set_track_internalized_substrates(True)
    assert np.all(me.internalized_substrates() == 0)
    me.close()


@pytest.mark.gpu
def test_gpu_tracking_fp32_within_tolerance():
    from bfvm import Microenvironment

    wl = W.small_random(51, nx=24, ny=16, nz=12, S=3, n_agents=58, steps=5, stack=True)
    want_f, want_in = _oracle_run(wl, wl.steps)
    me = Microenvironment.from_workload(wl, "fp32")
    me.set_track_internalized_substrates(True)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    got = me.internalized_substrates()
    me.close()
    # FP32 storage of the densities the agents read; the bookkeeping is FP64
    for s in range(wl.S):
        scale = np.abs(want_in[:, s]).max()
        if scale > 0:
            assert np.abs(got[:, s] - want_in[:, s]).max() <= 1e-5 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_gpu_tracking_in_batch_matches_alone(mode):
    from bfvm import Batch, Microenvironment

    wls = [W.small_random(60 + i, nx=10 + 3 * i, ny=9 + i, nz=7 + 2 * i, S=2, n_agents=40, steps=3, stack=True)
           for i in range(3)]
    batch = Batch("fp64")
    batch.set_schedule(mode=mode, graph_steps=1)
    mes = []
    for i, wl in enumerate(wls):
        me = Microenvironment.from_workload(wl)
        if i != 1:
            me.set_track_internalized_substrates(True)
        batch.add(me)
        mes.append(me)
    batch.step(3, sources=True)
    batch.synchronize()
    for i, (wl, me) in enumerate(zip(wls, mes)):
        want_f, want_in = _oracle_run(wl, 3)
        assert np.array_equal(me.download_field(), want_f), wl.name
        if i != 1:
            assert np.array_equal(me.internalized_substrates(), want_in), wl.name
    for me in mes:
        batch.remove(me)
        me.close()
    batch.close()
