"""Dirichlet nodes (Microenvironment::add_dirichlet_node,
set_substrate_dirichlet_activation per voxel, apply_dirichlet_conditions:
BioFVM/BioFVM_microenvironment.cpp:218-323) and the 2-D LOD solver
(diffusion_decay_solver__constant_coefficients_LOD_2D, BioFVM/BioFVM_solvers.cpp:
1668-1832).

CPU: the oracle against the reference build -- node pinning on 3-D grids
with face and interior nodes, and 2-D steps for one substrate on ny == 1,
the shapes where the reference's 2-D loops stay on their lines (elsewhere they
step by S and nx values through the array, and for more than one substrate
the reference build crashed) -- plus two properties of the oracle.  GPU: the
sm_100a path against the oracle, bit for bit in FP64."""
import numpy as np
import pytest

import pyoracle
from pyoracle import Port
from bfvm import workloads as W


def _face_nodes(wl):
    """Every face voxel as a node: values from the face table, activation per
    substrate (what the reference holds after its faces are set)."""
    nx, ny, nz, S = wl.shape
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    face = (i == 0) | (i == nx - 1) | (j == 0) | (j == ny - 1) | (k == 0) | (k == nz - 1)
    vox = ((i * ny + j) * nz + k)[face].ravel()
    vals = wl.dirichlet_values.reshape(-1, S)[vox]
    act = np.tile(np.asarray(wl.dirichlet_active, np.uint8), (vox.size, 1))
    return dict((int(v), [vals[q].copy(), act[q].copy()]) for q, v in enumerate(vox))


def _node_arrays(nodes, S):
    vox = np.array(sorted(nodes), np.int32)
    vals = np.array([nodes[v][0] for v in vox], np.float64).reshape(-1, S)
    act = np.array([nodes[v][1] for v in vox], np.uint8).reshape(-1, S)
    return vox, vals, act


def _interior_nodes(wl, rng, count, nodes, ref=None):
    """Add `count` random nodes (faces included) and switch some activations
    off, on the reference (if given) and in `nodes` alike."""
    nx, ny, nz, S = wl.shape
    for v in rng.choice(nx * ny * nz, count, replace=False):
        val = rng.uniform(0.0, 60.0, S)
        act = nodes[int(v)][1] if int(v) in nodes else np.asarray(wl.dirichlet_active, np.uint8).copy()
        nodes[int(v)] = [val, act.copy()]
        if ref is not None:
            ref.add_dirichlet_node(int(v), val)
    for v in rng.choice(sorted(nodes), max(1, len(nodes) // 4), replace=False):
        s = int(rng.integers(0, S))
        on = bool(rng.integers(0, 2))
        nodes[int(v)][1][s] = 1 if on else 0
        if ref is not None:
            ref.set_node_activation(int(v), s, on)
    return nodes


# --------------------------------------------------------------------- CPU --

@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_nodes_match_reference_apply_dirichlet_conditions(seed):
    wl = W.small_random(910 + seed, n_agents=0, steps=1)
    rng = np.random.default_rng(seed)
    ref = pyoracle.Reference(wl, threads=1)
    try:
        nodes = _interior_nodes(wl, rng, 12, _face_nodes(wl), ref)
        ref.apply_dirichlet_conditions()
        want = ref.field()
    finally:
        ref.close()
    vox, vals, act = _node_arrays(nodes, wl.S)
    f = Port.dirichlet_nodes(wl.field0.copy(), wl.S, vox, vals, act)
    assert np.array_equal(f, want)


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_oracle_lod2d_matches_reference_build(seed):
    """One substrate, ny = nz = 1: every voxel is a face node; most are
    switched off so the sweeps have work."""
    wl = W.small_random(930 + seed, nx=30 + 7 * seed, ny=1, nz=1, S=1, n_agents=0, steps=5)
    wl.dirichlet_active[:] = 1
    rng = np.random.default_rng(seed)
    ref = pyoracle.Reference(wl, threads=1)
    n = wl.nx
    act = np.ones((n, 1), np.uint8)
    keep = set(rng.choice(n, 4, replace=False).tolist())
    try:
        for v in range(n):
            if v not in keep:
                ref.set_node_activation(v, 0, False)
                act[v, 0] = 0
        for _ in range(wl.steps):
            ref.lod2d()
        want = ref.field()
    finally:
        ref.close()
    f = wl.field0.copy()
    for _ in range(wl.steps):
        Port.lod2d_step(f, wl.nx, 1, 1, wl.D, wl.decay, wl.dt, wl.dx, np.arange(n), wl.dirichlet_values.reshape(n, 1),
                        act)
    assert not np.array_equal(f, wl.field0)
    assert np.array_equal(f, want)


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
def test_oracle_nodes_follow_remove_dirichlet_node():
    """remove_dirichlet_node clears the voxel's flag: the reference stops
    pinning it and the oracle, given the list without it, agrees."""
    wl = W.small_random(925, n_agents=0, steps=1)
    rng = np.random.default_rng(25)
    ref = pyoracle.Reference(wl, threads=1)
    try:
        nodes = _interior_nodes(wl, rng, 10, _face_nodes(wl), ref)
        for v in rng.choice(sorted(nodes), 15, replace=False):
            ref.remove_dirichlet_node(int(v))
            del nodes[int(v)]
        ref.apply_dirichlet_conditions()
        want = ref.field()
    finally:
        ref.close()
    vox, vals, act = _node_arrays(nodes, wl.S)
    assert np.array_equal(Port.dirichlet_nodes(wl.field0.copy(), wl.S, vox, vals, act), want)


@pytest.mark.skipif(not pyoracle.Reference.available(dropin=True), reason="drop-in library not built")
def test_dropin_lod2d_rejects_a_3d_mesh():
    """The drop-in's 2-D solver on a mesh deeper than one voxel prints its
    error and returns before any device work, densities unchanged."""
    wl = W.small_random(926, n_agents=0, steps=1)
    assert wl.nz > 1
    ref = pyoracle.Reference(wl, threads=1, dropin=True)
    try:
        ref.dropin_lod2d()
        assert np.array_equal(ref.field(), wl.field0)
    finally:
        ref.close()


def test_oracle_lod2d_conserves_mass_and_commutes():
    """No nodes and no decay: zero-flux sweeps keep each substrate's sum (to
    rounding).  The x and y solves of constant-coefficient lines commute, so
    a transposed square grid gives the transposed result (to rounding)."""
    rng = np.random.default_rng(7)
    nx, ny, S = 48, 48, 2
    f0 = rng.uniform(0.0, 40.0, nx * ny * S)
    D, decay = np.array([1e5, 3e3]), np.zeros(S)
    f = f0.copy()
    for _ in range(5):
        Port.lod2d_step(f, nx, ny, S, D, decay, 0.01, 20.0, [], np.zeros((0, S)))
    np.testing.assert_allclose(f.reshape(-1, S).sum(0), f0.reshape(-1, S).sum(0), rtol=1e-12)
    g0 = f0.reshape(nx, ny, S).transpose(1, 0, 2).copy().ravel()
    g = g0.copy()
    decay = np.array([0.1, 0.01])
    f = f0.copy()
    Port.lod2d_step(f, nx, ny, S, D, decay, 0.01, 20.0, [], np.zeros((0, S)))
    Port.lod2d_step(g, nx, ny, S, D, decay, 0.01, 20.0, [], np.zeros((0, S)))
    np.testing.assert_allclose(g.reshape(ny, nx, S).transpose(1, 0, 2), f.reshape(nx, ny, S), rtol=1e-12)


# --------------------------------------------------------------------- GPU --

def _oracle_2d(wl, steps, vox, vals, act, sources=False):
    f = wl.field0.copy()
    c1, c2, e2 = Port.workload_constants(wl)
    for _ in range(steps):
        if sources:
            Port.sources(f, wl.S, wl.agent_voxel, c1, c2, e2)
        Port.lod2d_step(f, wl.nx, wl.ny, wl.S, wl.D, wl.decay, wl.dt, wl.dx, vox, vals, act)
    return f


@pytest.mark.gpu
@pytest.mark.parametrize("shape,sources", [((37, 1, 1, 1), False), ((50, 40, 1, 3), True), ((200, 150, 1, 2), True),
                                           ((31, 257, 1, 1), False), ((300, 300, 1, 2), True)])
def test_gpu_lod2d_bitwise(shape, sources):
    from bfvm import Microenvironment

    nx, ny, nz, S = shape
    wl = W.small_random(950 + nx, nx=nx, ny=ny, nz=nz, S=S, n_agents=400 if sources else 0, steps=4, stack=True)
    rng = np.random.default_rng(nx)
    nodes = _interior_nodes(wl, rng, min(40, nx * ny // 3), _face_nodes(wl))
    vox, vals, act = _node_arrays(nodes, S)
    want = _oracle_2d(wl, wl.steps, vox, vals, act, sources)
    for sched in (1, 0):
        me = Microenvironment.from_workload(wl, agents="rates" if sources else "none")
        me.set_sweep_schedule(sched)
        # a voxel given twice keeps its last entry
        dup = np.concatenate([vox[:3], vox])
        dvals = np.concatenate([vals[:3] + 1.0, vals])
        dact = np.concatenate([act[:3], act])
        me.set_dirichlet_nodes(dup, dvals, dact)
        me.simulate_diffusion_decay_2d(wl.steps, sources=sources)
        got = me.download_field()
        me.close()
        assert np.array_equal(got, want), (shape, sched)


@pytest.mark.gpu
def test_gpu_nodes_apply_and_fp32_2d():
    from bfvm import BfvmError, Microenvironment

    wl = W.small_random(970, nx=64, ny=48, nz=1, S=2, n_agents=0, steps=6)
    rng = np.random.default_rng(3)
    nodes = _interior_nodes(wl, rng, 30, _face_nodes(wl))
    vox, vals, act = _node_arrays(nodes, wl.S)
    # apply_dirichlet_conditions alone
    me = Microenvironment.from_workload(wl)
    me.set_dirichlet_nodes(vox, vals, act)
    me.apply_dirichlet_conditions()
    assert np.array_equal(me.download_field(), Port.dirichlet_nodes(wl.field0.copy(), wl.S, vox, vals, act))
    me.close()
    # FP32 form of the 2-D step: FP32 storage, FP64 recurrence
    want = _oracle_2d(wl, wl.steps, vox, vals, act)
    me = Microenvironment.from_workload(wl, "fp32")
    me.set_dirichlet_nodes(vox, vals, act)
    me.simulate_diffusion_decay_2d(wl.steps)
    got = me.download_field().reshape(-1, wl.S)
    me.close()
    ref = want.reshape(-1, wl.S)
    assert np.all(np.abs(got - ref).max(axis=0) <= 1e-5 * np.abs(ref).max(axis=0))
    # a 3-D solve has no 2-D step
    me = Microenvironment(8, 8, 8, 20.0, 0.01, [1e3], [0.1])
    with pytest.raises(BfvmError):
        me.simulate_diffusion_decay_2d(1)
    with pytest.raises(BfvmError):
        me.set_dirichlet_nodes([8 ** 3], np.zeros((1, 1)))
    me.close()


# ------------------------------------------------ GPU, C++ drop-in (2-D) --

_dropin = pytest.mark.skipif(not pyoracle.Reference.available(dropin=True), reason="drop-in library not built")


@pytest.mark.gpu
@_dropin
@pytest.mark.parametrize("seed", [0, 1])
def test_gpu_dropin_lod2d_matches_reference_solver(seed):
    """bfvm_b200_lod2d_serial in the serial slot of the reference's own
    Microenvironment against the reference's 2-D solver, bit for bit, on the
    shapes where the reference solver is defined (one substrate, ny == 1)."""
    wl = W.small_random(940 + seed, nx=40 + 9 * seed, ny=1, nz=1, S=1, n_agents=0, steps=5)
    wl.dirichlet_active[:] = 1
    rng = np.random.default_rng(40 + seed)
    keep = set(rng.choice(wl.nx, 3, replace=False).tolist())
    cpu = pyoracle.Reference(wl, threads=1, dropin=True)
    gpu = pyoracle.Reference(wl, threads=1, dropin=True)
    try:
        for r in (cpu, gpu):
            for v in range(wl.nx):
                if v not in keep:
                    r.set_node_activation(v, 0, False)
        for _ in range(wl.steps):
            cpu.lod2d()
            gpu.dropin_lod2d()
        a, b = cpu.field(), gpu.field()
    finally:
        cpu.close()
        gpu.close()
    assert not np.array_equal(a, wl.field0)
    assert np.array_equal(a, b)


@pytest.mark.gpu
@_dropin
@pytest.mark.parametrize("shape", [(50, 40, 1, 3), (33, 70, 1, 2)])
def test_gpu_dropin_lod2d_nodes_and_sources_bitwise(shape):
    """General 2-D meshes through the drop-in: interior nodes added, switched
    and removed through the reference's API between steps, the agents'
    sources fused on the GPU; bit for bit against the oracle."""
    nx, ny, nz, S = shape
    wl = W.small_random(960 + nx, nx=nx, ny=ny, nz=nz, S=S, n_agents=300, steps=3, stack=True)
    rng = np.random.default_rng(nx)
    gpu = pyoracle.Reference(wl, threads=1, dropin=True)
    c1, c2, e2 = Port.workload_constants(wl)
    f = wl.field0.copy()
    try:
        assert gpu.L.ref_env_dropin_fuse_sources(gpu.h, 1, wl.dt) == 0
        nodes = _interior_nodes(wl, rng, 25, _face_nodes(wl), gpu)
        for phase in range(2):
            if phase == 1:
                nodes = _interior_nodes(wl, rng, 5, nodes, gpu)
                for v in rng.choice(sorted(nodes), 20, replace=False):
                    gpu.remove_dirichlet_node(int(v))
                    del nodes[int(v)]
            vox, vals, act = _node_arrays(nodes, S)
            for _ in range(wl.steps):
                gpu.dropin_lod2d()
                Port.sources(f, S, wl.agent_voxel, c1, c2, e2)
                Port.lod2d_step(f, nx, ny, S, wl.D, wl.decay, wl.dt, wl.dx, vox, vals, act)
        got = gpu.field()
    finally:
        gpu.close()
    assert not np.array_equal(got, wl.field0)
    assert np.array_equal(got, f)
