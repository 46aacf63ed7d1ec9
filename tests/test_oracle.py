"""CPU tests of the oracle: the C restatement (oracle/lod3d_oracle.c) against
the golden fixtures made by the reference build, against the reference
build itself when it is present, and against analytic known answers."""
import hashlib
import json
import os

import numpy as np
import pytest

from bfvm import workloads as W
from pyoracle import Port, Reference


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"), allow_pickle=False)


def _manifest(golden_dir):
    with open(os.path.join(golden_dir, "MANIFEST.json")) as fh:
        return json.load(fh)["cases"]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _run_port_from_fixture(g):
    nx, ny, nz, S = (int(v) for v in g["shape"])
    field = g["field0"].copy()
    dv_wl = W.Workload(name="fx", nx=nx, ny=ny, nz=nz, S=S, dx=float(g["dx"]), dt=float(g["dt"]),
                       steps=int(g["steps"]), D=g["D"], decay=g["decay"], dirichlet_active=g["active"],
                       face_values=g["face_values"], origin=(0, 0, 0), seed=0, agent_pos=np.zeros((0, 3)),
                       agent_volume=np.zeros(0), secretion=np.zeros((0, S)), uptake=np.zeros((0, S)),
                       saturation=np.zeros((0, S)), net_export=np.zeros((0, S)))
    dv = dv_wl.dirichlet_values
    for _ in range(int(g["steps"])):
        if g["voxel"].size:
            Port.sources(field, S, g["voxel"], g["c1"], g["c2"], g["e2"])
        Port.lod_step(field, (nx, ny, nz, S), g["D"], g["decay"], float(g["dt"]), float(g["dx"]), g["active"], dv)
    return field


def test_port_matches_small_goldens_bitwise(golden_dir):
    names = [n for n in _manifest(golden_dir) if n.startswith("small_")]
    assert len(names) >= 10
    for name in names:
        g = _load(golden_dir, name)
        out = _run_port_from_fixture(g)
        assert np.array_equal(out, g["final"]), name


def test_port_agent_constants_match_goldens(golden_dir):
    for name in [n for n in _manifest(golden_dir) if n.startswith("small_")]:
        g = _load(golden_dir, name)
        if g["voxel"].size == 0:
            continue
        dt = float(g["dt"])
        vv = float(g["dx"]) ** 3
        c1, c2, e2 = Port.agent_constants(dt, g["volume"], vv, g["secretion"], g["uptake"], g["saturation"],
                                          g["net_export"])
        assert np.array_equal(c1, g["c1"]) and np.array_equal(c2, g["c2"]) and np.array_equal(e2, g["e2"]), name


def test_port_matches_cube50_golden_hash(golden_dir):
    """cube50 (50^3 x 2, 2000 agents) for all 1000 steps: bit-identical to the
    reference's own solver (SHA-256 of the final field)."""
    g = _load(golden_dir, "cube50_1000")
    wl = W.cube50(steps=1000)
    assert _sha(wl.field0) == str(g["field0_sha"])
    assert _sha(wl.agent_voxel) == str(g["voxel_sha"])
    field = wl.field0.copy()
    c1, c2, e2 = Port.agent_constants(wl.dt, wl.agent_volume, wl.voxel_volume, wl.secretion, wl.uptake,
                                      wl.saturation, wl.net_export)
    assert _sha(c1) == str(g["c1_sha"]) and _sha(c2) == str(g["c2_sha"]) and _sha(e2) == str(g["e2_sha"])
    dv = wl.dirichlet_values
    for _ in range(wl.steps):
        Port.sources(field, wl.S, wl.agent_voxel, c1, c2, e2)
        Port.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv)
    assert _sha(field) == str(g["final_sha"])
    assert np.array_equal(field[g["sample_idx"]], g["sample_val"])


def test_port_matches_uneven_env_golden_hash(golden_dir):
    g = _load(golden_dir, "uneven_env_50")
    wl = W.uneven_env(index=7, steps=50)
    assert _sha(wl.field0) == str(g["field0_sha"])
    field = wl.field0.copy()
    c1, c2, e2 = Port.agent_constants(wl.dt, wl.agent_volume, wl.voxel_volume, wl.secretion, wl.uptake,
                                      wl.saturation, wl.net_export)
    dv = wl.dirichlet_values
    for _ in range(wl.steps):
        Port.sources(field, wl.S, wl.agent_voxel, c1, c2, e2)
        Port.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv)
    assert _sha(field) == str(g["final_sha"])


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_port_matches_cube640_line_goldens(golden_dir, axis):
    """cube640's substrates, coefficients and Gaussian agent ball on its
    640-voxel lines along each axis: the C restatement gives the reference's
    bits (the fixtures come from the reference build)."""
    wl = W.cube640_slab(axis)
    g = _load(golden_dir, f"{wl.name}_{wl.steps}")
    assert _sha(wl.field0) == str(g["field0_sha"])
    assert _sha(wl.agent_voxel) == str(g["voxel_sha"])
    c1, c2, e2 = Port.workload_constants(wl)
    assert _sha(c1) == str(g["c1_sha"]) and _sha(c2) == str(g["c2_sha"]) and _sha(e2) == str(g["e2_sha"])
    field = Port.run(wl)
    assert np.array_equal(field[g["sample_idx"]], g["sample_val"])
    assert _sha(field) == str(g["final_sha"])


# ---- analytic known answers (from the mathematics, not the reference) -------

def _uniform_wl(n, S, D, decay, value, steps=5, active=0):
    fv = np.ones((6, S))
    wl = W.make("uniform", n, n + 1, n + 2, S, 20.0, 0.01, steps, D, decay, [active] * S, fv, 0, 0,
                init_kind=[("const", value)] * S)
    return wl


def test_kat_uniform_zero_flux_decays_geometrically():
    """A uniform field under zero flux is an eigenvector of every sweep: each
    sweep divides it by (1 + dt*lambda/3), so a step divides by its cube."""
    D, lam = [1e5, 1e3], [0.1, 0.9]
    wl = _uniform_wl(9, 2, D, lam, 7.5)
    field = wl.field0.copy()
    for _ in range(wl.steps):
        Port.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    f = field.reshape(-1, 2)
    for d in range(2):
        expect = 7.5 / (1.0 + wl.dt * lam[d] / 3.0) ** (3 * wl.steps)
        np.testing.assert_allclose(f[:, d], expect, rtol=1e-12)


def test_kat_no_diffusion_is_pure_decay():
    rng = np.random.default_rng(0)
    wl = _uniform_wl(6, 1, [0.0], [0.3], 1.0)
    field = rng.uniform(0, 5, wl.n_values)
    f0 = field.copy()
    Port.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    np.testing.assert_allclose(field, f0 / (1 + wl.dt * 0.3 / 3) ** 3, rtol=1e-14)


def test_kat_dirichlet_only_converges_to_pinned_value():
    wl = W.make("dir", 8, 8, 8, 1, 20.0, 0.01, 1, [1e5], [0.0], [1], np.full((6, 1), 38.0), 0, 0,
                init_kind=[("const", 0.0)])
    field = wl.field0.copy()
    for _ in range(3000):
        Port.lod_step(field, wl.shape, wl.D, wl.decay, 0.5, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    np.testing.assert_allclose(field, 38.0, rtol=1e-9)


def test_kat_single_agent_closed_form():
    wl = W.small_random(5, n_agents=1)
    field = wl.field0.copy()
    c1, c2, e2 = Port.agent_constants(wl.dt, wl.agent_volume, wl.voxel_volume, wl.secretion, wl.uptake,
                                      wl.saturation, wl.net_export)
    v = int(wl.agent_voxel[0])
    before = field[v * wl.S:(v + 1) * wl.S].copy()
    Port.sources(field, wl.S, wl.agent_voxel, c1, c2, e2)
    np.testing.assert_array_equal(field[v * wl.S:(v + 1) * wl.S], (before + c1[0]) / c2[0] + e2[0])


def test_kat_zero_agents_equals_diffusion_only():
    wl = W.small_random(3, n_agents=0)
    a = wl.field0.copy()
    b = wl.field0.copy()
    Port.sources(a, wl.S, np.zeros(0, np.int32), np.zeros((0, wl.S)), np.zeros((0, wl.S)), np.zeros((0, wl.S)))
    Port.lod_step(a, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    Port.lod_step(b, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    assert np.array_equal(a, b)


def test_port_sweeps_independent_of_thread_count():
    wl = W.small_random(8, steps=3)
    a = Port.run(wl, threads=1)
    b = Port.run(wl, threads=4)
    assert np.array_equal(a, b)


# ---- against the reference build itself (only where its sources were built) --

needs_ref = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built (no reference sources)")


@needs_ref
@pytest.mark.parametrize("seed", [11, 12, 13, 14])
def test_port_matches_reference_build(seed):
    wl = W.small_random(seed, steps=5, stack=True)
    ref = Reference(wl)
    assert np.array_equal(ref.agent_voxels(), wl.agent_voxel)
    got = ref.run(wl.steps, solver=0, threads=2, sources_threads=1)
    assert np.array_equal(Port.run(wl), got)


@needs_ref
def test_reference_avx256d_equals_blocking_after_final_pin():
    """The reference's _AVX256D solver omits the final Dirichlet pin
    (BioFVM_solvers.cpp:1664-1665 vs :778); with it applied the two reference
    solvers agree bit for bit, so one oracle covers both."""
    wl = W.small_random(21, nx=13, ny=9, nz=11, S=3, n_agents=0, steps=1)
    r0 = Reference(wl)
    r1 = Reference(wl)
    for _ in range(4):
        r0.diffusion(solver=0, threads=2)
        r1.diffusion(solver=1, threads=2)
        r1.apply_dirichlet()
    assert np.array_equal(r0.field(), r1.field())
