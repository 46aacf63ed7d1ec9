"""GPU parity tests: the sm_100a path through the C ABI against the oracle.

FP64 bar: bit-identical to the reference (its golden fixtures, and the C
restatement on fresh seeded inputs).  FP32 bar: normwise relative L-inf
error per substrate, max|g - r| / max|r| <= 1e-5, against the FP64 oracle.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from bfvm import Microenvironment, kernel_launches
from bfvm import workloads as W
from pyoracle import Port

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"), allow_pickle=False)


def _fixture_solve(g, precision="fp64"):
    nx, ny, nz, S = (int(v) for v in g["shape"])
    wl = W.Workload(name="fx", nx=nx, ny=ny, nz=nz, S=S, dx=float(g["dx"]), dt=float(g["dt"]), steps=int(g["steps"]),
                    D=g["D"], decay=g["decay"], dirichlet_active=g["active"], face_values=g["face_values"],
                    origin=(0, 0, 0), seed=0, agent_pos=np.zeros((0, 3)), agent_volume=np.zeros(0),
                    secretion=np.zeros((0, S)), uptake=np.zeros((0, S)), saturation=np.zeros((0, S)),
                    net_export=np.zeros((0, S)))
    me = Microenvironment.from_workload(wl, precision=precision, upload=False)
    me.upload_field(g["field0"])
    if g["voxel"].size:
        me.set_agents(g["voxel"], g["c1"], g["c2"], g["e2"])
    return me, int(g["steps"])


def _normwise(got, ref, S):
    g = got.reshape(-1, S)
    r = ref.reshape(-1, S)
    return np.max(np.abs(g - r), axis=0) / np.maximum(np.max(np.abs(r), axis=0), 1e-300)


def test_small_goldens_bitwise(golden_dir):
    names = [n for n in json.load(open(os.path.join(golden_dir, "MANIFEST.json")))["cases"] if n.startswith("small_")]
    for name in names:
        g = _load(golden_dir, name)
        me, steps = _fixture_solve(g)
        me.simulate_diffusion_decay(steps, sources=True)
        out = me.download_field()
        me.close()
        bad = np.flatnonzero(out != g["final"])
        assert bad.size == 0, f"{name}: {bad.size} values differ, first {bad[:5]}"


def test_cube50_full_run_matches_reference_hash(golden_dir):
    """cube50 (50^3 x 2 substrates, 2000 agents), all 1000 LOD steps with
    sources: the final field is bit-identical to the reference's."""
    g = _load(golden_dir, "cube50_1000")
    wl = W.cube50(steps=1000)
    assert _sha(wl.field0) == str(g["field0_sha"])
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    out = me.download_field()
    assert np.array_equal(out[g["sample_idx"]], g["sample_val"])
    assert _sha(out) == str(g["final_sha"])


def test_cube200_and_uneven_env_match_reference_hash(golden_dir):
    for name, wl in (("cube200_10", W.cube200(steps=10)), ("uneven_env_50", W.uneven_env(index=7, steps=50))):
        g = _load(golden_dir, name)
        assert _sha(wl.field0) == str(g["field0_sha"])
        me = Microenvironment.from_workload(wl)
        me.simulate_diffusion_decay(wl.steps, sources=True)
        out = me.download_field()
        me.close()
        assert np.array_equal(out[g["sample_idx"]], g["sample_val"]), name
        assert _sha(out) == str(g["final_sha"]), name


@pytest.mark.parametrize("seed", list(range(200, 212)))
def test_random_cases_bitwise_against_port(seed):
    wl = W.small_random(seed, steps=4, stack=(seed % 2 == 0), agent_mode="gauss" if seed % 3 == 0 else "uniform")
    expect = Port.run(wl)
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    assert np.array_equal(me.download_field(), expect)


@pytest.mark.parametrize("shape", [(1, 1, 1, 1), (1, 7, 3, 2), (256, 3, 5, 1), (3, 256, 4, 2), (5, 4, 256, 1),
                                   (129, 65, 33, 3), (200, 200, 8, 4)])
def test_edge_shapes_bitwise(shape):
    nx, ny, nz, S = shape
    wl = W.small_random(7, nx=nx, ny=ny, nz=nz, S=S, n_agents=min(500, nx * ny * nz), steps=2, stack=True)
    expect = Port.run(wl)
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    assert np.array_equal(me.download_field(), expect)


def _screen_field(kind, n, rng):
    if kind == "signed":  # negative inputs: the screen fails, every line is checked
        return rng.uniform(-40.0, 40.0, n)
    # zeros, -0, subnormals and values just around 2^-960 (numerators the
    # Markstein quotient cannot take), mixed with ordinary values
    pool = np.array([0.0, -0.0, 5e-324, 1e-310, 2.0 ** -1000, 2.0 ** -960, 2.0 ** -959, 1e-300, 3.0, 1e-5])
    f = pool[rng.integers(0, pool.size, n)]
    return np.where(rng.random(n) < 0.5, f, rng.uniform(0.0, 40.0, n))


@pytest.mark.parametrize("kind", ["signed", "tiny"])
def test_exact_division_fallbacks_bitwise(kind):
    """Inputs that fail the exactness screen (negative values, zeros, -0,
    subnormals, values near 2^-960) take the checked path and, where a
    numerator needs it, IEEE division: bit-identical to the oracle under
    every sweep schedule and tensor-memory level, on a small case and on
    ones with enough tiles that every persistent CTA walks several (lines in
    TMEM, and past 256 partly resident in shared memory)."""
    rng = np.random.default_rng(4242)
    cases = (((23, 19, 17, 2), (0, 1, 2), (1,)), ((40, 300, 300, 1), (1, 2), (1,)),
             ((40, 200, 100, 1), (1, 2), (1, 2)), ((300, 40, 36, 1), (2,), (1,)))
    for shape, schedules, levels in cases:
        nx, ny, nz, S = shape
        wl = W.small_random(78, nx=nx, ny=ny, nz=nz, S=S, n_agents=300, steps=2, stack=True)
        wl._field0 = _screen_field(kind, wl.n_values, rng)
        expect = Port.run(wl)
        for sched in schedules:
            for level in levels:
                me = Microenvironment.from_workload(wl)
                me.set_sweep_schedule(sched)
                me.set_sweep_tmem(level)
                me.simulate_diffusion_decay(wl.steps, sources=True)
                got = me.download_field()
                me.close()
                assert np.array_equal(got.view(np.int64), expect.view(np.int64)), (kind, shape, sched, level)


def test_constants_from_rates_equal_precomputed():
    wl = W.small_random(31, n_agents=300, steps=3, stack=True)
    c1, c2, e2 = Port.workload_constants(wl)
    a = Microenvironment.from_workload(wl)  # constants computed on the device
    b = Microenvironment.from_workload(wl, agents="none")
    b.set_agents(wl.agent_voxel, c1, c2, e2)
    for me in (a, b):
        me.simulate_diffusion_decay(wl.steps, sources=True)
    assert np.array_equal(a.download_field(), b.download_field())


def test_standalone_sources_then_diffusion_equals_fused():
    wl = W.small_random(32, n_agents=400, steps=3, stack=True)
    expect = Port.run(wl)
    me = Microenvironment.from_workload(wl)
    for _ in range(wl.steps):
        me.simulate_cell_sources_and_sinks()
        me.simulate_diffusion_decay(1, sources=False)
    assert np.array_equal(me.download_field(), expect)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fused_and_standalone_sources_give_the_same_bits(precision):
    """bfvm_step with sources: the agents inside the x sweep or with the
    standalone kernel ahead of it (the default), under every sweep schedule,
    with stacked Gaussian agents and a grid large enough for many tiles."""
    wl = W.small_random(37, nx=90, ny=120, nz=100, S=2, n_agents=30000, steps=3, agent_mode="gauss", stack=True)
    outs = []
    for fused in (True, False):
        for sched in (0, 1, 2):
            me = Microenvironment.from_workload(wl, precision)
            me.set_fused_sources(fused)
            me.set_sweep_schedule(sched)
            me.simulate_diffusion_decay(wl.steps, sources=True)
            outs.append(me.download_field())
            me.close()
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    if precision == "fp64":
        assert np.array_equal(outs[0], Port.run(wl))


def test_sources_only_matches_port_and_sampling():
    wl = W.small_random(33, n_agents=250, steps=1, stack=True)
    c1, c2, e2 = Port.workload_constants(wl)
    field = wl.field0.copy()
    Port.sources(field, wl.S, wl.agent_voxel, c1, c2, e2)
    me = Microenvironment.from_workload(wl)
    me.simulate_cell_sources_and_sinks()
    got = me.download_field()
    assert np.array_equal(got, field)
    samp = me.sample_agents()
    expect = field.reshape(-1, wl.S)[wl.agent_voxel]
    assert np.array_equal(samp, expect)


def test_inactive_and_outside_agents_are_skipped():
    wl = W.small_random(34, n_agents=100, steps=2)
    c1, c2, e2 = Port.workload_constants(wl)
    vox = wl.agent_voxel.copy()
    vox[::7] = -1
    active = np.ones(wl.n_agents, np.uint8)
    active[::5] = 0
    field = wl.field0.copy()
    dv = wl.dirichlet_values
    for _ in range(wl.steps):
        Port.sources(field, wl.S, vox, c1, c2, e2, active=active)
        Port.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv)
    me = Microenvironment.from_workload(wl, agents="none")
    me.set_agents(vox, c1, c2, e2, active=active)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    assert np.array_equal(me.download_field(), field)


def test_runs_are_deterministic_and_launch_shape_independent():
    wl = W.small_random(35, nx=70, ny=45, nz=90, S=2, n_agents=3000, steps=3, agent_mode="gauss")
    outs = []
    for launch in (None, (8, 16, 7), (64, 64, 64), (32, 32, 256), (16, 32, 40)):
        me = Microenvironment.from_workload(wl)
        if launch:
            me.set_launch(*launch)
        me.simulate_diffusion_decay(wl.steps, sources=True)
        outs.append(me.download_field())
        me.close()
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


def test_persistent_schedule_many_tiles_bitwise():
    """Enough tiles that every CTA of the persistent sweeps walks several of
    them (both slot orders, refills under the back substitution), with
    stacked agents and internalized-substrate tracking: FP64 equals the
    oracle bit for bit, and both schedules give the same bits in FP64 and FP32."""
    wl = W.small_random(36, nx=40, ny=300, nz=300, S=2, n_agents=20000, steps=2, agent_mode="gauss", stack=True)
    c1, c2, e2 = Port.workload_constants(wl)
    f = wl.field0.copy()
    internal = np.zeros((wl.n_agents, wl.S))
    V = wl.dx * wl.dx * wl.dx
    for _ in range(wl.steps):
        Port.sources_tracked(f, wl.S, wl.agent_voxel, c1, c2, e2, wl.net_export * wl.dt, V, internal)
        Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    for precision in ("fp64", "fp32"):
        outs = []
        for persistent in (2, 1, 0):
            me = Microenvironment.from_workload(wl, precision)
            me.set_sweep_schedule(persistent)
            assert me.get_sweep_schedule() == persistent
            me.set_track_internalized_substrates(True)
            me.simulate_diffusion_decay(wl.steps, sources=True)
            outs.append((me.download_field(), me.internalized_substrates()))
            me.close()
        for o in outs[1:]:
            assert np.array_equal(outs[0][0], o[0]), precision
            assert np.array_equal(outs[0][1], o[1]), precision
        if precision == "fp64":
            assert np.array_equal(outs[0][0], f)
            assert np.array_equal(outs[0][1], internal)
        else:
            assert np.all(_normwise(outs[0][0], f, wl.S) <= FP32_TOL)


def test_upload_download_roundtrip_and_sums():
    wl = W.small_random(36, nx=37, ny=41, nz=29, S=3, n_agents=0)
    for prec in ("fp64", "fp32"):
        me = Microenvironment.from_workload(wl, precision=prec)
        back = me.download_field()
        if prec == "fp64":
            assert np.array_equal(back, wl.field0)
        else:
            # stored as an FP32 deviation from a per-substrate FP64 offset
            err = np.max(np.abs(back - wl.field0))
            assert err <= 2.0 ** -23 * np.max(np.abs(wl.field0)) * 2, err
        sums = me.field_sums()
        np.testing.assert_allclose(sums, back.reshape(-1, wl.S).sum(axis=0), rtol=1e-12)


def test_device_pointer_upload_matches_host_upload():
    import torch

    wl = W.small_random(37, n_agents=50, steps=2)
    a = Microenvironment.from_workload(wl)
    b = Microenvironment.from_workload(wl, upload=False)
    d = torch.from_numpy(wl.field0).cuda()
    b.upload_field_device(d.data_ptr())
    for me in (a, b):
        me.simulate_diffusion_decay(wl.steps, sources=True)
    out = torch.empty_like(d)
    b.download_field_device(out.data_ptr())
    b.synchronize()
    assert np.array_equal(a.download_field(), out.cpu().numpy())


def test_kat_uniform_field_at_cube200_size():
    """Size-independent property at the full cube200 grid (200^3 x 4): a
    uniform zero-flux field divides by (1 + dt*lambda/3)^3 per step."""
    wl = W.cube200(n_agents=0, steps=3)
    me = Microenvironment(wl.nx, wl.ny, wl.nz, wl.dx, wl.dt, wl.D, wl.decay)
    me.set_dirichlet_activation(np.zeros(wl.S, np.uint8))
    me.upload_field(np.full(wl.n_values, 5.0))
    me.simulate_diffusion_decay(wl.steps)
    f = me.download_field().reshape(-1, wl.S)
    for d in range(wl.S):
        np.testing.assert_allclose(f[:, d], 5.0 / (1 + wl.dt * wl.decay[d] / 3) ** (3 * wl.steps), rtol=1e-12)


@pytest.mark.parametrize("seed", [300, 301, 302])
def test_fp32_within_tolerance_small(seed):
    wl = W.small_random(seed, steps=20, n_agents=200, stack=True)
    ref = Port.run(wl)
    me = Microenvironment.from_workload(wl, precision="fp32")
    me.simulate_diffusion_decay(wl.steps, sources=True)
    err = _normwise(me.download_field(), ref, wl.S)
    assert np.all(err <= FP32_TOL), err


def test_fp32_cube50_full_run_within_tolerance():
    wl = W.cube50(steps=1000)
    ref = Port.run(wl)
    me = Microenvironment.from_workload(wl, precision="fp32")
    me.simulate_diffusion_decay(wl.steps, sources=True)
    err = _normwise(me.download_field(), ref, wl.S)
    assert np.all(err <= FP32_TOL), err


def test_kernel_launch_counter_moves():
    before = kernel_launches()
    wl = W.small_random(38, steps=2)
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(2, sources=True)
    me.synchronize()
    assert kernel_launches() - before >= 6


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 48, 40, 2), (33, 100, 57, 3), (200, 200, 120, 1), (70, 256, 130, 2),
                                   (40, 257, 50, 1), (256, 40, 36, 2), (20, 64, 48, 1), (257, 33, 34, 1),
                                   (36, 400, 70, 2), (34, 40, 640, 1), (400, 36, 34, 2), (640, 33, 35, 1),
                                   (36, 33, 700, 1), (700, 33, 34, 1), (36, 210, 736, 1), (736, 33, 34, 1),
                                   (34, 650, 36, 1)])
def test_tmem_sweeps_bitwise(shape):
    """The persistent sweeps with tensor-memory rings (lines of up to 16
    chunks in TMEM and, past 256, 16 in TMEM plus the rest resident in shared
    memory, up to the longest planned line of 736, one TMEM ring from 657;
    two input slots per TMEM ring at lines of 210, 650 and 736, three
    elsewhere; x lines of up to 256 only at level 2):
    with and without TMEM, under the persistent schedules, bit for bit
    against the oracle, with sources, faces, ragged line ends and partial
    tiles."""
    nx, ny, nz, S = shape
    wl = W.small_random(990 + nx, nx=nx, ny=ny, nz=nz, S=S, n_agents=3000, steps=3, stack=True)
    expect = Port.run(wl)
    for sched, tmem in ((2, 2), (1, 2), (1, 1), (2, 0)):
        me = Microenvironment.from_workload(wl)
        me.set_sweep_schedule(sched)
        me.set_sweep_tmem(tmem)
        me.simulate_diffusion_decay(wl.steps, sources=True)
        got = me.download_field()
        me.close()
        assert np.array_equal(got, expect), (shape, sched, tmem)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 48, 40, 2), (33, 100, 57, 3), (70, 256, 130, 2), (40, 257, 50, 1),
                                   (20, 64, 48, 1), (36, 400, 70, 2), (34, 40, 640, 1), (36, 33, 700, 1),
                                   (36, 210, 736, 1), (34, 650, 36, 1), (200, 200, 40, 4), (257, 33, 34, 1),
                                   (640, 33, 35, 1), (300, 70, 36, 2), (1000, 33, 34, 1)])
@pytest.mark.parametrize("chain", [0, 1])
def test_tmem_sweeps_fp32_bitwise(shape, chain):
    """The FP32 sweeps with tensor-memory rings (two rings per TMEM lane
    quarter; y/z lines of up to 16 chunks of 16 rows in TMEM, x lines of up
    to 8 chunks of 32 values, the rest resident in shared memory): bit for bit
    the FP32 shared-memory sweeps (TMEM off), under both persistent schedules
    and both forms of the recurrence, and within the FP32 form's tolerance of
    the oracle."""
    nx, ny, nz, S = shape
    wl = W.small_random(1990 + nx + ny, nx=nx, ny=ny, nz=nz, S=S, n_agents=3000, steps=3, stack=True)
    runs = {}
    for sched, tmem in ((1, 0), (1, 1), (2, 1), (1, 2)):
        me = Microenvironment.from_workload(wl, precision="fp32")
        me.set_fp64_chain(chain)
        me.set_sweep_schedule(sched)
        me.set_sweep_tmem(tmem)
        me.simulate_diffusion_decay(wl.steps, sources=True)
        runs[(sched, tmem)] = me.download_field()
        me.close()
    base = runs[(1, 0)]
    for key, got in runs.items():
        assert np.array_equal(got, base), (shape, chain, key)
    err = _normwise(base, Port.run(wl), S)
    assert np.all(err <= FP32_TOL), err


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_substrate_streams_give_the_same_bits(precision):
    """Runs of steps with the substrates split over two streams (the default)
    equal one sequence of launches bit for bit: an odd substrate count (groups
    of 2 and 1), stacked agents with internalized-substrate tracking, fused
    and standalone sources, a run long enough to replay the captured graph
    plus a remainder, and a short uncaptured run.  FP64 equals the oracle."""
    wl = W.small_random(37, nx=200, ny=64, nz=40, S=3, n_agents=6000, steps=21, agent_mode="gauss", stack=True)
    c1, c2, e2 = Port.workload_constants(wl)
    f = wl.field0.copy()
    internal = np.zeros((wl.n_agents, wl.S))
    V = wl.dx * wl.dx * wl.dx
    for _ in range(wl.steps + 3):
        Port.sources_tracked(f, wl.S, wl.agent_voxel, c1, c2, e2, wl.net_export * wl.dt, V, internal)
        Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    for fused in (False, True):
        outs = []
        for streams in (1, 2):
            me = Microenvironment.from_workload(wl, precision)
            me.set_substrate_streams(streams)
            assert me.substrate_streams() == streams
            me.set_fused_sources(fused)
            me.set_track_internalized_substrates(True)
            me.simulate_diffusion_decay(wl.steps, sources=True)
            me.simulate_diffusion_decay(3, sources=True)
            outs.append((me.download_field(), me.internalized_substrates()))
            me.close()
        assert np.array_equal(outs[0][0], outs[1][0]), (precision, fused)
        assert np.array_equal(outs[0][1], outs[1][1]), (precision, fused)
        if precision == "fp64":
            assert np.array_equal(outs[1][0], f), fused
            assert np.array_equal(outs[1][1], internal), fused
        else:
            assert np.all(_normwise(outs[1][0], f, wl.S) <= FP32_TOL), fused


@pytest.mark.parametrize("shape", [(42, 70, 45, 2), (48, 40, 37, 1), (81, 50, 33, 2), (100, 36, 70, 3)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_packed_partial_tiles(shape, precision):
    """The y/z sweeps pack the partial x tiles of several planes into one
    tile (x extents whose remainder mod 32 is 10, 16, 17 -- not packed -- and
    4), and the x sweep runs its lines in row order across y-row ends: FP64
    bit for bit against the oracle, FP32 within its tolerance, both with the
    sweeps in tensor memory forced on every axis."""
    nx, ny, nz, S = shape
    wl = W.small_random(38 + nx, nx=nx, ny=ny, nz=nz, S=S, n_agents=1500, steps=3, stack=True)
    me = Microenvironment.from_workload(wl, precision)
    me.set_sweep_schedule(2)
    me.set_sweep_tmem(2)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    got = me.download_field()
    me.close()
    expect = Port.run(wl)
    if precision == "fp64":
        assert np.array_equal(got, expect)
    else:
        assert np.all(_normwise(got, expect, S) <= FP32_TOL)
