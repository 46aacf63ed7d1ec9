"""The FP64 chains that are not the reference's operation order -- the short
chain (bfvm_set_fp64_chain(ctx, 1)) and the partitioned sweeps (chain 2) --
against the oracle: within the 1e-12 relative per-voxel bound the FP64 path
is held to, on the benchmark configurations' shapes and step counts, under
every sweep kernel (per-tile, persistent, tensor memory, partitioned,
batched)."""
import numpy as np
import pytest

from bfvm import Batch, Microenvironment
from bfvm import workloads as W
from pyoracle import Port

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12  # relative per voxel (floor 1e-30 on the magnitude)


def _per_voxel(got, ref):
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-30)))


@pytest.mark.parametrize("chain", [1, 2])
def test_short_chain_cube50_all_steps_within_bound(chain):
    wl = W.cube50(steps=1000)
    me = Microenvironment.from_workload(wl)
    me.set_fp64_chain(chain)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    got = me.download_field()
    err = _per_voxel(got, Port.run(wl))
    assert 0.0 < err <= FP64_TOL, err


@pytest.mark.parametrize("sched,tmem,chain", [(0, 0, 1), (1, 1, 1), (2, 2, 1), (2, 0, 1), (1, 1, 2)])
def test_short_chain_every_kernel(sched, tmem, chain):
    wl = W.small_random(821, nx=70, ny=257, nz=40, S=3, n_agents=3000, steps=20, stack=True)
    expect = Port.run(wl)
    me = Microenvironment.from_workload(wl)
    me.set_sweep_schedule(sched)
    me.set_sweep_tmem(tmem)
    me.set_fp64_chain(chain)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    assert _per_voxel(me.download_field(), expect) <= FP64_TOL
    # back to the reference's arithmetic: the reference's bits again
    me.upload_field(wl.field0)
    me.set_fp64_chain(0)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    np.testing.assert_array_equal(me.download_field(), expect)
    me.close()


def test_short_chain_in_the_batch():
    wls = [W.uneven_env(i, steps=30) for i in range(4)]
    b = Batch("fp64")
    mes = []
    for wl in wls:
        me = Microenvironment.from_workload(wl)
        me.set_fp64_chain(1)
        b.add(me)
        mes.append(me)
    b.step(30, sources=True)
    b.synchronize()
    for wl, me in zip(wls, mes):
        assert _per_voxel(me.download_field(), Port.run(wl)) <= FP64_TOL, wl.name
    b.close()


@pytest.mark.parametrize("chain", [1, 2])
def test_short_chain_fp32_within_tolerance(chain):
    """The FP32 form's FP64 recurrence with the short chain stays within the
    FP32 form's 1e-5 normwise bound of the FP64 oracle."""
    wl = W.cube50(steps=1000)
    ref = Port.run(wl).reshape(-1, wl.S)
    me = Microenvironment.from_workload(wl, precision="fp32")
    me.set_fp64_chain(chain)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    got = me.download_field().reshape(-1, wl.S)
    me.close()
    err = np.max(np.abs(got - ref), axis=0) / np.max(np.abs(ref), axis=0)
    assert np.all(err <= 1e-5), err


@pytest.mark.parametrize("chain", [1, 2])
def test_short_chain_cube200_all_steps_against_reference_sample(golden_dir, chain):
    """cube200 for all 500 steps with the short chain: the 4096 sampled
    voxels of the reference's own final field (its golden fixture) agree to
    1e-12 relative, and the per-substrate sums to 1e-12."""
    import os

    g = np.load(os.path.join(golden_dir, "cube200_500.npz"))
    wl = W.cube200(steps=500)
    me = Microenvironment.from_workload(wl)
    me.set_fp64_chain(chain)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    out = me.download_field()
    me.close()
    idx = g["sample_idx"]
    assert _per_voxel(out[idx], g["sample_val"]) <= FP64_TOL
    np.testing.assert_allclose(out.reshape(-1, wl.S).sum(axis=0), g["sums"], rtol=FP64_TOL)


@pytest.mark.parametrize("shape", [(1, 1, 1, 1), (1, 7, 3, 2), (9, 2, 5, 3), (256, 3, 5, 1), (3, 256, 4, 2),
                                   (5, 4, 256, 1), (129, 65, 33, 3), (33, 100, 57, 3), (200, 40, 37, 2),
                                   (640, 33, 35, 1), (36, 640, 40, 1), (40, 34, 700, 2)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_partitioned_sweeps_edge_shapes(shape, precision):
    """The partitioned sweeps on ragged and tiny shapes (segments shorter than
    the eight warps, empty segments, partial tiles, faces with their own
    values, stacked agents) against the oracle: FP64 within 1e-12 per voxel,
    FP32 within the FP32 form's 1e-5 normwise bound."""
    nx, ny, nz, S = shape
    wl = W.small_random(1300 + nx + 7 * ny + 3 * nz, nx=nx, ny=ny, nz=nz, S=S, n_agents=300, steps=6, stack=True)
    expect = Port.run(wl)
    me = Microenvironment.from_workload(wl, precision=precision)
    me.set_fp64_chain(2)
    assert me.get_partition_min_line() == (512 if precision == "fp64" else 448)
    me.set_partition_min_line(1)  # every y and z line, however short, runs partitioned
    me.simulate_diffusion_decay(wl.steps, sources=True)
    got = me.download_field()
    me.close()
    if precision == "fp64":
        assert _per_voxel(got, expect) <= FP64_TOL
    else:
        g, r = got.reshape(-1, S), expect.reshape(-1, S)
        assert np.all(np.max(np.abs(g - r), axis=0) <= 1e-5 * np.max(np.abs(r), axis=0))


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_partitioned_sweeps_cube640_lines_against_reference(golden_dir, axis):
    """cube640's 640-voxel lines (one CTA per tile along that axis) with the
    partitioned sweeps: every value of the reference's own 5-step fixture
    sample within 1e-12 relative, and the sums."""
    import os

    wl = W.cube640_slab(axis)
    g = np.load(os.path.join(golden_dir, f"{wl.name}_{wl.steps}.npz"))
    me = Microenvironment.from_workload(wl)
    me.set_fp64_chain(2)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    out = me.download_field()
    me.close()
    assert _per_voxel(out[g["sample_idx"]], g["sample_val"]) <= FP64_TOL
    np.testing.assert_allclose(out.reshape(-1, wl.S).sum(axis=0), g["sums"], rtol=FP64_TOL)
