"""GPU parity at the benchmark configurations themselves.

* cube200 (200^3 x 4 substrates, 100,000 agents) for all 500 of its steps,
  bit-identical to the reference's own solver (its golden hash).
* cube640's 640-voxel lines along each axis (the cube640 slabs) and, where
  the fixture exists, the full 640^3 x 2 grid with 1,000,000 agents in a
  Gaussian ball for 5 steps: bit-identical to the fixture.
* The FP32 form on cube640 for all 1000 steps: per substrate, normwise
  relative L-infinity error max|g - r| / max|r| <= 1e-5 against the FP64
  path, which the fixtures pin to the reference bit for bit.
* The FP32 batched engine on the first 16 solves of the uneven batch
  (edges 24-128, 1-6 substrates, 0-20k agents, 200 steps) against the FP64
  oracle, same bound.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from bfvm import Microenvironment
from bfvm import workloads as W
from pyoracle import Port

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5  # normwise relative L-infinity per substrate


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"), allow_pickle=False)


def _cases(golden_dir):
    with open(os.path.join(golden_dir, "MANIFEST.json")) as fh:
        return json.load(fh)["cases"]


def _check_hash(golden_dir, name, wl):
    g = _load(golden_dir, name)
    assert tuple(int(v) for v in g["shape"]) == wl.shape
    assert _sha(wl.field0) == str(g["field0_sha"]), name
    assert _sha(wl.agent_voxel) == str(g["voxel_sha"]), name
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    out = me.download_field()
    me.close()
    assert np.array_equal(out[g["sample_idx"]], g["sample_val"]), name
    np.testing.assert_array_equal(out.reshape(-1, wl.S).sum(axis=0), g["sums"])
    assert _sha(out) == str(g["final_sha"]), name


def test_cube200_all_500_steps_match_reference_hash(golden_dir):
    _check_hash(golden_dir, "cube200_500", W.cube200(steps=500))


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_cube640_lines_match_reference_hash(golden_dir, axis):
    wl = W.cube640_slab(axis)
    _check_hash(golden_dir, f"{wl.name}_{wl.steps}", wl)


def test_cube640_full_grid_matches_fixture(golden_dir):
    if "cube640_5" not in _cases(golden_dir):
        pytest.skip("no cube640_5 fixture")
    _check_hash(golden_dir, "cube640_5", W.cube640(steps=5))


def _device_field(me):
    import torch

    nx, ny, nz, S = me.shape
    out = torch.empty((nx * ny * nz, S), dtype=torch.float64, device="cuda:0")
    me.download_field_device(out.data_ptr())
    me.synchronize()
    return out


def test_fp32_cube640_1000_steps_within_tolerance():
    torch = pytest.importorskip("torch")
    wl = W.cube640(steps=1000)
    fields = {}
    for prec in ("fp64", "fp32"):
        me = Microenvironment.from_workload(wl, precision=prec)
        me.simulate_diffusion_decay(wl.steps, sources=True)
        fields[prec] = _device_field(me)
        me.close()
    r, g = fields["fp64"], fields["fp32"]
    err = ((g - r).abs().amax(dim=0) / r.abs().amax(dim=0)).cpu().numpy()
    del fields, r, g
    torch.cuda.empty_cache()
    assert np.all(err <= FP32_TOL), err


def test_fp32_batch_uneven_slice_within_tolerance():
    from bfvm.batch import Batch

    wls = W.uneven_batch(16)
    b = Batch("fp32", 0)
    mes = [Microenvironment.from_workload(wl, "fp32", 0) for wl in wls]
    for me in mes:
        b.add(me)
    b.step(wls[0].steps, sources=True)
    b.synchronize()
    worst = 0.0
    for wl, me in zip(wls, mes):
        ref = Port.run(wl).reshape(-1, wl.S)
        got = me.download_field().reshape(-1, wl.S)
        err = np.max(np.abs(got - ref), axis=0) / np.max(np.abs(ref), axis=0)
        worst = max(worst, float(err.max()))
        assert np.all(err <= FP32_TOL), (wl.name, err)
        me.close()
    b.close()
    assert worst > 0.0  # the FP32 form does round
