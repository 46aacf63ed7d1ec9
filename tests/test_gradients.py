"""Substrate gradients (Microenvironment::compute_all_gradient_vectors,
BioFVM/BioFVM_microenvironment.cpp:1454-1616): the oracle against the
reference build on CPU, the GPU kernel against the oracle bit for bit."""
import numpy as np
import pytest

import pyoracle
from bfvm import workloads as W

SHAPES = [(9, 7, 5, 2), (2, 3, 4, 1), (17, 1, 6, 3), (5, 4, 1, 2), (33, 20, 12, 3)]


def _case(i, shape):
    nx, ny, nz, S = shape
    return W.small_random(500 + i, nx=nx, ny=ny, nz=nz, S=S, n_agents=20, steps=2)


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
def test_oracle_gradients_match_reference_build():
    # every axis at least 2 long: the reference reads outside its array otherwise
    for i, shape in enumerate([s for s in SHAPES if min(s[:3]) >= 2]):
        wl = _case(i, shape)
        ref = pyoracle.Reference(wl, threads=2)
        field = ref.run(2)
        got = pyoracle.Port.gradients(field, wl.shape, wl.dx)
        want = ref.gradients()
        ref.close()
        assert np.array_equal(got, want), shape


def test_oracle_gradients_of_a_linear_field():
    nx, ny, nz, S, dx = 6, 5, 4, 2, 10.0
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    f = np.stack([2.0 * i + 3.0 * j - 1.0 * k, 0.5 * k], axis=-1).astype(np.float64)
    g = pyoracle.Port.gradients(f.ravel(), (nx, ny, nz, S), dx)
    np.testing.assert_allclose(g[:, 0, :], np.tile([0.2, 0.3, -0.1], (nx * ny * nz, 1)), rtol=0, atol=1e-15)
    np.testing.assert_allclose(g[:, 1, :], np.tile([0.0, 0.0, 0.05], (nx * ny * nz, 1)), rtol=0, atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("idx", range(len(SHAPES)))
def test_gpu_gradients_bitwise_fp64(idx):
    from bfvm import Microenvironment

    wl = _case(idx, SHAPES[idx])
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    field = me.download_field()
    got = me.compute_all_gradient_vectors()
    me.close()
    assert np.array_equal(got, pyoracle.Port.gradients(field, wl.shape, wl.dx))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(70, 45, 37, 3), (65, 33, 40, 6), (200, 200, 30, 4), (31, 9, 17, 5),
                                   (40, 300, 9, 1)])
def test_gpu_gradients_plane_kernel_bitwise(shape):
    """The plane-ring kernel on shapes with partial x/z tiles, several y
    ranges, substrate groups of 4 with a partial last group."""
    from bfvm import Microenvironment

    nx, ny, nz, S = shape
    wl = W.small_random(777 + nx, nx=nx, ny=ny, nz=nz, S=S, n_agents=500, steps=2)
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    field = me.download_field()
    got = me.compute_all_gradient_vectors()
    me.synchronize()
    me.close()
    assert np.array_equal(got, pyoracle.Port.gradients(field, wl.shape, wl.dx))


@pytest.mark.gpu
def test_gpu_gradients_fp32_and_device_output():
    import torch

    from bfvm import Microenvironment

    wl = W.cube50(steps=20)
    me64 = Microenvironment.from_workload(wl, "fp64")
    me32 = Microenvironment.from_workload(wl, "fp32")
    for me in (me64, me32):
        me.simulate_diffusion_decay(wl.steps, sources=True)
    g64 = me64.compute_all_gradient_vectors()
    g32 = me32.compute_all_gradient_vectors()
    dev = torch.empty(g64.size, dtype=torch.float64, device="cuda:0")
    me64.compute_all_gradient_vectors_device(dev.data_ptr())
    me64.synchronize()
    assert np.array_equal(dev.cpu().numpy().reshape(g64.shape), g64)
    # an output 8 bytes past a 16-byte boundary (S even: the kernel's 16-byte
    # row stores give way to 8-byte ones)
    dev8 = torch.zeros(g64.size + 1, dtype=torch.float64, device="cuda:0")
    me64.compute_all_gradient_vectors_device(dev8.data_ptr() + 8)
    me64.synchronize()
    assert np.array_equal(dev8[1:].cpu().numpy().reshape(g64.shape), g64)
    for s in range(wl.S):
        scale = np.abs(g64[:, s, :]).max()
        assert np.abs(g32[:, s, :] - g64[:, s, :]).max() <= 1e-5 * scale
    me64.close()
    me32.close()
