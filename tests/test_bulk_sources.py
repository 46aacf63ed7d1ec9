"""Bulk (per-voxel) sources and sinks (Microenvironment::simulate_bulk_sources_
and_sinks, BioFVM/BioFVM_microenvironment.cpp:1327-1368): the oracle against
the reference build on CPU, the GPU pass against the oracle bit for bit."""
import numpy as np
import pytest

import pyoracle
from bfvm import workloads as W


def _rates(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0, 5, n), rng.uniform(0, 40, n), rng.uniform(0, 3, n)


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_bulk_matches_reference_build(seed):
    wl = W.small_random(600 + seed, n_agents=0, steps=1)
    S_, T_, U_ = _rates(wl.n_values, seed)
    ref = pyoracle.Reference(wl, threads=1)
    f = ref.field().copy()
    ref.bulk_sources(S_, T_, U_)
    pyoracle.Port.bulk_sources(f, wl.dt, S_, T_, U_)
    want = ref.field()
    ref.close()
    assert np.array_equal(f, want)


def test_oracle_bulk_fixed_point():
    # with S = 0 the update is rho / (1 + U dt); with U = 0 and rho = T it keeps rho = T
    f = np.full(10, 7.0)
    pyoracle.Port.bulk_sources(f, 0.1, np.full(10, 2.0), np.full(10, 7.0), np.zeros(10))
    np.testing.assert_allclose(f, 7.0, rtol=1e-15)
    f = np.full(4, 3.0)
    pyoracle.Port.bulk_sources(f, 0.5, np.zeros(4), np.zeros(4), np.full(4, 2.0))
    np.testing.assert_array_equal(f, 3.0 / 2.0)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [4, 5])
def test_gpu_bulk_bitwise_and_with_steps(seed):
    from bfvm import Microenvironment

    wl = W.small_random(700 + seed, nx=23, ny=17, nz=11, S=3, n_agents=40, steps=3)
    S_, T_, U_ = _rates(wl.n_values, seed)
    me = Microenvironment.from_workload(wl)
    me.set_bulk_rates(S_, T_, U_)
    f = wl.field0.copy()
    c1, c2, e2 = pyoracle.Port.workload_constants(wl)
    for _ in range(wl.steps):
        me.simulate_bulk_sources_and_sinks()
        me.simulate_diffusion_decay(1, sources=True)
        pyoracle.Port.bulk_sources(f, wl.dt, S_, T_, U_)
        pyoracle.Port.sources(f, wl.S, wl.agent_voxel, c1, c2, e2)
        pyoracle.Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    assert np.array_equal(me.download_field(), f)
    me.set_bulk_rates(None, None, None)
    me.close()


@pytest.mark.gpu
def test_gpu_bulk_fp32_within_tolerance_and_state_error():
    from bfvm import BfvmError, Microenvironment

    wl = W.small_random(710, nx=30, ny=20, nz=10, S=2, n_agents=0, steps=1)
    me = Microenvironment.from_workload(wl, "fp32")
    with pytest.raises(BfvmError):
        me.simulate_bulk_sources_and_sinks()  # no rates yet
    S_, T_, U_ = _rates(wl.n_values, 6)
    me.set_bulk_rates(S_, T_, U_)
    for _ in range(5):
        me.simulate_bulk_sources_and_sinks()
    f = wl.field0.copy()
    for _ in range(5):
        pyoracle.Port.bulk_sources(f, wl.dt, S_, T_, U_)
    got = me.download_field().reshape(-1, wl.S)
    want = f.reshape(-1, wl.S)
    for s in range(wl.S):
        assert np.abs(got[:, s] - want[:, s]).max() <= 1e-6 * np.abs(want[:, s]).max()
    me.close()
