"""The synthetic workloads the bench and the suites run (bfvm/workloads.py)
against the configurations they are quoted on: extents, spacing, substrates
and their parameters, Dirichlet data, agent counts, rates and placement, step
counts, and that a seed always draws the same workload.  The initial fields
(up to 4 GB for cube640) are not drawn here."""
import math

import numpy as np
import pytest

from bfvm import workloads as W


def _inside(wl):
    o = np.asarray(wl.origin, np.float64)
    ext = np.array([wl.nx, wl.ny, wl.nz], np.float64) * wl.dx
    return np.all(wl.agent_pos > o) and np.all(wl.agent_pos < o + ext)


def test_cube50():
    wl = W.cube50()
    assert (wl.nx, wl.ny, wl.nz, wl.S) == (50, 50, 50, 2)
    assert (wl.dx, wl.dt, wl.steps) == (20.0, 0.01, 1000)
    assert list(wl.D) == [1e5, 1e3] and list(wl.decay) == [0.1, 0.01]
    assert list(wl.dirichlet_active) == [1, 0] and np.all(wl.face_values[:, 0] == 38.0)
    assert wl.n_agents == 2000 and _inside(wl)
    assert np.all(wl.uptake[:, 0] == 10.0) and np.all(wl.uptake[:, 1] == 0.0)
    assert np.all(wl.secretion[:, 1] == 1.0) and np.all(wl.secretion[:, 0] == 0.0)
    assert np.all(wl.saturation == 1.0) and np.all(wl.agent_volume == 2494.0)
    assert wl.init_kind == (("const", 38.0), ("uniform", 0.0, 0.1))


def test_cube200():
    wl = W.cube200()
    assert (wl.nx, wl.ny, wl.nz, wl.S) == (200, 200, 200, 4)
    assert (wl.dx, wl.dt, wl.steps) == (10.0, 0.01, 500)
    assert np.all((wl.D >= 1e2) & (wl.D <= 1e5)) and np.all((wl.decay >= 1e-3) & (wl.decay <= 1.0))
    assert list(wl.dirichlet_active) == [1, 0, 0, 0] and np.all(wl.face_values[:, 0] == 38.0)
    assert wl.n_agents == 100_000 and _inside(wl)
    assert wl.uptake.min() >= 0.0 and wl.uptake.max() <= 10.0
    assert wl.secretion.min() >= 0.0 and wl.secretion.max() <= 1.0
    assert wl.n_voxels * wl.S == 32_000_000


def test_cube640():
    wl = W.cube640()
    assert (wl.nx, wl.ny, wl.nz, wl.S) == (640, 640, 640, 2)
    assert (wl.dx, wl.steps) == (10.0, 1000)
    assert wl.n_agents == 1_000_000 and _inside(wl)
    # Gaussian about the centre (sigma 1500 um per axis), clamped into the box
    # (half-width a = 3200 um): the clamped normal's standard deviation is
    # sigma * sqrt(P(|Z|<k) - 2 k phi(k) + k^2 P(|Z|>k)), k = a / sigma;
    # many agents share voxels
    sigma, a = 1500.0, 3200.0
    k = a / sigma
    inside = math.erf(k / math.sqrt(2.0))
    phi = math.exp(-0.5 * k * k) / math.sqrt(2.0 * math.pi)
    want_std = sigma * math.sqrt(inside - 2.0 * k * phi + k * k * (1.0 - inside))
    centre = np.asarray(wl.origin) + 640 * 10.0 / 2
    assert np.all(np.abs(wl.agent_pos.mean(0) - centre) < 20.0)
    assert np.all(np.abs(wl.agent_pos.std(0) - want_std) < 10.0)
    assert np.unique(wl.agent_voxel).size < wl.n_agents


def test_uneven_batch_and_serving_streams():
    envs = W.uneven_batch()
    assert len(envs) == 256
    for wl in envs:
        assert all(24 <= n <= 128 for n in (wl.nx, wl.ny, wl.nz))
        assert 1 <= wl.S <= 6 and 0 <= wl.n_agents <= 20_000 and wl.steps == 200
    for i in range(24):
        wl = W.serve_request(i)
        assert all(32 <= n <= 256 for n in (wl.nx, wl.ny, wl.nz))
        assert 1 <= wl.S <= 8 and 0 <= wl.n_agents <= 200_000 and 100 <= wl.steps <= 10_000
        assert wl.dx == 10.0


@pytest.mark.parametrize("make", [lambda: W.cube200(n_agents=1000), lambda: W.uneven_env(7),
                                  lambda: W.serve_request(3), lambda: W.small_random(11, stack=True)])
def test_a_seed_draws_the_same_workload(make):
    a, b = make(), make()
    for key in ("agent_pos", "uptake", "secretion", "D", "decay", "face_values"):
        assert np.array_equal(getattr(a, key), getattr(b, key)), key
    if a.n_voxels * a.S < 5_000_000:
        assert np.array_equal(a.field0, b.field0)
