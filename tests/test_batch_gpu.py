"""The batched engine: one fused launch per LOD step over many uneven solves.

Every member must give the same result as when stepped alone -- bit for bit
in FP64 against the oracle, and bit for bit against its own single-solve
FP32 run (the fused kernel runs the same per-tile code)."""
import numpy as np
import pytest

from bfvm import Batch, Microenvironment
from bfvm import workloads as W
from pyoracle import Port

pytestmark = pytest.mark.gpu


def _envs(n, seed, steps, agents_hi=300, edge_lo=3, edge_hi=40):
    out = []
    for i in range(n):
        rng = np.random.default_rng([seed, i])
        nx, ny, nz = (int(v) for v in rng.integers(edge_lo, edge_hi + 1, 3))
        out.append(W.small_random(seed * 1000 + i, nx=nx, ny=ny, nz=nz, S=int(rng.integers(1, 5)),
                                  n_agents=int(rng.integers(0, agents_hi)), steps=steps, stack=bool(i % 2)))
    return out


@pytest.mark.parametrize("mode,graph_steps", [(0, 1), (0, 4), (1, 1), (1, 4)])
def test_batch_fp64_members_match_oracle_bitwise(mode, graph_steps):
    wls = _envs(12, 7, steps=9)
    batch = Batch("fp64")
    batch.set_schedule(mode=mode, graph_steps=graph_steps)
    mes = []
    for wl in wls:
        me = Microenvironment.from_workload(wl)
        batch.add(me)
        mes.append(me)
    batch.step(9, sources=True)
    batch.synchronize()
    for wl, me in zip(wls, mes):
        assert np.array_equal(me.download_field(), Port.run(wl)), wl.name


def test_batch_fp32_equals_single_fp32_bitwise():
    wls = _envs(8, 8, steps=6)
    batch = Batch("fp32")
    singles, mes = [], []
    for wl in wls:
        me = Microenvironment.from_workload(wl, precision="fp32")
        batch.add(me)
        mes.append(me)
        one = Microenvironment.from_workload(wl, precision="fp32")
        one.simulate_diffusion_decay(wl.steps, sources=True)
        singles.append(one.download_field())
    batch.step(6, sources=True)
    for ref, me in zip(singles, mes):
        assert np.array_equal(me.download_field(), ref)


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_membership_changes_between_steps(mode):
    """Members join and leave between steps (continuous batching); each still
    ends bit-identical to its solo run."""
    wls = _envs(6, 9, steps=8)
    batch = Batch("fp64")
    batch.set_schedule(mode=mode, graph_steps=2)
    mes = [Microenvironment.from_workload(wl) for wl in wls]
    done = {}
    for me in mes[:3]:
        batch.add(me)
    batch.step(4, sources=True)
    batch.remove(mes[0])
    for me in mes[3:]:
        batch.add(me)
    batch.step(4, sources=True)
    done[0] = mes[0].download_field()
    for i in (1, 2):
        done[i] = mes[i].download_field()
    batch.step(4, sources=True)
    for i in (3, 4, 5):
        done[i] = mes[i].download_field()
    assert np.array_equal(done[0], Port.run(wls[0], nsteps=4))
    for i in (1, 2):
        assert np.array_equal(done[i], Port.run(wls[i], nsteps=8))
    for i in (3, 4, 5):
        assert np.array_equal(done[i], Port.run(wls[i], nsteps=8))


def test_batch_autotune_keeps_fields():
    wls = _envs(5, 10, steps=3, edge_hi=64)
    batch = Batch("fp64")
    mes = [Microenvironment.from_workload(wl) for wl in wls]
    for me in mes:
        batch.add(me)
    before = [me.download_field() for me in mes]
    ms = batch.autotune(sources=True, trial_steps=2)
    assert ms > 0
    for b, me in zip(before, mes):
        assert np.array_equal(b, me.download_field())
    batch.step(3, sources=True)
    for wl, me in zip(wls, mes):
        assert np.array_equal(me.download_field(), Port.run(wl))


def test_uneven_batch_slice_runs():
    """A slice of the uneven_batch workload (uneven 24-128 edges, 1-6 substrates,
    random Dirichlet faces): a few fused steps, checked against solo runs."""
    wls = W.uneven_batch(n_envs=6, steps=3, agents_hi=2000)
    batch = Batch("fp64")
    mes = []
    for wl in wls:
        me = Microenvironment.from_workload(wl)
        batch.add(me)
        mes.append(me)
    batch.step(3, sources=True)
    for wl, me in zip(wls, mes):
        solo = Microenvironment.from_workload(wl)
        solo.simulate_diffusion_decay(3, sources=True)
        assert np.array_equal(me.download_field(), solo.download_field())
