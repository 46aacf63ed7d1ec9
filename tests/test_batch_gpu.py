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


# mode 2 with a threshold of 5000 voxel-substrate values: the larger members
# step with their own kernels, the rest through the batched sweeps
DIRECT_TEST = 5000


@pytest.mark.parametrize("mode,graph_steps", [(0, 1), (0, 4), (1, 1), (1, 4), (2, 1), (2, 4)])
def test_batch_fp64_members_match_oracle_bitwise(mode, graph_steps):
    wls = _envs(12, 7, steps=9)
    batch = Batch("fp64")
    batch.set_schedule(mode=mode, graph_steps=graph_steps)
    batch.set_direct_threshold(DIRECT_TEST)
    mes = []
    for wl in wls:
        me = Microenvironment.from_workload(wl)
        batch.add(me)
        mes.append(me)
    batch.step(9, sources=True)
    batch.synchronize()
    for wl, me in zip(wls, mes):
        assert np.array_equal(me.download_field(), Port.run(wl)), wl.name


@pytest.mark.parametrize("mode", [0, 2])
def test_batch_fp32_equals_single_fp32_bitwise(mode):
    wls = _envs(8, 8, steps=6)
    batch = Batch("fp32")
    batch.set_schedule(mode=mode, graph_steps=4)
    batch.set_direct_threshold(DIRECT_TEST)
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


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_batch_membership_changes_between_steps(mode):
    """Members join and leave between steps (continuous batching); each still
    ends bit-identical to its solo run."""
    wls = _envs(6, 9, steps=8)
    batch = Batch("fp64")
    batch.set_schedule(mode=mode, graph_steps=2)
    batch.set_direct_threshold(DIRECT_TEST)
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


def test_batch_direct_members_count_their_launches():
    """Mode 2: the launch counter counts the directly stepped members' kernels
    once per step, whether launched one step at a time or replayed from the
    batch's graph."""
    from bfvm import kernel_launches

    wls = [W.small_random(9100 + i, nx=24 + 8 * i, ny=20 + 8 * i, nz=18 + 8 * i, S=2, n_agents=300, steps=1)
           for i in range(3)]
    batch = Batch("fp64")
    batch.set_schedule(mode=2, graph_steps=4)
    batch.set_direct_threshold(20000)  # the two larger members step directly
    mes = [Microenvironment.from_workload(wl) for wl in wls]
    for me in mes:
        batch.add(me)
    assert batch.get_direct_threshold() == 20000
    batch.step(1, sources=True)
    batch.synchronize()
    per_step = 3 + 2 * 4  # three batched sweeps, two members x (sources + 3 sweeps)
    for n in (1, 8):
        before = kernel_launches()
        batch.step(n, sources=True)
        batch.synchronize()
        assert kernel_launches() - before == n * per_step
    batch.close()
