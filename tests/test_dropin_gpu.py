"""The C++ drop-in inside the reference's own Microenvironment.

oracle/_ref/libbiofvm_dropin.so is the reference BioFVM built from its
sources plus physicell-x_b200/host/biofvm_b200_dropin.cpp, which defines the
reference's declared friend entry point
diffusion_decay_solver__constant_coefficients_LOD_3D(M, dt, world, cart).
The tests install it in the solver slot (diffusion_decay_solver_mpi) and call
Microenvironment::simulate_diffusion_decay(dt, world, cart) exactly as
PhysiCell-X does, then compare with the reference's _BLOCKING solver on an
identical Microenvironment.
"""
import numpy as np
import pytest

from bfvm import workloads as W
from pyoracle import Reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not Reference.available(dropin=True), reason="drop-in library not built")]


def _pair(wl):
    cpu = Reference(wl, threads=4, dropin=True)
    gpu = Reference(wl, threads=4, dropin=True)
    return cpu, gpu


@pytest.mark.parametrize("seed", [401, 402, 403])
def test_dropin_solver_slot_bitwise(seed):
    """Host-side sources (the reference's own agent loop), GPU diffusion through
    the solver pointer, field mirrored to the host every step."""
    wl = W.small_random(seed, steps=4, stack=True)
    cpu, gpu = _pair(wl)
    a = cpu.run(wl.steps, solver=0, sources_threads=1)
    b = gpu.run(wl.steps, solver=2, sources_threads=1)
    assert np.array_equal(a, b)


def test_dropin_fused_sources_bitwise():
    """Agents gathered from the reference's Basic_Agent list and applied on the
    GPU fused ahead of the sweep; the host agent loop is not called."""
    wl = W.small_random(404, nx=30, ny=22, nz=26, S=3, n_agents=500, steps=5, stack=True)
    cpu, gpu = _pair(wl)
    a = cpu.run(wl.steps, solver=0, sources_threads=1)
    assert gpu.L.ref_env_dropin_fuse_sources(gpu.h, 1, wl.dt) == 0
    for _ in range(wl.steps):
        gpu.diffusion(solver=2)
    assert np.array_equal(a, gpu.field())


def test_dropin_fused_sources_track_internalized():
    """track_internalized_substrates_in_each_agent on: the drop-in carries each
    Basic_Agent's internalized_substrates through the fused GPU stage and
    writes them back; field and amounts equal the reference's host loop."""
    wl = W.small_random(406, nx=19, ny=15, nz=13, S=3, n_agents=300, steps=4, stack=True)
    assert np.any(wl.net_export != 0)
    cpu, gpu = _pair(wl)
    cpu.set_tracking(True)
    try:
        a = cpu.run(wl.steps, solver=0, sources_threads=1)
        a_in = cpu.internalized()
        assert gpu.L.ref_env_dropin_fuse_sources(gpu.h, 1, wl.dt) == 0
        for _ in range(wl.steps):
            gpu.diffusion(solver=2)
        b_in = gpu.internalized()
    finally:
        cpu.set_tracking(False)
    assert np.any(a_in != 0)
    assert np.array_equal(a, gpu.field())
    assert np.array_equal(a_in, b_in)


def test_dropin_cube50_hundred_steps():
    wl = W.cube50(steps=100)
    cpu, gpu = _pair(wl)
    a = cpu.run(wl.steps, solver=0, sources_threads=1)
    b = gpu.run(wl.steps, solver=2, sources_threads=1)
    assert np.array_equal(a, b)


def test_dropin_follows_dirichlet_changes_between_steps():
    wl = W.small_random(405, steps=2)
    cpu, gpu = _pair(wl)
    for ref in (cpu, gpu):
        ref.run(2, solver=0 if ref is cpu else 2)
        for d in range(wl.S):
            ref.L.ref_env_set_dirichlet_activation(ref.h, d, 1)
        dv = wl.dirichlet_values * 0.5
        ref.L.ref_env_set_dirichlet_face_values(ref.h, dv)
    a = cpu.run(3, solver=0)
    b = gpu.run(3, solver=2)
    assert np.array_equal(a, b)


def test_dropin_keeps_first_dt_like_the_reference():
    """The reference factors its Thomas systems on its first call only
    (diffusion_solver_setup_done, BioFVM_solvers.cpp:125,335) and keeps that
    call's dt afterwards; the drop-in keeps it too, so calls with another dt
    still give the reference's bits."""
    wl = W.small_random(407, steps=2)
    cpu, gpu = _pair(wl)
    for ref, solver in ((cpu, 0), (gpu, 2)):
        ref.diffusion(solver=solver)
        for dt in (wl.dt * 2.0, wl.dt * 0.5):
            with __import__("pyoracle")._stdout_to_stderr():
                assert ref.L.ref_env_diffusion(ref.h, dt, solver, 4) == 0
    assert np.array_equal(cpu.field(), gpu.field())
