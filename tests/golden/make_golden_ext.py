"""Generate golden fixtures for the calls around the diffusion-decay step from
the reference itself: internalized-substrate tracking and release, interior
Dirichlet nodes, the 2-D LOD solver, substrate gradients and bulk sources.

Like make_golden.py, every output here comes from running the reference's own
BioFVM code, compiled from its sources by oracle/Makefile into
oracle/_ref/libbiofvm_ref.so (single MPI rank, one thread for agent loops):

  tracking   track_internalized_substrates_in_each_agent on; steps of
             simulate_cell_sources_and_sinks + the _BLOCKING LOD solver
             (BioFVM_basic_agent.cpp:509-559, BioFVM_solvers.cpp:102-780)
  release    Basic_Agent::release_internalized_substrates (:310-333)
  nodes      add_dirichlet_node / per-voxel set_substrate_dirichlet_activation
             then apply_dirichlet_conditions (BioFVM_microenvironment.cpp:218-323)
  lod2d      diffusion_decay_solver__constant_coefficients_LOD_2D
             (BioFVM_solvers.cpp:1668-1832), one substrate on ny = 1, where
             that solver stays on its lines
  gradients  compute_all_gradient_vectors (BioFVM_microenvironment.cpp:1454-1616)
  bulk       simulate_bulk_sources_and_sinks (:1327-1368)
  matlab     write_to_matlab (:1222-1249): the file's size and SHA-256

Each fixture stores every generated input (node lists, rates, amounts, the
workload's parameters and a hash of its initial field) with the reference's
outputs, so tests/test_golden_ext.py checks the oracle against them without
the reference tree.

Run from the repository root (needs the reference sources):
    make -C oracle ref && python tests/golden/make_golden_ext.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "physicell-x_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from bfvm import workloads as W  # noqa: E402
from pyoracle import Reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def save(name, kw, wl, **arrays):
    np.savez_compressed(os.path.join(OUT, name + ".npz"), meta=json.dumps({"kw": kw}), field0_sha=sha(wl.field0),
                        **arrays)
    print(name, wl.shape, {k: v.shape for k, v in arrays.items() if hasattr(v, "shape")})
    return name


def tracking(seed, stack):
    kw = dict(seed=800 + seed, n_agents=50, steps=3, stack=stack)
    wl = W.small_random(**kw)
    ref = Reference(wl, threads=1)
    try:
        ref.set_tracking(True)
        assert np.array_equal(ref.agent_voxels(), wl.agent_voxel)
        for _ in range(wl.steps):
            ref.sources()
            ref.diffusion()
        final, internal = ref.field(), ref.internalized()
    finally:
        ref.set_tracking(False)
        ref.close()
    return save(f"ext_tracking_{seed}", kw, wl, final=final, internal=internal)


def release():
    kw = dict(seed=811, n_agents=40, steps=1, stack=True)
    wl = W.small_random(**kw)
    rng = np.random.default_rng(5)
    amounts = rng.uniform(-3e4, 3e4, (wl.n_agents, wl.S))
    agents = rng.permutation(wl.n_agents)[:25]
    fraction = rng.uniform(0.0, 1.0, (agents.size, wl.S))
    ref = Reference(wl, threads=1)
    try:
        ref.set_internalized(amounts)
        ref.release(agents, fraction)
        final, internal = ref.field(), ref.internalized()
    finally:
        ref.close()
    return save("ext_release", kw, wl, amounts=amounts, agents=agents, fraction=fraction, final=final,
                internal=internal)


def _face_nodes(wl):
    """Every face voxel with its face value and each substrate's activation
    (what the reference holds after its faces are set)."""
    nx, ny, nz, S = wl.shape
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    face = (i == 0) | (i == nx - 1) | (j == 0) | (j == ny - 1) | (k == 0) | (k == nz - 1)
    vox = ((i * ny + j) * nz + k)[face].ravel()
    vals = wl.dirichlet_values.reshape(-1, S)[vox]
    act = np.tile(np.asarray(wl.dirichlet_active, np.uint8), (vox.size, 1))
    return {int(v): [vals[q].copy(), act[q].copy()] for q, v in enumerate(vox)}


def nodes(seed):
    kw = dict(seed=910 + seed, n_agents=0, steps=1)
    wl = W.small_random(**kw)
    nx, ny, nz, S = wl.shape
    rng = np.random.default_rng(seed)
    table = _face_nodes(wl)
    ref = Reference(wl, threads=1)
    try:
        for v in rng.choice(nx * ny * nz, 12, replace=False):
            val = rng.uniform(0.0, 60.0, S)
            act = table[int(v)][1] if int(v) in table else np.asarray(wl.dirichlet_active, np.uint8).copy()
            table[int(v)] = [val, act.copy()]
            ref.add_dirichlet_node(int(v), val)
        for v in rng.choice(sorted(table), max(1, len(table) // 4), replace=False):
            s = int(rng.integers(0, S))
            on = bool(rng.integers(0, 2))
            table[int(v)][1][s] = 1 if on else 0
            ref.set_node_activation(int(v), s, on)
        ref.apply_dirichlet_conditions()
        final = ref.field()
    finally:
        ref.close()
    vox = np.array(sorted(table), np.int32)
    vals = np.array([table[v][0] for v in vox], np.float64).reshape(-1, S)
    act = np.array([table[v][1] for v in vox], np.uint8).reshape(-1, S)
    return save(f"ext_nodes_{seed}", kw, wl, voxel=vox, values=vals, activation=act, final=final)


def lod2d(seed):
    kw = dict(seed=930 + seed, nx=30 + 7 * seed, ny=1, nz=1, S=1, n_agents=0, steps=5)
    wl = W.small_random(**kw)
    wl.dirichlet_active[:] = 1
    n = wl.nx
    rng = np.random.default_rng(seed)
    keep = set(rng.choice(n, 4, replace=False).tolist())
    act = np.ones((n, 1), np.uint8)
    ref = Reference(wl, threads=1)
    try:
        for v in range(n):
            if v not in keep:
                ref.set_node_activation(v, 0, False)
                act[v, 0] = 0
        for _ in range(wl.steps):
            ref.lod2d()
        final = ref.field()
    finally:
        ref.close()
    return save(f"ext_lod2d_{seed}", kw, wl, activation=act, values=wl.dirichlet_values.reshape(n, 1).copy(),
                final=final)


def gradients(i, shape):
    nx, ny, nz, S = shape
    kw = dict(seed=500 + i, nx=nx, ny=ny, nz=nz, S=S, n_agents=20, steps=2)
    wl = W.small_random(**kw)
    ref = Reference(wl, threads=2)
    try:
        field = ref.run(2)
        grad = ref.gradients()
    finally:
        ref.close()
    return save(f"ext_gradients_{i}", kw, wl, field=field, gradients=grad)


def bulk(seed):
    kw = dict(seed=600 + seed, n_agents=0, steps=1)
    wl = W.small_random(**kw)
    rng = np.random.default_rng(seed)
    n = wl.n_values
    supply, target, uptake = rng.uniform(0, 5, n), rng.uniform(0, 40, n), rng.uniform(0, 3, n)
    ref = Reference(wl, threads=1)
    try:
        ref.bulk_sources(supply, target, uptake)
        final = ref.field()
    finally:
        ref.close()
    return save(f"ext_bulk_{seed}", kw, wl, supply=supply, target=target, uptake=uptake, final=final)


def matlab(i):
    """Microenvironment::write_to_matlab (BioFVM_microenvironment.cpp:1222-1249)
    after one step: the field it wrote from, and the file's size and hash."""
    import dataclasses
    import tempfile

    kw = dict(seed=3, nx=13, ny=7, nz=9, S=2, n_agents=5, steps=1)
    wl = W.small_random(**kw)
    repl = [{}, {"dx": 1.3, "origin": [-7.77, 2.9, -0.123]}][i]
    if repl:
        wl = dataclasses.replace(wl, dx=repl["dx"], origin=tuple(repl["origin"]))
    ref = Reference(wl, threads=1)
    try:
        ref.run(1)
        field = ref.field()
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "r.mat")
            ref.write_matlab(path)
            raw = open(path, "rb").read()
    finally:
        ref.close()
    kw["replace"] = repl
    return save(f"ext_matlab_{i}", kw, W.small_random(**{k: v for k, v in kw.items() if k != "replace"}),
                field=field, file_sha=hashlib.sha256(raw).hexdigest(), file_size=len(raw))


CASES = ([("tracking", (seed, stack)) for seed, stack in ((1, False), (2, True), (3, True))] + [("release", ())] +
         [("nodes", (seed,)) for seed in (0, 1, 2)] + [("lod2d", (seed,)) for seed in (0, 1, 2, 3)] +
         # every axis at least 2 long: the reference reads outside its array otherwise
         [("gradients", (i, shape)) for i, shape in enumerate([(9, 7, 5, 2), (2, 3, 4, 1), (33, 20, 12, 3)])] +
         [("bulk", (seed,)) for seed in (1, 2, 3)] + [("matlab", (i,)) for i in (0, 1)])


def main():
    """Each case runs in a process of its own: the reference keeps state
    across calls in one process (its gradient routine caches 2*dx in function
    statics on the first call), which must not leak from one case into the
    next."""
    import subprocess

    names = []
    for idx in range(len(CASES)):
        out = subprocess.run([sys.executable, os.path.abspath(__file__), str(idx)], capture_output=True, text=True,
                             check=True).stdout
        name = [ln for ln in out.splitlines() if ln.startswith("ext_")][-1].split()[0]
        print(name)
        names.append(name)
    with open(os.path.join(OUT, "MANIFEST_EXT.json"), "w") as fh:
        json.dump({"cases": names, "generator": "tests/golden/make_golden_ext.py",
                   "oracle": "oracle/_ref/libbiofvm_ref.so (reference BioFVM sources, single rank)"}, fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        fn, args = CASES[int(sys.argv[1])]
        globals()[fn](*args)
    else:
        main()
