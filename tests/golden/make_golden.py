"""Generate the golden fixtures for the diffusion-decay path from the
reference itself.

The reference ships no numeric fixtures for this path, so these are made by
running the reference's own BioFVM code -- compiled from its sources by
oracle/Makefile into oracle/_ref/libbiofvm_ref.so (single MPI rank, one
OpenMP thread for the agent loop) -- on seeded synthetic workloads:

  step = simulate_cell_sources_and_sinks(dt)            (1 thread)
         diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING

Small cases store their inputs and the final field in full; large cases
store hashes of their inputs and of the final field bytes (SHA-256 of the
float64 array), per-substrate sums and a fixed sample of voxels.

Run from the repository root (needs the reference sources):
    make -C oracle ref && python tests/golden/make_golden.py
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


def small_cases():
    cases = []
    for seed in range(10):
        cases.append(("small", dict(seed=seed, steps=4, stack=(seed % 3 == 0))))
    cases.append(("small", dict(seed=100, nx=1, ny=5, nz=7, S=2, n_agents=5, steps=3)))
    cases.append(("small", dict(seed=101, nx=9, ny=1, nz=1, S=3, n_agents=4, steps=3)))
    cases.append(("small", dict(seed=102, nx=33, ny=17, nz=40, S=3, n_agents=200, steps=5, stack=True)))
    cases.append(("small", dict(seed=103, nx=2, ny=2, nz=2, S=1, n_agents=0, steps=6)))
    cases.append(("small", dict(seed=104, nx=24, ny=130, nz=3, S=2, n_agents=50, steps=3, agent_mode="gauss")))
    return cases


def build(kind, kw):
    if kind == "small":
        return W.small_random(**kw)
    if kind == "cube50":
        return W.cube50(**kw)
    if kind == "cube200":
        return W.cube200(**kw)
    if kind == "uneven_env":
        return W.uneven_env(**kw)
    raise ValueError(kind)


def run_reference(wl, steps):
    ref = Reference(wl, threads=os.cpu_count() or 1)
    vox = ref.agent_voxels()
    if not np.array_equal(vox, wl.agent_voxel):
        raise SystemExit(f"{wl.name}: reference voxel mapping differs from the workload's")
    c1, c2, e2 = ref.agent_constants(wl.dt) if wl.n_agents else (np.zeros((0, wl.S)),) * 3
    final = ref.run(steps, solver=0, sources_threads=1)
    ref.close()
    return final, c1, c2, e2


def main():
    manifest = []
    for idx, (kind, kw) in enumerate(small_cases()):
        wl = build(kind, kw)
        final, c1, c2, e2 = run_reference(wl, wl.steps)
        name = f"small_{idx:02d}"
        np.savez_compressed(os.path.join(OUT, name + ".npz"), meta=json.dumps({"kind": kind, "kw": kw}),
                            shape=np.array(wl.shape), dx=wl.dx, dt=wl.dt, steps=wl.steps, D=wl.D, decay=wl.decay,
                            active=wl.dirichlet_active, face_values=wl.face_values, field0=wl.field0,
                            voxel=wl.agent_voxel, volume=wl.agent_volume, secretion=wl.secretion, uptake=wl.uptake,
                            saturation=wl.saturation, net_export=wl.net_export, c1=c1, c2=c2, e2=e2, final=final)
        manifest.append(name)
        print(name, wl.shape, wl.n_agents, "agents")

    big = [("cube50", dict(steps=1000)), ("cube200", dict(steps=10)), ("uneven_env", dict(index=7, steps=50))]
    rng = np.random.Generator(np.random.PCG64(2024))
    for kind, kw in big:
        wl = build(kind, kw)
        final, c1, c2, e2 = run_reference(wl, wl.steps)
        sample = np.sort(rng.choice(final.size, size=min(4096, final.size), replace=False))
        name = f"{kind}_{wl.steps}"
        np.savez_compressed(os.path.join(OUT, name + ".npz"), meta=json.dumps({"kind": kind, "kw": kw}),
                            shape=np.array(wl.shape), steps=wl.steps, field0_sha=sha(wl.field0),
                            voxel_sha=sha(wl.agent_voxel), c1_sha=sha(c1), c2_sha=sha(c2), e2_sha=sha(e2),
                            final_sha=sha(final), sums=final.reshape(-1, wl.S).sum(axis=0), sample_idx=sample,
                            sample_val=final[sample])
        manifest.append(name)
        print(name, wl.shape, wl.n_agents, "agents", sha(final)[:16])
    with open(os.path.join(OUT, "MANIFEST.json"), "w") as fh:
        json.dump({"cases": manifest, "generator": "tests/golden/make_golden.py",
                   "oracle": "oracle/_ref/libbiofvm_ref.so (reference BioFVM sources, single rank)"}, fh, indent=1)


if __name__ == "__main__":
    main()
