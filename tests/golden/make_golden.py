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
    python tests/golden/make_golden.py --only cube200_500 cube640_slabx_5

The full-size cube640 case (640^3 voxels, 2 substrates, 1,000,000 Gaussian
agents, 5 steps) is made only when asked for by name (--only cube640_5): the
reference keeps several heap objects per voxel (mesh voxels, gradient and
Dirichlet vectors), about 650 bytes per voxel, so it needs a host with some
200 GB of memory.  --oracle port makes that case with the C restatement
(oracle/lod3d_oracle.c) instead; the fixture records which oracle made it.
The cube640_slab cases pin the reference itself on cube640's 640-voxel lines
along each axis.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import zlib

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
    if kind == "cube640_slab":
        return W.cube640_slab(**kw)
    if kind == "cube640":
        return W.cube640(**kw)
    raise ValueError(kind)


# Large cases: hashes, sums and a sample of the final field.  The first three
# were generated with one sample generator shared in this order; the later
# ones draw their sample from a generator seeded by the case's name.
BIG = [("cube50", dict(steps=1000)), ("cube200", dict(steps=10)), ("uneven_env", dict(index=7, steps=50))]
BIG_NAMED = [("cube200", dict(steps=500)), ("cube640_slab", dict(axis=0)), ("cube640_slab", dict(axis=1)),
             ("cube640_slab", dict(axis=2))]
ON_REQUEST = [("cube640", dict(steps=5))]


def big_name(kind, wl):
    return f"{wl.name}_{wl.steps}" if kind == "cube640_slab" else f"{kind}_{wl.steps}"


def run_port(wl, steps):
    """The same steps with the C restatement (agents in list order)."""
    from pyoracle import Port

    c1, c2, e2 = Port.workload_constants(wl)
    field = wl.field0.copy()
    dv = wl.dirichlet_values
    for _ in range(steps):
        Port.sources(field, wl.S, wl.agent_voxel, c1, c2, e2)
        Port.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv, os.cpu_count() or 1)
    return field, c1, c2, e2


def save_big(name, kind, kw, wl, final, c1, c2, e2, rng, oracle):
    sample = np.sort(rng.choice(final.size, size=min(4096, final.size), replace=False))
    np.savez_compressed(os.path.join(OUT, name + ".npz"), meta=json.dumps({"kind": kind, "kw": kw, "oracle": oracle}),
                        shape=np.array(wl.shape), steps=wl.steps, field0_sha=sha(wl.field0),
                        voxel_sha=sha(wl.agent_voxel), c1_sha=sha(c1), c2_sha=sha(c2), e2_sha=sha(e2),
                        final_sha=sha(final), sums=final.reshape(-1, wl.S).sum(axis=0), sample_idx=sample,
                        sample_val=final[sample])
    print(name, wl.shape, wl.n_agents, "agents", sha(final)[:16], "by", oracle, flush=True)


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
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None, help="case names to (re)generate; default: all but "
                    "the on-request cases")
    ap.add_argument("--oracle", choices=["reference", "port"], default="reference",
                    help="what makes the on-request cases (the others always come from the reference)")
    args = ap.parse_args()
    only = set(args.only) if args.only else None
    mpath = os.path.join(OUT, "MANIFEST.json")
    manifest = []
    if only is not None and os.path.exists(mpath):
        with open(mpath) as fh:
            manifest = json.load(fh)["cases"]

    def want(name):
        return only is None or name in only

    def note(name):
        if name not in manifest:
            manifest.append(name)

    for idx, (kind, kw) in enumerate(small_cases()):
        name = f"small_{idx:02d}"
        if not want(name):
            continue
        wl = build(kind, kw)
        final, c1, c2, e2 = run_reference(wl, wl.steps)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), meta=json.dumps({"kind": kind, "kw": kw}),
                            shape=np.array(wl.shape), dx=wl.dx, dt=wl.dt, steps=wl.steps, D=wl.D, decay=wl.decay,
                            active=wl.dirichlet_active, face_values=wl.face_values, field0=wl.field0,
                            voxel=wl.agent_voxel, volume=wl.agent_volume, secretion=wl.secretion, uptake=wl.uptake,
                            saturation=wl.saturation, net_export=wl.net_export, c1=c1, c2=c2, e2=e2, final=final)
        note(name)
        print(name, wl.shape, wl.n_agents, "agents")

    rng = np.random.Generator(np.random.PCG64(2024))
    for kind, kw in BIG:
        wl = build(kind, kw)
        name = big_name(kind, wl)
        if not want(name):
            # keep the shared sample generator in step with a full run
            rng.choice(wl.n_values, size=min(4096, wl.n_values), replace=False)
            continue
        final, c1, c2, e2 = run_reference(wl, wl.steps)
        save_big(name, kind, kw, wl, final, c1, c2, e2, rng, "reference")
        note(name)
    for kind, kw in BIG_NAMED + ON_REQUEST:
        wl = build(kind, kw)
        name = big_name(kind, wl)
        on_request = (kind, kw) in ON_REQUEST
        if (on_request and (only is None or name not in only)) or not want(name):
            continue
        oracle = args.oracle if on_request else "reference"
        if oracle == "reference":
            final, c1, c2, e2 = run_reference(wl, wl.steps)
        else:
            final, c1, c2, e2 = run_port(wl, wl.steps)
        own = np.random.Generator(np.random.PCG64(zlib.crc32(name.encode())))
        save_big(name, kind, kw, wl, final, c1, c2, e2, own, oracle)
        note(name)
    with open(mpath, "w") as fh:
        json.dump({"cases": manifest, "generator": "tests/golden/make_golden.py",
                   "oracle": "oracle/_ref/libbiofvm_ref.so (reference BioFVM sources, single rank); a case's "
                             "meta names another oracle where one made it"}, fh, indent=1)


if __name__ == "__main__":
    main()
