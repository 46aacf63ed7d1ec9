"""The oracle against the golden fixtures of the calls around the step
(tests/golden/make_golden_ext.py: outputs of the reference's own BioFVM code
for internalized-substrate tracking and release, Dirichlet nodes, the 2-D LOD
solver, gradients, bulk sources, and the MATLAB density file byte for byte),
bit for bit, without the reference tree.
Each fixture's workload is regenerated from its stored parameters and checked
against the stored hash of its initial field first."""
import dataclasses
import hashlib
import json
import os

import numpy as np
import pytest

from pyoracle import Port
from bfvm import workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = json.load(open(os.path.join(GOLD, "MANIFEST_EXT.json")))["cases"]


def _load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    kw = json.loads(str(z["meta"]))["kw"]
    repl = kw.pop("replace", None)
    wl = W.small_random(**kw)
    assert hashlib.sha256(np.ascontiguousarray(wl.field0).tobytes()).hexdigest() == str(z["field0_sha"]), name
    if repl:
        wl = dataclasses.replace(wl, dx=repl["dx"], origin=tuple(repl["origin"]))
    return z, wl


def _check_tracking(z, wl):
    f = wl.field0.copy()
    c1, c2, e2 = Port.workload_constants(wl)
    internal = np.zeros((wl.n_agents, wl.S))
    V = wl.dx ** 3
    for _ in range(wl.steps):
        Port.sources_tracked(f, wl.S, wl.agent_voxel, c1, c2, e2, wl.net_export * wl.dt, V, internal)
        Port.lod_step(f, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, wl.dirichlet_values)
    assert np.any(z["internal"] != 0)
    assert np.array_equal(f, z["final"])
    assert np.array_equal(internal, z["internal"])


def _check_release(z, wl):
    f = wl.field0.copy()
    internal = z["amounts"].copy()
    Port.release_internalized(f, wl.S, z["agents"], wl.agent_voxel, z["fraction"], wl.dx ** 3, internal)
    assert np.array_equal(f, z["final"])
    assert np.array_equal(internal, z["internal"])


def _check_nodes(z, wl):
    f = Port.dirichlet_nodes(wl.field0.copy(), wl.S, z["voxel"], z["values"], z["activation"])
    assert np.array_equal(f, z["final"])


def _check_lod2d(z, wl):
    f = wl.field0.copy()
    n = wl.nx
    for _ in range(wl.steps):
        Port.lod2d_step(f, n, 1, 1, wl.D, wl.decay, wl.dt, wl.dx, np.arange(n), z["values"], z["activation"])
    assert not np.array_equal(f, wl.field0)
    assert np.array_equal(f, z["final"])


def _check_gradients(z, wl):
    assert np.array_equal(Port.run(wl), z["field"])
    assert np.array_equal(Port.gradients(z["field"], wl.shape, wl.dx), z["gradients"])


def _check_bulk(z, wl):
    f = wl.field0.copy()
    Port.bulk_sources(f, wl.dt, z["supply"], z["target"], z["uptake"])
    assert np.array_equal(f, z["final"])


def _check_matlab(z, wl, tmp):
    path = os.path.join(tmp, "p.mat")
    Port.write_matlab(path, z["field"], wl.shape, wl.origin, wl.dx)
    raw = open(path, "rb").read()
    assert len(raw) == int(z["file_size"])
    assert hashlib.sha256(raw).hexdigest() == str(z["file_sha"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden_extension(name, tmp_path):
    z, wl = _load(name)
    kind = name.split("_")[1]
    if kind == "matlab":
        _check_matlab(z, wl, str(tmp_path))
        return
    {"tracking": _check_tracking, "release": _check_release, "nodes": _check_nodes, "lod2d": _check_lod2d,
     "gradients": _check_gradients, "bulk": _check_bulk}[kind](z, wl)
