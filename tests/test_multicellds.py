"""MultiCellDS output of the microenvironment (add_BioFVM_substrates_to_open_xml_pugi,
BioFVM/BioFVM_MultiCellDS.cpp:518-823; save_BioFVM_to_MultiCellDS_xml_pugi,
:1880-1890; General_Mesh::write_to_matlab, BioFVM/BioFVM_mesh.cpp:425-447).

The reference builds its document once per process into a global, so each
reference document is made in a fresh Python process.  GPU: the XML
document and both MATLAB files written from the device equal the
reference's byte for byte, names with XML special characters included."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import pyoracle
from bfvm import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [
    dict(seed=1, shape=(4, 3, 2, 2), domain="oracle", mesh_units="none", spatial_units="none", time_units="none",
         names=["s0", "s1"], units=["none", "none"]),
    dict(seed=2, shape=(23, 17, 9, 3), domain="tumor & <stroma>", mesh_units="micron", spatial_units="micron",
         time_units="min", names=['oxygen "O2"', "drug<A>&B", "tab\there"], units=["mmHg", "mol/L", "dimensionless"]),
    dict(seed=3, shape=(61, 5, 40, 1), domain="x", mesh_units="m", spatial_units="m", time_units="s",
         names=["z'"], units=["line\nfeed"]),
]

_CHILD = r"""
import json, sys
sys.path[:0] = [sys.argv[1] + "/physicell-x_b200", sys.argv[1] + "/oracle"]
import pyoracle
from bfvm import workloads as W
c = json.loads(sys.argv[2])
nx, ny, nz, S = c["shape"]
wl = W.small_random(c["seed"], nx=nx, ny=ny, nz=nz, S=S, n_agents=0, steps=1)
ref = pyoracle.Reference(wl, threads=1)
text = ref.multicellds_substrates(c["base"], c["domain"], c["mesh_units"], c["spatial_units"], c["time_units"],
                                  c["names"], c["units"])
sys.stdout.write(json.dumps({"xml": text, "bb": list(ref.bounding_box())}))
"""


def _reference(case, base):
    c = dict(case, base=str(base))
    out = subprocess.run([sys.executable, "-c", _CHILD, ROOT, json.dumps(c)], capture_output=True, text=True,
                         timeout=120, check=True)
    return json.loads(out.stdout)


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
def test_reference_document_is_deterministic(tmp_path):
    """The pinned part of the document: two reference processes on the same
    inputs write the same text and files."""
    a = _reference(CASES[1], tmp_path / "a")
    b = _reference(CASES[1], tmp_path / "b")
    assert b["xml"].replace("b_mesh0", "a_mesh0").replace("b_microenvironment0", "a_microenvironment0") == a["xml"]
    for suffix in ("_mesh0.mat", "_microenvironment0.mat"):
        assert (tmp_path / ("a" + suffix)).read_bytes() == (tmp_path / ("b" + suffix)).read_bytes()


@pytest.mark.gpu
@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
@pytest.mark.parametrize("case", CASES, ids=["plain", "escapes", "thin"])
def test_gpu_multicellds_matches_reference_bytes(case, tmp_path):
    from bfvm import Microenvironment

    want = _reference(case, tmp_path / "ref")
    nx, ny, nz, S = case["shape"]
    wl = W.small_random(case["seed"], nx=nx, ny=ny, nz=nz, S=S, n_agents=0, steps=1)
    me = Microenvironment.from_workload(wl)
    base = tmp_path / "gpu"
    text = me.write_multicellds(base, want["bb"], case["names"], case["units"], domain_name=case["domain"],
                                mesh_units=case["mesh_units"], spatial_units=case["spatial_units"],
                                time_units=case["time_units"])
    me.close()
    assert text == want["xml"].replace("ref_mesh0", "gpu_mesh0").replace("ref_microenvironment0",
                                                                         "gpu_microenvironment0")
    for suffix in ("_mesh0.mat", "_microenvironment0.mat"):
        assert (tmp_path / ("gpu" + suffix)).read_bytes() == (tmp_path / ("ref" + suffix)).read_bytes(), suffix
