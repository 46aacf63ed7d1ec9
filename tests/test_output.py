"""Density output in the reference's MATLAB v4 format
(Microenvironment::write_to_matlab, BioFVM/BioFVM_microenvironment.cpp:
1222-1249): the oracle writer against the reference build on CPU, the GPU
writer against the oracle byte for byte."""
import dataclasses

import numpy as np
import pytest

import pyoracle
from bfvm import workloads as W


def _read_mat(path):
    raw = open(path, "rb").read()
    hdr = np.frombuffer(raw[:20], np.uint32)
    name = raw[20:20 + int(hdr[4])].decode()
    data = np.frombuffer(raw[20 + int(hdr[4]):], np.float64).reshape(int(hdr[2]), int(hdr[1]))
    return hdr, name, data


def _cases():
    base = W.small_random(3, nx=13, ny=7, nz=9, S=2, n_agents=5, steps=2)
    return [base, dataclasses.replace(base, dx=1.3, origin=(-7.77, 2.9, -0.123))]


@pytest.mark.skipif(not pyoracle.Reference.available(), reason="reference build not present")
def test_oracle_matlab_file_matches_reference(tmp_path):
    for n, wl in enumerate(_cases()):
        ref = pyoracle.Reference(wl, threads=1)
        ref.run(1)
        ref.write_matlab(tmp_path / f"r{n}.mat")
        pyoracle.Port.write_matlab(tmp_path / f"p{n}.mat", ref.field(), wl.shape, wl.origin, wl.dx)
        ref.close()
        assert (tmp_path / f"r{n}.mat").read_bytes() == (tmp_path / f"p{n}.mat").read_bytes()
        hdr, name, data = _read_mat(tmp_path / f"p{n}.mat")
        assert list(hdr) == [0, 4 + wl.S, wl.n_voxels, 0, len("multiscale_microenvironment")]
        assert name == "multiscale_microenvironment"
        assert np.allclose(data[:, 3], wl.dx ** 3)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [0, 1])
def test_gpu_matlab_file_bytewise(tmp_path, n):
    from bfvm import Microenvironment

    wl = _cases()[n]
    me = Microenvironment.from_workload(wl)
    me.simulate_diffusion_decay(wl.steps, sources=True)
    me.write_to_matlab(tmp_path / "g.mat", wl.origin)
    pyoracle.Port.write_matlab(tmp_path / "o.mat", me.download_field(), wl.shape, wl.origin, wl.dx)
    me.close()
    assert (tmp_path / "g.mat").read_bytes() == (tmp_path / "o.mat").read_bytes()


@pytest.mark.gpu
def test_gpu_matlab_file_fp32_and_large(tmp_path):
    from bfvm import Microenvironment

    wl = W.small_random(9, nx=130, ny=90, nz=100, S=3, n_agents=0, steps=1)  # more than one transfer chunk
    m64 = Microenvironment.from_workload(wl, "fp64")
    m32 = Microenvironment.from_workload(wl, "fp32")
    m64.write_to_matlab(tmp_path / "a.mat", wl.origin)
    m32.write_to_matlab(tmp_path / "b.mat", wl.origin)
    ha, _, a = _read_mat(tmp_path / "a.mat")
    hb, _, b = _read_mat(tmp_path / "b.mat")
    assert np.array_equal(ha, hb) and np.array_equal(a[:, :4], b[:, :4])
    assert np.array_equal(a[:, 4:], wl.field0.reshape(-1, wl.S))
    assert np.abs(b[:, 4:] - a[:, 4:]).max() <= 1e-6 * np.abs(a[:, 4:]).max()
    m64.close()
    m32.close()
