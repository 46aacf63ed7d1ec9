"""CPU tests of the C ABI library: it loads, exports every function that
include/biofvm_b200.h declares, and reports a missing device instead of
failing silently.  No compute call is made here."""
import ctypes as C
import os
import re

import pytest

from bfvm import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bfvm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = _lib.lib()
    names = _declared("biofvm_b200.h")
    assert "bfvm_create" in names and "bfvm_step" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    names = _declared("biofvm_b200.h")
    assert sorted(n for n in names if n in _lib._SIGS) == names


def test_status_strings():
    assert _lib.status_string(0) == "ok"
    assert _lib.status_string(_lib.BFVM_ERR_TIMEOUT) == "device wait timed out"


def _cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_cuda_available(), reason="checks the no-device path")
def test_create_without_device_reports_nodevice():
    L = _lib.lib()
    D = (C.c_double * 1)(1e5)
    lam = (C.c_double * 1)(0.1)
    cfg = _lib.bfvm_config(4, 4, 4, 1, 20.0, 0.01, D, lam, _lib.BFVM_FP64, 0)
    h = C.c_void_p()
    assert L.bfvm_create(C.byref(cfg), C.byref(h)) == _lib.BFVM_ERR_NODEVICE
    assert not h.value


def test_create_rejects_bad_arguments():
    L = _lib.lib()
    D = (C.c_double * 1)(1e5)
    lam = (C.c_double * 1)(0.1)
    h = C.c_void_p()
    for bad in (dict(nx=0), dict(dx=-1.0), dict(dt=0.0), dict(precision=7)):
        kw = dict(nx=4, ny=4, nz=4, S=1, dx=20.0, dt=0.01, precision=_lib.BFVM_FP64)
        kw.update(bad)
        cfg = _lib.bfvm_config(kw["nx"], kw["ny"], kw["nz"], kw["S"], kw["dx"], kw["dt"], D, lam, kw["precision"], 0)
        assert L.bfvm_create(C.byref(cfg), C.byref(h)) == _lib.BFVM_ERR_ARG
    assert L.bfvm_create(None, C.byref(h)) == _lib.BFVM_ERR_ARG


def _plan(axis, n, level=1):
    L = _lib.lib()
    a, b, c = C.c_int(-1), C.c_int(-1), C.c_int(-1)
    assert L.bfvm_tmem_sweep_plan(axis, n, level, C.byref(a), C.byref(b), C.byref(c)) == _lib.BFVM_OK
    return a.value, b.value, c.value


def test_tmem_sweep_plan():
    """The tensor-memory sweep configurations (shared-memory rings, TMEM
    rings, input slots per TMEM ring) chosen per line length: those measured
    on B200 (y/z: 3 + 4 rings at lines of 200, fewer shared-memory rings as
    lines grow, TMEM rings partly resident past 256, the forward coefficient
    pairs staged in shared memory where that costs no ring; x by default from
    33, at level 2 from 17), two input slots where a third would cost a ring
    (or the staged pairs), and where the
    shared-memory schedules take over (y/z lines under 3 chunks of 16 rows,
    x lines under 2 at level 2, any line past 736 = 46 chunks, whose 30
    resident chunks and 2 input slots fill a ring's 32 slots); and the FP32
    sweeps' (axis 2 y/z: up to 3 shared-memory and 8 TMEM rings, two per
    lane quarter; axis 3 x: TMEM rings only, up to 8, 32-value chunks, 8
    of them in a ring's TMEM columns)."""
    yz = {33: (3, 4, 3), 40: (3, 4, 3), 200: (3, 4, 2), 210: (3, 4, 2), 256: (2, 4, 3), 300: (1, 4, 3),
          400: (0, 4, 2), 500: (0, 2, 3), 640: (0, 2, 3), 650: (0, 2, 2), 657: (0, 1, 3), 700: (0, 1, 3),
          720: (0, 1, 3), 736: (0, 1, 2), 32: (0, 0, 0), 737: (0, 0, 0), 800: (0, 0, 0)}
    for n, want in yz.items():
        assert _plan(1, n) == want, n
        assert _plan(1, n, 0) == (0, 0, 0), n
    x1 = {32: (0, 0, 0), 33: (3, 4, 3), 200: (3, 4, 2), 256: (2, 4, 3), 257: (2, 4, 3), 300: (1, 4, 3),
          400: (0, 4, 3), 640: (0, 2, 2), 700: (0, 1, 3), 736: (0, 1, 2), 737: (0, 0, 0), 800: (0, 0, 0)}
    for n, want in x1.items():
        assert _plan(0, n) == want, n
    x2 = {17: (3, 4, 2), 20: (3, 4, 2), 200: (3, 4, 2), 256: (2, 4, 3), 640: (0, 2, 2), 16: (0, 0, 0)}
    for n, want in x2.items():
        assert _plan(0, n, 2) == want, n
    L = _lib.lib()
    a = C.c_int()
    f32 = {32: (0, 0, 0), 33: (3, 8, 3), 200: (3, 8, 3), 256: (3, 8, 3), 257: (3, 8, 3), 300: (3, 8, 2),
           400: (0, 8, 3), 512: (0, 5, 2), 640: (0, 3, 3), 736: (0, 3, 2), 737: (0, 0, 0)}
    for n, want in f32.items():
        assert _plan(2, n) == want, n
        assert _plan(2, n, 0) == (0, 0, 0), n
    fx32 = {32: (0, 0, 0), 33: (0, 8, 2), 200: (0, 8, 3), 256: (0, 8, 3), 257: (0, 8, 3), 300: (0, 8, 3),
            400: (0, 7, 2), 640: (0, 3, 3), 1024: (0, 1, 3), 1216: (0, 1, 2), 1217: (0, 0, 0)}
    for n, want in fx32.items():
        assert _plan(3, n) == want, n
        assert _plan(3, n, 2) == want, n
        assert _plan(3, n, 0) == (0, 0, 0), n
    for args in ((4, 100, 1), (-1, 100, 1), (1, 0, 1), (1, 100, 3), (0, 100, -1)):
        assert L.bfvm_tmem_sweep_plan(*args, C.byref(a), C.byref(a), C.byref(a)) == _lib.BFVM_ERR_ARG
    assert L.bfvm_tmem_sweep_plan(1, 100, 1, None, C.byref(a), C.byref(a)) == _lib.BFVM_ERR_ARG


# entry points that return a value rather than a status: what a NULL handle gives
_NULL_VALUES = {"bfvm_stream": None, "bfvm_batch_stream": None, "bfvm_device_bytes": 0, "bfvm_batch_size": 0}


def test_null_handles_are_rejected_before_any_device_work():
    """Every entry point that takes a solve or batch handle first returns
    BFVM_ERR_ARG for a NULL handle (zero and NULL for its other arguments),
    without touching a device; the value-returning ones give NULL or 0."""
    L = _lib.lib()
    seen = 0
    for name, (_, args) in _lib._SIGS.items():
        if not args or args[0] is not C.c_void_p:
            continue
        vals = [0 if issubclass(a, C._SimpleCData) and a not in (C.c_void_p, C.c_char_p) else None for a in args]
        got = getattr(L, name)(*vals)
        assert got == _NULL_VALUES.get(name, _lib.BFVM_ERR_ARG), name
        seen += 1
    assert seen >= 50


def test_wait_limit_arguments_checked_first():
    """The wait-limit setter rejects limits outside [1 us, 60 s] before it
    looks for a device."""
    L = _lib.lib()
    assert L.bfvm_set_wait_limit_ns(0, 999) == _lib.BFVM_ERR_ARG
    assert L.bfvm_set_wait_limit_ns(0, 60_000_000_001) == _lib.BFVM_ERR_ARG
    if not _cuda_available():
        assert L.bfvm_set_wait_limit_ns(0, 1_000_000) == _lib.BFVM_ERR_NODEVICE
