"""Loader for libbiofvm_b200.so (the C ABI in include/biofvm_b200.h).

There is no CPU fallback: if the library is missing or cannot be loaded the
import of :mod:`bfvm` fails with an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libbiofvm_b200.so")

BFVM_OK = 0
BFVM_ERR_ARG = -1
BFVM_ERR_CUDA = -2
BFVM_ERR_OOM = -3
BFVM_ERR_SHAPE = -4
BFVM_ERR_NODEVICE = -5
BFVM_ERR_TIMEOUT = -6
BFVM_ERR_STATE = -7

BFVM_FP64 = 0
BFVM_FP32 = 1
BFVM_STEP_SOURCES = 1

FACES = {"xmin": 0, "xmax": 1, "ymin": 2, "ymax": 3, "zmin": 4, "zmax": 5}


class bfvm_config(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("n_substrates", C.c_int),
        ("dx", C.c_double), ("dt", C.c_double),
        ("diffusion_coefficients", C.POINTER(C.c_double)), ("decay_rates", C.POINTER(C.c_double)),
        ("precision", C.c_int), ("device", C.c_int),
    ]


class BfvmError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


_lib = None

# Exported symbols and their signatures; tests check that the library exports
# every function the header declares.
_SIGS = {
    "bfvm_create": (C.c_int, [C.POINTER(bfvm_config), C.POINTER(C.c_void_p)]),
    "bfvm_destroy": (C.c_int, [C.c_void_p]),
    "bfvm_set_dirichlet_activation": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_set_dirichlet_face": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "bfvm_set_dirichlet_uniform": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_upload_field": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_download_field": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_upload_field_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_download_field_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_set_agents": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 5),
    "bfvm_set_agents_from_rates": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 7),
    "bfvm_update_agents": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 4),
    "bfvm_step": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "bfvm_agent_constants_device": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double] + [C.c_void_p] * 9),
    "bfvm_apply_sources": (C.c_int, [C.c_void_p]),
    "bfvm_apply_sources_noalloc": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 5),
    "bfvm_sample_agents": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_set_sweep_schedule": (C.c_int, [C.c_void_p, C.c_int]),
    "bfvm_set_fused_sources": (C.c_int, [C.c_void_p, C.c_int]),
    "bfvm_set_substrate_streams": (C.c_int, [C.c_void_p, C.c_int]),
    "bfvm_get_substrate_streams": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "bfvm_set_sweep_tmem": (C.c_int, [C.c_void_p, C.c_int]),
    "bfvm_set_fp64_chain": (C.c_int, [C.c_void_p, C.c_int]),
    "bfvm_get_fp64_chain": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "bfvm_set_partition_min_line": (C.c_int, [C.c_void_p, C.c_int]),
    "bfvm_get_partition_min_line": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "bfvm_tmem_sweep_plan": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int)]),
    "bfvm_get_sweep_schedule": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "bfvm_set_dirichlet_nodes": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bfvm_write_mesh_matlab": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_double, C.c_double]),
    "bfvm_write_multicellds": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                                         C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), C.c_void_p, C.c_char_p,
                                         C.c_size_t, C.POINTER(C.c_size_t)]),
    "bfvm_apply_dirichlet_nodes": (C.c_int, [C.c_void_p]),
    "bfvm_step_2d": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "bfvm_set_agent_tracking": (C.c_int, [C.c_void_p, C.c_int]),
    "bfvm_set_agent_exports": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_get_internalized": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_set_internalized": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_release_internalized": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "bfvm_field_sums": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_set_mass_log": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "bfvm_read_mass_log": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "bfvm_synchronize": (C.c_int, [C.c_void_p]),
    "bfvm_set_wait_limit_ns": (C.c_int, [C.c_int, C.c_ulonglong]),
    "bfvm_stream": (C.c_void_p, [C.c_void_p]),
    "bfvm_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_device_field": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "bfvm_device_bytes": (C.c_size_t, [C.c_void_p]),
    "bfvm_estimate_bytes": (C.c_size_t, [C.POINTER(bfvm_config), C.c_int]),
    "bfvm_release_staging": (C.c_int, [C.c_void_p]),
    "bfvm_compute_gradients": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_set_bulk_rates": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bfvm_apply_bulk_sources": (C.c_int, [C.c_void_p]),
    "bfvm_write_matlab": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_double, C.c_double]),
    "bfvm_compute_gradients_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_field_offsets": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_get_launch": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "bfvm_set_launch": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "bfvm_kernel_launches": (C.c_longlong, []),
    "bfvm_timing_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "bfvm_timing_read": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "bfvm_timing_read_kernels": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "bfvm_status_string": (C.c_char_p, [C.c_int]),
    "bfvm_batch_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "bfvm_batch_destroy": (C.c_int, [C.c_void_p]),
    "bfvm_batch_add": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_batch_remove": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfvm_batch_size": (C.c_int, [C.c_void_p]),
    "bfvm_batch_step": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "bfvm_batch_synchronize": (C.c_int, [C.c_void_p]),
    "bfvm_batch_stream": (C.c_void_p, [C.c_void_p]),
    "bfvm_batch_set_schedule": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "bfvm_batch_get_schedule": (C.c_int, [C.c_void_p] + [C.POINTER(C.c_int)] * 5),
    "bfvm_batch_set_direct_threshold": (C.c_int, [C.c_void_p, C.c_longlong]),
    "bfvm_batch_get_direct_threshold": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "bfvm_batch_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "bfvm_batch_inject_stall": (C.c_int, [C.c_void_p, C.c_void_p]),
}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `make -C physicell-x_b200` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(status):
    return lib().bfvm_status_string(int(status)).decode()


def check(status, what):
    if status != BFVM_OK:
        raise BfvmError(status, what)


def kernel_launches():
    return int(lib().bfvm_kernel_launches())
