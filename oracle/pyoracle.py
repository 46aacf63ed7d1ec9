"""ctypes bindings for the CPU oracle -- TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
(and its ``--impl reference`` arm) import this module, always as the test
oracle or the timed CPU reference, never as the product path.

Two oracles share one numpy-facing interface:

* :class:`Port` wraps ``oracle/liboracle_lod3d.so``, the plain-C restatement
  (``oracle/lod3d_oracle.c``), which needs no reference sources.
* :class:`Reference` wraps ``oracle/_ref/libbiofvm_ref.so``, the reference's
  own BioFVM + DistPhy sources compiled by ``oracle/Makefile`` against a
  single-rank MPI shim, driven through ``oracle/ref_driver.cpp``.

Both take and return fields in the reference layout: a flat float64 array
indexed ``((i*ny + j)*nz + k)*S + d`` (BioFVM/BioFVM_mesh.cpp:1149-1158).
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle_lod3d.so")
REF_LIB = os.path.join(HERE, "_ref", "libbiofvm_ref.so")
DROPIN_LIB = os.path.join(HERE, "_ref", "libbiofvm_dropin.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Port:
    """The plain-C restatement of the reference path."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(PORT_LIB):
                raise FileNotFoundError(f"{PORT_LIB} missing: run `make -C oracle port`")
            L = C.CDLL(PORT_LIB)
            L.orc_thomas_axis.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double, _dp, _dp, _dp]
            L.orc_apply_dirichlet.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, _bp, _dp]
            L.orc_lod3d_step.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_double,
                                         C.c_double, _bp, _dp, C.c_int]
            L.orc_agent_constants.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp,
                                              _dp, _dp, _dp, _dp]
            L.orc_sources.argtypes = [_dp, C.c_int, C.c_int, _ip, C.c_void_p, _dp, _dp, _dp]
            L.orc_nearest_voxel.argtypes = [C.c_double] * 7 + [C.c_int] * 3
            L.orc_nearest_voxel.restype = C.c_int
            L.orc_gradients.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _dp]
            L.orc_gradients.restype = None
            L.orc_bulk_sources.argtypes = [_dp, C.c_long, C.c_double, _dp, _dp, _dp]
            L.orc_bulk_sources.restype = None
            L.orc_write_matlab.argtypes = [C.c_char_p, _dp] + [C.c_int] * 4 + [C.c_double] * 4
            L.orc_write_matlab.restype = C.c_int
            L.orc_sources_tracked.argtypes = [_dp, C.c_int, C.c_int, _ip, C.c_void_p, _dp, _dp, _dp, _dp, C.c_double,
                                              _dp]
            L.orc_sources_tracked.restype = None
            L.orc_release_internalized.argtypes = [_dp, C.c_int, C.c_int, _ip, _ip, _dp, C.c_double, _dp]
            L.orc_release_internalized.restype = None
            L.orc_dirichlet_nodes.argtypes = [_dp, C.c_int, C.c_int, _ip, _dp, C.c_void_p]
            L.orc_dirichlet_nodes.restype = None
            L.orc_lod2d_step.argtypes = [_dp, C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int,
                                         _ip, _dp, C.c_void_p]
            L.orc_lod2d_step.restype = None
            cls._lib = L
        return cls._lib

    @classmethod
    def thomas_axis(cls, n, D, decay, dt, dx):
        S = len(D)
        denom = np.zeros(n * S)
        cup = np.zeros(n * S)
        c1 = np.zeros(S)
        cls.lib().orc_thomas_axis(n, S, _f64(D), _f64(decay), dt, dx, denom, cup, c1)
        return denom.reshape(n, S), cup.reshape(n, S), c1

    @classmethod
    def apply_dirichlet(cls, field, shape, active, dvals):
        nx, ny, nz, S = shape
        cls.lib().orc_apply_dirichlet(field, nx, ny, nz, S, np.ascontiguousarray(active, np.uint8), _f64(dvals))

    @classmethod
    def lod_step(cls, field, shape, D, decay, dt, dx, active, dvals, threads=0):
        """One LOD diffusion-decay step, in place on ``field`` (float64, reference layout)."""
        nx, ny, nz, S = shape
        cls.lib().orc_lod3d_step(field, nx, ny, nz, S, _f64(D), _f64(decay), dt, dx,
                                 np.ascontiguousarray(active, np.uint8), _f64(dvals), threads)

    @classmethod
    def agent_constants(cls, dt, volume, voxel_volume, sec, upt, sat, exp_):
        """Per-agent (c1, c2, e2) rows for arrays of shape [n, S]."""
        sec, upt, sat, exp_ = (np.atleast_2d(_f64(a)) for a in (sec, upt, sat, exp_))
        n, S = sec.shape
        vol = np.broadcast_to(np.asarray(volume, np.float64), (n,))
        c1 = np.zeros((n, S))
        c2 = np.zeros((n, S))
        e2 = np.zeros((n, S))
        L = cls.lib()
        o1, o2, o3 = np.zeros(S), np.zeros(S), np.zeros(S)
        for a in range(n):
            L.orc_agent_constants(S, dt, float(vol[a]), voxel_volume, _f64(sec[a]), _f64(upt[a]),
                                  _f64(sat[a]), _f64(exp_[a]), o1, o2, o3)
            c1[a], c2[a], e2[a] = o1, o2, o3
        return c1, c2, e2

    @classmethod
    def sources(cls, field, S, voxel, c1, c2, e2, active=None):
        voxel = np.ascontiguousarray(voxel, np.int32)
        act = None
        if active is not None:
            act_arr = np.ascontiguousarray(active, np.uint8)
            act = act_arr.ctypes.data
        cls.lib().orc_sources(field, S, len(voxel), voxel, act, _f64(c1).ravel(), _f64(c2).ravel(),
                              _f64(e2).ravel())

    @classmethod
    def bulk_sources(cls, field, dt, supply, target, uptake):
        """simulate_bulk_sources_and_sinks on `field` in place."""
        f = field if field.dtype == np.float64 and field.flags.c_contiguous else None
        if f is None:
            raise ValueError("field must be a contiguous float64 array")
        cls.lib().orc_bulk_sources(f.reshape(-1), f.size, float(dt), _f64(supply).ravel(), _f64(target).ravel(),
                                   _f64(uptake).ravel())
        return f

    @classmethod
    def sources_tracked(cls, field, S, voxel, c1, c2, e2, e1, vvox, internal, active=None):
        """sources() with internalized-substrate tracking; internal [n, S]
        accumulates in place."""
        voxel = np.ascontiguousarray(voxel, np.int32)
        act = None if active is None else np.ascontiguousarray(active, np.uint8)
        cls.lib().orc_sources_tracked(field.reshape(-1), S, len(voxel), voxel,
                                      None if act is None else act.ctypes.data_as(C.c_void_p),
                                      _f64(c1).ravel(), _f64(c2).ravel(), _f64(e2).ravel(), _f64(e1).ravel(),
                                      float(vvox), internal.reshape(-1))
        return field

    @staticmethod
    def _nodes(voxel, values, act, S):
        voxel = np.ascontiguousarray(voxel, np.int32)
        values = _f64(values).reshape(voxel.size, S)
        act = None if act is None else np.ascontiguousarray(act, np.uint8).reshape(voxel.size, S)
        return voxel, values, act

    @classmethod
    def dirichlet_nodes(cls, field, S, voxel, values, act=None):
        """Pin a node list (distinct voxels) in place; act [n, S] or None (all)."""
        voxel, values, act = cls._nodes(voxel, values, act, S)
        cls.lib().orc_dirichlet_nodes(field.reshape(-1), S, voxel.size, voxel, values.ravel(),
                                      None if act is None else act.ctypes.data_as(C.c_void_p))
        return field

    @classmethod
    def lod2d_step(cls, field, nx, ny, S, D, decay, dt, dx, voxel, values, act=None):
        """One 2-D LOD step (nz = 1) with the node list pinned around the sweeps."""
        voxel, values, act = cls._nodes(voxel, values, act, S)
        cls.lib().orc_lod2d_step(field.reshape(-1), nx, ny, S, _f64(D), _f64(decay), float(dt), float(dx),
                                 voxel.size, voxel, values.ravel(),
                                 None if act is None else act.ctypes.data_as(C.c_void_p))
        return field

    @classmethod
    def release_internalized(cls, field, S, agents, voxel, fraction, vvox, internal):
        """Release the listed agents' internalized amounts into their voxels
        (in order); internal [n, S] and field change in place."""
        agents = np.ascontiguousarray(agents, np.int32)
        cls.lib().orc_release_internalized(field.reshape(-1), S, len(agents), agents,
                                           np.ascontiguousarray(voxel, np.int32), _f64(fraction).ravel(),
                                           float(vvox), internal.reshape(-1))
        return field

    @classmethod
    def write_matlab(cls, path, field, shape, origin, dx):
        nx, ny, nz, S = shape
        rc = cls.lib().orc_write_matlab(os.fsencode(path), _f64(field).ravel(), nx, ny, nz, S,
                                        float(origin[0]), float(origin[1]), float(origin[2]), float(dx))
        if rc != 0:
            raise OSError(f"could not write {path}")

    @classmethod
    def gradients(cls, field, shape, dx):
        """compute_all_gradient_vectors: array [voxels, S, 3]."""
        nx, ny, nz, S = shape
        f = _f64(field).ravel()
        out = np.empty(nx * ny * nz * S * 3, np.float64)
        cls.lib().orc_gradients(f, nx, ny, nz, S, float(dx), out)
        return out.reshape(nx * ny * nz, S, 3)

    @classmethod
    def nearest_voxel(cls, pos, origin, dx, dims):
        L = cls.lib()
        out = np.empty(len(pos), np.int32)
        for a, (x, y, z) in enumerate(pos):
            out[a] = L.orc_nearest_voxel(x, y, z, origin[0], origin[1], origin[2], dx, *dims)
        return out

    @classmethod
    def run(cls, wl, nsteps=None, threads=0):
        """Run a workload (see physicell-x_b200/bfvm/workloads.py) for nsteps of
        [agent sources ; LOD diffusion step], returning the final field."""
        nsteps = wl.steps if nsteps is None else nsteps
        field = wl.field0.copy()
        c1, c2, e2 = cls.workload_constants(wl)
        dv = wl.dirichlet_values
        for _ in range(nsteps):
            if wl.n_agents:
                cls.sources(field, wl.S, wl.agent_voxel, c1, c2, e2)
            cls.lod_step(field, wl.shape, wl.D, wl.decay, wl.dt, wl.dx, wl.dirichlet_active, dv, threads)
        return field

    @classmethod
    def workload_constants(cls, wl):
        """(c1, c2, e2) of every agent of a workload, [n, S] each."""
        if wl.n_agents == 0:
            z = np.zeros((0, wl.S))
            return z, z, z
        return cls.agent_constants(wl.dt, wl.agent_volume, wl.voxel_volume, wl.secretion, wl.uptake,
                                   wl.saturation, wl.net_export)


@contextlib.contextmanager
def _stdout_to_stderr():
    """The reference prints its banner and progress lines on stdout; send them
    to stderr so a caller's stdout carries only its own output."""
    sys.stdout.flush()
    saved = os.dup(1)
    try:
        os.dup2(2, 1)
        yield
    finally:
        try:
            C.CDLL(None).fflush(None)
        except Exception:
            pass
        os.dup2(saved, 1)
        os.close(saved)


class Reference:
    """The reference's own BioFVM solver and agents, built from its sources."""

    _libs: dict = {}

    def __init__(self, wl, threads=0, dropin=False):
        self.L = self.lib(dropin)
        self.wl = wl
        with _stdout_to_stderr():
            self._setup(wl)
        self.threads = threads

    def _setup(self, wl):
        nx, ny, nz, S = wl.shape
        self.h = self.L.ref_env_create(nx, ny, nz, wl.dx, wl.origin[0], wl.origin[1], wl.origin[2], S,
                                       _f64(wl.D), _f64(wl.decay))
        if not self.h:
            raise RuntimeError("reference mesh creation failed")
        for d in range(S):
            self.L.ref_env_set_dirichlet_activation(self.h, d, int(wl.dirichlet_active[d]))
        self.L.ref_env_set_dirichlet_face_values(self.h, _f64(wl.dirichlet_values))
        self.L.ref_env_set_field(self.h, _f64(wl.field0))
        self.agent_index = []
        for a in range(wl.n_agents):
            idx = self.L.ref_env_add_agent(self.h, *map(float, wl.agent_pos[a]), float(wl.agent_volume[a]),
                                           _f64(wl.secretion[a]), _f64(wl.uptake[a]), _f64(wl.saturation[a]),
                                           _f64(wl.net_export[a]))
            self.agent_index.append(idx)

    @classmethod
    def available(cls, dropin=False):
        return os.path.exists(DROPIN_LIB if dropin else REF_LIB)

    @classmethod
    def lib(cls, dropin=False):
        path = DROPIN_LIB if dropin else REF_LIB
        if path not in cls._libs:
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` (needs the reference sources)")
            L = C.CDLL(path)
            vp = C.c_void_p
            L.ref_env_create.restype = vp
            L.ref_env_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_int, _dp, _dp]
            L.ref_env_destroy.argtypes = [vp]
            L.ref_env_set_field.argtypes = [vp, _dp]
            L.ref_env_get_field.argtypes = [vp, _dp]
            L.ref_env_set_dirichlet_activation.argtypes = [vp, C.c_int, C.c_int]
            L.ref_env_set_dirichlet_face_values.argtypes = [vp, _dp]
            L.ref_env_apply_dirichlet.argtypes = [vp]
            L.ref_env_add_agent.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _dp]
            L.ref_env_add_agent.restype = C.c_int
            L.ref_env_num_agents.argtypes = [vp]
            L.ref_env_agent_voxel.argtypes = [vp, C.c_int]
            L.ref_env_agent_constants.argtypes = [vp, C.c_int, C.c_double, _dp, _dp, _dp]
            L.ref_env_sources.argtypes = [vp, C.c_double, C.c_int]
            L.ref_env_diffusion.argtypes = [vp, C.c_double, C.c_int, C.c_int]
            L.ref_env_diffusion.restype = C.c_int
            L.ref_env_run.argtypes = [vp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]
            L.ref_env_run.restype = C.c_int
            L.ref_max_threads.restype = C.c_int
            L.ref_env_gradients.argtypes = [vp, _dp]
            L.ref_env_gradients.restype = None
            L.ref_env_bulk.argtypes = [vp, C.c_double, _dp, _dp, _dp, C.c_int]
            L.ref_env_bulk.restype = None
            L.ref_env_write_matlab.argtypes = [vp, C.c_char_p]
            L.ref_env_write_matlab.restype = None
            L.ref_set_tracking.argtypes = [C.c_int]
            L.ref_set_tracking.restype = None
            L.ref_env_agent_internalized.argtypes = [vp, C.c_int, _dp]
            L.ref_env_agent_internalized.restype = None
            L.ref_env_agent_set_internalized.argtypes = [vp, C.c_int, _dp]
            L.ref_env_agent_set_internalized.restype = None
            L.ref_env_agent_release.argtypes = [vp, C.c_int, _dp]
            L.ref_env_agent_release.restype = None
            L.ref_env_add_dirichlet_node.argtypes = [vp, C.c_int, _dp]
            L.ref_env_add_dirichlet_node.restype = None
            L.ref_env_remove_dirichlet_node.argtypes = [vp, C.c_int]
            L.ref_env_remove_dirichlet_node.restype = None
            L.ref_env_set_node_activation.argtypes = [vp, C.c_int, C.c_int, C.c_int]
            L.ref_env_set_node_activation.restype = None
            L.ref_env_apply_dirichlet_conditions.argtypes = [vp]
            L.ref_env_apply_dirichlet_conditions.restype = None
            L.ref_env_lod2d.argtypes = [vp, C.c_double]
            L.ref_env_lod2d.restype = None
            L.ref_env_set_names.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p]
            L.ref_env_set_names.restype = None
            L.ref_env_set_density_name.argtypes = [vp, C.c_int, C.c_char_p, C.c_char_p]
            L.ref_env_set_density_name.restype = None
            L.ref_env_bounding_box.argtypes = [vp, _dp]
            L.ref_env_bounding_box.restype = None
            L.ref_env_multicellds_substrates.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_long]
            L.ref_env_multicellds_substrates.restype = C.c_long
            if dropin:
                L.ref_env_dropin_fuse_sources.argtypes = [vp, C.c_int, C.c_double]
                L.ref_env_dropin_fuse_sources.restype = C.c_int
                L.ref_env_dropin_lod2d.argtypes = [vp, C.c_double]
                L.ref_env_dropin_lod2d.restype = None
            cls._libs[path] = L
        return cls._libs[path]

    def close(self):
        if self.h:
            self.L.ref_env_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self):
        out = np.empty(int(np.prod(self.wl.shape)), np.float64)
        self.L.ref_env_get_field(self.h, out)
        return out

    def set_field(self, f):
        self.L.ref_env_set_field(self.h, _f64(f))

    def agent_voxels(self):
        return np.array([self.L.ref_env_agent_voxel(self.h, a) for a in range(self.L.ref_env_num_agents(self.h))],
                        np.int32)

    def agent_constants(self, dt):
        S = self.wl.S
        n = self.L.ref_env_num_agents(self.h)
        c1, c2, e2 = np.zeros((n, S)), np.zeros((n, S)), np.zeros((n, S))
        o1, o2, o3 = np.zeros(S), np.zeros(S), np.zeros(S)
        for a in range(n):
            self.L.ref_env_agent_constants(self.h, a, dt, o1, o2, o3)
            c1[a], c2[a], e2[a] = o1, o2, o3
        return c1, c2, e2

    def sources(self, threads=1):
        with _stdout_to_stderr():
            self.L.ref_env_sources(self.h, self.wl.dt, threads)

    def diffusion(self, solver=0, threads=None):
        with _stdout_to_stderr():
            rc = self.L.ref_env_diffusion(self.h, self.wl.dt, solver, self.threads if threads is None else threads)
        if rc != 0:
            raise RuntimeError(f"ref_env_diffusion solver={solver} rc={rc}")

    def apply_dirichlet(self):
        self.L.ref_env_apply_dirichlet(self.h)

    def bulk_sources(self, supply, target, uptake, threads=1):
        """The reference's simulate_bulk_sources_and_sinks(dt) with these
        per-voxel rates (arrays like the field)."""
        self._bulk = tuple(_f64(a).ravel().copy() for a in (supply, target, uptake))  # kept alive
        with _stdout_to_stderr():
            self.L.ref_env_bulk(self.h, self.wl.dt, *self._bulk, threads)

    def set_tracking(self, on):
        """The process-wide track_internalized_substrates_in_each_agent option."""
        self.L.ref_set_tracking(1 if on else 0)

    def internalized(self):
        """Every agent's internalized_substrates, [n, S]."""
        n, S = self.wl.n_agents, self.wl.S
        out = np.zeros((n, S))
        o = np.zeros(S)
        for a in range(n):
            self.L.ref_env_agent_internalized(self.h, a, o)
            out[a] = o
        return out

    def add_dirichlet_node(self, voxel, values):
        self.L.ref_env_add_dirichlet_node(self.h, int(voxel), _f64(values))

    def remove_dirichlet_node(self, voxel):
        self.L.ref_env_remove_dirichlet_node(self.h, int(voxel))

    def set_node_activation(self, voxel, substrate, on):
        self.L.ref_env_set_node_activation(self.h, int(voxel), int(substrate), 1 if on else 0)

    def apply_dirichlet_conditions(self):
        """Microenvironment::apply_dirichlet_conditions: every Dirichlet node."""
        self.L.ref_env_apply_dirichlet_conditions(self.h)

    def bounding_box(self):
        out = np.zeros(6)
        self.L.ref_env_bounding_box(self.h, out)
        return out

    def multicellds_substrates(self, base, domain, mesh_units, spatial_units, time_units, names, units):
        """The reference's add_BioFVM_substrates_to_open_xml_pugi + document
        text (and its two MATLAB files under base).  The reference builds the
        element once per process (a static flag) into a global document, so
        call this at most once per process."""
        e = lambda x: str(x).encode()
        self.L.ref_env_set_names(self.h, e(domain), e(mesh_units), e(spatial_units), e(time_units))
        for d, (nm, un) in enumerate(zip(names, units)):
            self.L.ref_env_set_density_name(self.h, d, e(nm), e(un))
        buf = C.create_string_buffer(1 << 24)
        with _stdout_to_stderr():
            n = self.L.ref_env_multicellds_substrates(self.h, e(base), buf, 1 << 24)
        if n < 0:
            raise RuntimeError("MultiCellDS document too large")
        return buf.raw[:n].decode()

    def lod2d(self):
        """The reference's 2-D LOD solver, one step (use with ny == 1 only)."""
        with _stdout_to_stderr():
            self.L.ref_env_lod2d(self.h, self.wl.dt)

    def dropin_lod2d(self):
        """One step of the GPU drop-in's 2-D solver through the serial slot
        (a Reference opened with dropin=True)."""
        with _stdout_to_stderr():
            self.L.ref_env_dropin_lod2d(self.h, self.wl.dt)

    def set_internalized(self, amounts):
        for a in range(self.wl.n_agents):
            self.L.ref_env_agent_set_internalized(self.h, a, _f64(amounts[a]))

    def release(self, agents, fraction):
        """release_internalized_substrates for the listed agents, in order."""
        for q, a in enumerate(agents):
            self.L.ref_env_agent_release(self.h, int(a), _f64(fraction[q]))

    def write_matlab(self, path):
        """The reference's Microenvironment::write_to_matlab(path)."""
        with _stdout_to_stderr():
            self.L.ref_env_write_matlab(self.h, os.fsencode(path))

    def gradients(self):
        """The reference's compute_all_gradient_vectors on the current field,
        as [voxels, S, 3]."""
        nx, ny, nz, S = self.wl.shape
        out = np.empty(nx * ny * nz * S * 3, np.float64)
        with _stdout_to_stderr():
            self.L.ref_env_gradients(self.h, out)
        return out.reshape(nx * ny * nz, S, 3)

    def run(self, nsteps=None, solver=0, threads=None, sources_threads=1, fetch=True):
        nsteps = self.wl.steps if nsteps is None else nsteps
        with _stdout_to_stderr():
            rc = self.L.ref_env_run(self.h, self.wl.dt, nsteps, solver, self.threads if threads is None else threads,
                                    sources_threads)
        if rc != 0:
            raise RuntimeError(f"ref_env_run rc={rc}")
        return self.field() if fetch else None


def max_threads():
    if Reference.available():
        return int(Reference.lib().ref_max_threads())
    return os.cpu_count() or 1


def timed(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0
