"""Python mirror of the reference's Microenvironment interface for the
diffusion-decay path, over the C ABI.

Names follow the reference API so that a test reads like the reference's
own calls:

=====================================================  ==========================================
reference (BioFVM, PhysiCell-X 1.14.0)                 here
=====================================================  ==========================================
``Microenvironment::resize_space`` + ``set_density``   ``Microenvironment(nx, ny, nz, dx, dt, D, decay)``
``set_substrate_dirichlet_activation(d, bool)``        ``set_substrate_dirichlet_activation(d, on)``
``update_dirichlet_node`` on face voxels               ``set_dirichlet_face`` / ``set_dirichlet_uniform``
``density_vector`` writes / reads                      ``upload_field`` / ``download_field``
``simulate_diffusion_decay(dt, world, cart)``          ``simulate_diffusion_decay(nsteps=1)``
``simulate_cell_sources_and_sinks(dt)``                ``simulate_cell_sources_and_sinks()``
``Basic_Agent::nearest_density_vector``                ``sample_agents()``
=====================================================  ==========================================

Errors raise :class:`bfvm._lib.BfvmError` carrying the C status code; the
solve is left unchanged on failure, as the reference prints and returns
(BioFVM/BioFVM_solvers.cpp:116-121).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import BFVM_FP32, BFVM_FP64, BFVM_STEP_SOURCES, FACES, check


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Microenvironment:
    """One microenvironment resident on one GPU."""

    def __init__(self, nx, ny, nz, dx, dt, diffusion_coefficients, decay_rates, precision="fp64", device=0):
        self.L = _lib.lib()
        D = _f64(diffusion_coefficients).ravel()
        lam = _f64(decay_rates).ravel()
        if D.shape != lam.shape:
            raise ValueError("diffusion_coefficients and decay_rates differ in length")
        self.shape = (int(nx), int(ny), int(nz), int(D.size))
        self.dx, self.dt = float(dx), float(dt)
        self.precision = precision
        cfg = _lib.bfvm_config(int(nx), int(ny), int(nz), int(D.size), float(dx), float(dt),
                               D.ctypes.data_as(C.POINTER(C.c_double)), lam.ctypes.data_as(C.POINTER(C.c_double)),
                               BFVM_FP64 if precision == "fp64" else BFVM_FP32, int(device))
        h = C.c_void_p()
        check(self.L.bfvm_create(C.byref(cfg), C.byref(h)), "bfvm_create")
        self.h = h
        self.n_agents = 0

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.bfvm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def S(self):
        return self.shape[3]

    @property
    def n_values(self):
        nx, ny, nz, S = self.shape
        return nx * ny * nz * S

    # -- Dirichlet ----------------------------------------------------------
    def set_dirichlet_activation(self, active):
        a = np.ascontiguousarray(active, np.uint8).ravel()
        if a.size != self.S:
            raise ValueError("activation needs one flag per substrate")
        check(self.L.bfvm_set_dirichlet_activation(self.h, _ptr(a)), "bfvm_set_dirichlet_activation")

    def set_substrate_dirichlet_activation(self, substrate, on):
        act = getattr(self, "_active", np.ones(self.S, np.uint8)).copy()
        act[substrate] = 1 if on else 0
        self.set_dirichlet_activation(act)
        self._active = act

    def set_dirichlet_uniform(self, values):
        v = _f64(values).ravel()
        check(self.L.bfvm_set_dirichlet_uniform(self.h, _ptr(v)), "bfvm_set_dirichlet_uniform")

    def set_dirichlet_face(self, face, plane):
        f = FACES[face] if isinstance(face, str) else int(face)
        p = _f64(plane)
        check(self.L.bfvm_set_dirichlet_face(self.h, f, _ptr(p)), "bfvm_set_dirichlet_face")

    # -- field --------------------------------------------------------------
    def upload_field(self, field):
        f = _f64(field).ravel()
        if f.size != self.n_values:
            raise ValueError(f"field has {f.size} values, expected {self.n_values}")
        check(self.L.bfvm_upload_field(self.h, _ptr(f)), "bfvm_upload_field")

    def download_field(self, out=None):
        out = np.empty(self.n_values, np.float64) if out is None else out
        check(self.L.bfvm_download_field(self.h, _ptr(out)), "bfvm_download_field")
        return out

    def upload_field_device(self, ptr):
        check(self.L.bfvm_upload_field_device(self.h, C.c_void_p(int(ptr))), "bfvm_upload_field_device")

    def download_field_device(self, ptr):
        check(self.L.bfvm_download_field_device(self.h, C.c_void_p(int(ptr))), "bfvm_download_field_device")

    # -- agents -------------------------------------------------------------
    def set_agents(self, voxel, c1, c2, e2, active=None):
        v = np.ascontiguousarray(voxel, np.int32).ravel()
        n = v.size
        c1, c2, e2 = (_f64(x).reshape(n, self.S) for x in (c1, c2, e2))
        act = None if active is None else np.ascontiguousarray(active, np.uint8).ravel()
        check(self.L.bfvm_set_agents(self.h, n, _ptr(v), _ptr(act), _ptr(c1), _ptr(c2), _ptr(e2)),
              "bfvm_set_agents")
        self.n_agents = n

    def update_agents(self, idx, c1, c2, e2):
        """New constants for the agents at list indices ``idx`` (the ones
        whose volume changed, as Basic_Agent::simulate_secretion_and_uptake
        recomputes only those); the list and its voxel sort are kept."""
        i = np.ascontiguousarray(idx, np.int32).ravel()
        m = i.size
        c1, c2, e2 = (_f64(x).reshape(m, self.S) for x in (c1, c2, e2))
        check(self.L.bfvm_update_agents(self.h, m, _ptr(i), _ptr(c1), _ptr(c2), _ptr(e2)), "bfvm_update_agents")

    def set_agents_from_rates(self, voxel, volume, secretion, uptake, saturation, net_export, active=None):
        v = np.ascontiguousarray(voxel, np.int32).ravel()
        n = v.size
        vol = _f64(np.broadcast_to(np.asarray(volume, np.float64), (n,)))
        rates = [_f64(x).reshape(n, self.S) for x in (secretion, uptake, saturation, net_export)]
        act = None if active is None else np.ascontiguousarray(active, np.uint8).ravel()
        check(self.L.bfvm_set_agents_from_rates(self.h, n, _ptr(v), _ptr(act), _ptr(vol), *[_ptr(r) for r in rates]),
              "bfvm_set_agents_from_rates")
        self.n_agents = n

    def sample_agents(self):
        out = np.empty((self.n_agents, self.S), np.float64)
        check(self.L.bfvm_sample_agents(self.h, _ptr(out)), "bfvm_sample_agents")
        return out

    # -- Dirichlet nodes and the 2-D solver ---------------------------------
    def set_dirichlet_nodes(self, voxel, values, activation=None):
        """Dirichlet nodes (Microenvironment::add_dirichlet_node and the
        per-voxel set_substrate_dirichlet_activation): voxel [n] reference
        indices, values [n, S], activation [n, S] or None (each substrate's
        current activation).  Replaces the node list; an empty list clears it."""
        v = np.ascontiguousarray(voxel, np.int32).ravel()
        vals = _f64(values).reshape(v.size, self.S)
        act = None if activation is None else np.ascontiguousarray(activation, np.uint8).reshape(v.size, self.S)
        check(self.L.bfvm_set_dirichlet_nodes(self.h, int(v.size), _ptr(v), _ptr(vals), _ptr(act)),
              "bfvm_set_dirichlet_nodes")

    def apply_dirichlet_conditions(self):
        """Microenvironment::apply_dirichlet_conditions over the node list."""
        check(self.L.bfvm_apply_dirichlet_nodes(self.h), "bfvm_apply_dirichlet_nodes")

    def simulate_diffusion_decay_2d(self, nsteps=1, sources=False):
        """nsteps steps of the 2-D LOD solver (nz must be 1)."""
        check(self.L.bfvm_step_2d(self.h, int(nsteps), BFVM_STEP_SOURCES if sources else 0), "bfvm_step_2d")

    # -- internalized substrates ---------------------------------------------
    def set_track_internalized_substrates(self, on=True):
        """Microenvironment_Options::track_internalized_substrates_in_each_agent
        for this solve: every source/sink stage also keeps each agent's
        internalized amounts (Basic_Agent::internalized_substrates)."""
        check(self.L.bfvm_set_agent_tracking(self.h, 1 if on else 0), "bfvm_set_agent_tracking")

    def set_agent_exports(self, export1):
        """Per-agent export per step (net_export_rate * dt), [n, S], for a list
        given as constants by set_agents."""
        e1 = _f64(export1).reshape(self.n_agents, self.S)
        check(self.L.bfvm_set_agent_exports(self.h, _ptr(e1)), "bfvm_set_agent_exports")

    def internalized_substrates(self):
        """Every agent's internalized amounts, [n, S] in agent-list order."""
        out = np.empty((self.n_agents, self.S), np.float64)
        check(self.L.bfvm_get_internalized(self.h, _ptr(out)), "bfvm_get_internalized")
        return out

    def set_internalized_substrates(self, amounts=None):
        """Overwrite the internalized amounts ([n, S]; None: zeros)."""
        a = None if amounts is None else _f64(amounts).reshape(self.n_agents, self.S)
        check(self.L.bfvm_set_internalized(self.h, _ptr(a)), "bfvm_set_internalized")

    def release_internalized_substrates(self, agents, fraction):
        """Basic_Agent::release_internalized_substrates for the listed agents
        (in order); fraction [len(agents), S] is each one's
        fraction_released_at_death."""
        idx = np.ascontiguousarray(agents, np.int32).ravel()
        fr = _f64(np.broadcast_to(np.asarray(fraction, np.float64), (idx.size, self.S)))
        check(self.L.bfvm_release_internalized(self.h, int(idx.size), _ptr(idx), _ptr(fr)),
              "bfvm_release_internalized")

    # -- stepping -----------------------------------------------------------
    def simulate_diffusion_decay(self, nsteps=1, sources=False):
        """nsteps LOD steps; with sources=True each step first applies the agents
        (fused into the x sweep)."""
        check(self.L.bfvm_step(self.h, int(nsteps), BFVM_STEP_SOURCES if sources else 0), "bfvm_step")

    def simulate_cell_sources_and_sinks(self):
        check(self.L.bfvm_apply_sources(self.h), "bfvm_apply_sources")

    def set_bulk_rates(self, supply, target, uptake):
        """Per-voxel supply rate, target density and uptake rate (arrays like
        the field, reference layout); None for all three clears them."""
        if supply is None and target is None and uptake is None:
            check(self.L.bfvm_set_bulk_rates(self.h, None, None, None), "bfvm_set_bulk_rates")
            return
        arrs = [_f64(a).ravel() for a in (supply, target, uptake)]
        for a in arrs:
            if a.size != self.n_values:
                raise ValueError(f"rate array has {a.size} values, expected {self.n_values}")
        check(self.L.bfvm_set_bulk_rates(self.h, *[_ptr(a) for a in arrs]), "bfvm_set_bulk_rates")

    def simulate_bulk_sources_and_sinks(self):
        check(self.L.bfvm_apply_bulk_sources(self.h), "bfvm_apply_bulk_sources")

    def write_to_matlab(self, path, origin):
        """Microenvironment::write_to_matlab: the MATLAB v4 density file;
        origin is the domain's lower corner (x, y, z)."""
        import os

        check(self.L.bfvm_write_matlab(self.h, os.fsencode(str(path)), float(origin[0]), float(origin[1]),
                                       float(origin[2])), "bfvm_write_matlab")

    def write_mesh_matlab(self, path, origin):
        """General_Mesh::write_to_matlab: the MATLAB v4 mesh file (voxel
        centres and volumes); origin is the domain's lower corner."""
        import os

        check(self.L.bfvm_write_mesh_matlab(self.h, os.fsencode(str(path)), float(origin[0]), float(origin[1]),
                                            float(origin[2])), "bfvm_write_mesh_matlab")

    def write_multicellds(self, filename_base, bounding_box, names, units, domain_name="microenvironment",
                          mesh_units="micron", spatial_units="micron", time_units="min"):
        """The microenvironment's MultiCellDS output (<base>.xml,
        <base>_mesh0.mat, <base>_microenvironment0.mat), as
        save_BioFVM_to_MultiCellDS_xml_pugi writes them for the substrates;
        returns the XML text."""
        import os

        enc = lambda x: str(x).encode()
        n = (C.c_char_p * self.S)(*[enc(x) for x in names])
        u = (C.c_char_p * self.S)(*[enc(x) for x in units])
        bb = _f64(np.asarray(bounding_box, np.float64).ravel())
        length = C.c_size_t()
        check(self.L.bfvm_write_multicellds(self.h, os.fsencode(str(filename_base)), enc(domain_name), enc(mesh_units),
                                            enc(spatial_units), enc(time_units), n, u, _ptr(bb), None, 0,
                                            C.byref(length)), "bfvm_write_multicellds")
        with open(str(filename_base) + ".xml", "rb") as fh:
            return fh.read().decode()

    def compute_all_gradient_vectors(self, out=None):
        """Gradients of every substrate at every voxel, [voxels, S, 3] in the
        reference's voxel order (Microenvironment::compute_all_gradient_vectors)."""
        nx, ny, nz, S = self.shape
        out = np.empty((nx * ny * nz, S, 3), np.float64) if out is None else out
        check(self.L.bfvm_compute_gradients(self.h, _ptr(out)), "bfvm_compute_gradients")
        return out

    def compute_all_gradient_vectors_device(self, ptr):
        check(self.L.bfvm_compute_gradients_device(self.h, C.c_void_p(int(ptr))), "bfvm_compute_gradients_device")

    def synchronize(self):
        check(self.L.bfvm_synchronize(self.h), "bfvm_synchronize")

    def field_sums(self):
        out = np.empty(self.S, np.float64)
        check(self.L.bfvm_field_sums(self.h, _ptr(out)), "bfvm_field_sums")
        return out

    def set_mass_log(self, every, capacity=4096):
        """Record the FP64 per-substrate field sums after every `every`-th
        step (0: off); see :meth:`mass_log`."""
        check(self.L.bfvm_set_mass_log(self.h, int(every), int(capacity)), "bfvm_set_mass_log")
        self._mass_capacity = int(capacity)

    def mass_log(self):
        """The mass-balance records still kept, oldest first, [records, S]."""
        cap = getattr(self, "_mass_capacity", 0)
        out = np.empty((cap, self.S), np.float64)
        n = C.c_int()
        check(self.L.bfvm_read_mass_log(self.h, _ptr(out), cap, C.byref(n)), "bfvm_read_mass_log")
        return out[: min(n.value, cap)]

    # -- introspection --------------------------------------------------------
    @property
    def stream(self):
        return int(self.L.bfvm_stream(self.h) or 0)

    def set_stream(self, stream_ptr):
        check(self.L.bfvm_set_stream(self.h, C.c_void_p(int(stream_ptr) if stream_ptr else None)), "bfvm_set_stream")

    def device_field(self):
        p, pitch, eb = C.c_void_p(), C.c_int(), C.c_int()
        check(self.L.bfvm_device_field(self.h, C.byref(p), C.byref(pitch), C.byref(eb)), "bfvm_device_field")
        return int(p.value or 0), int(pitch.value), int(eb.value)

    def device_bytes(self):
        return int(self.L.bfvm_device_bytes(self.h))

    def timing_enable(self, on=True):
        check(self.L.bfvm_timing_enable(self.h, 1 if on else 0), "bfvm_timing_enable")

    def timing_read(self):
        """(ms_x, ms_y, ms_z) summed over the recorded steps (the source kernel
        counted with x), and the step count."""
        ms = np.zeros(3, np.float64)
        n = C.c_int()
        check(self.L.bfvm_timing_read(self.h, _ptr(ms), C.byref(n)), "bfvm_timing_read")
        return ms, int(n.value)

    def timing_read_kernels(self):
        """(ms_sources, ms_x, ms_y, ms_z) summed over the recorded steps, and
        the step count."""
        ms = np.zeros(4, np.float64)
        n = C.c_int()
        check(self.L.bfvm_timing_read_kernels(self.h, _ptr(ms), C.byref(n)), "bfvm_timing_read_kernels")
        return ms, int(n.value)

    def set_sweep_schedule(self, persistent=1):
        """0: one CTA per tile; 1 (default): persistent y/z sweeps (a CTA walks
        many tiles, the next loading while the current one finishes), x per
        tile; 2: all three sweeps persistent.  True/False map to 1/0."""
        check(self.L.bfvm_set_sweep_schedule(self.h, int(persistent)), "bfvm_set_sweep_schedule")

    def set_fused_sources(self, fused=True):
        """Apply the agents inside the x sweep (True) or with the standalone
        source kernel ahead of the sweeps (False, the default)."""
        check(self.L.bfvm_set_fused_sources(self.h, 1 if fused else 0), "bfvm_set_fused_sources")

    def set_substrate_streams(self, streams=1):
        """Runs of steps sweep every substrate in one sequence of launches (1,
        the default) or the two halves of the substrates on two streams (2);
        the same bits either way."""
        check(self.L.bfvm_set_substrate_streams(self.h, int(streams)), "bfvm_set_substrate_streams")

    def substrate_streams(self):
        v = C.c_int(0)
        check(self.L.bfvm_get_substrate_streams(self.h, C.byref(v)), "bfvm_get_substrate_streams")
        return v.value

    def set_sweep_tmem(self, level=1):
        """Tensor-memory rings in the FP64 persistent sweeps: 1 (the default)
        in the y/z sweeps, 2 in the x sweep as well, 0 (or False) none; same
        bits at every level."""
        check(self.L.bfvm_set_sweep_tmem(self.h, int(level)), "bfvm_set_sweep_tmem")

    def set_fp64_chain(self, chain):
        """FP64 forward elimination: 0 (default) the reference's arithmetic,
        bit for bit; 1 the short chain (one FMA per element, within a few
        ulp of the reference per sweep); 2 the short chain with long y and z
        lines solved by the partition method."""
        check(self.L.bfvm_set_fp64_chain(self.h, int(chain)), "bfvm_set_fp64_chain")

    def set_partition_min_line(self, n_line):
        """The shortest y/z line chain 2 solves partitioned (-1: the
        precision's default)."""
        check(self.L.bfvm_set_partition_min_line(self.h, int(n_line)), "bfvm_set_partition_min_line")

    def get_partition_min_line(self):
        v = C.c_int()
        check(self.L.bfvm_get_partition_min_line(self.h, C.byref(v)), "bfvm_get_partition_min_line")
        return int(v.value)

    def get_sweep_schedule(self):
        v = C.c_int()
        check(self.L.bfvm_get_sweep_schedule(self.h, C.byref(v)), "bfvm_get_sweep_schedule")
        return int(v.value)

    def get_launch(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(self.L.bfvm_get_launch(self.h, C.byref(a), C.byref(b), C.byref(c)), "bfvm_get_launch")
        return a.value, b.value, c.value

    def set_launch(self, x_lines, yz_tile, yz_chunk):
        check(self.L.bfvm_set_launch(self.h, int(x_lines), int(yz_tile), int(yz_chunk)), "bfvm_set_launch")

    # -- convenience ----------------------------------------------------------
    @classmethod
    def from_workload(cls, wl, precision="fp64", device=0, agents="rates", upload=True):
        """Build a solve from a :class:`bfvm.workloads.Workload`: coefficients,
        Dirichlet activation and per-face values, initial field and agents."""
        me = cls(wl.nx, wl.ny, wl.nz, wl.dx, wl.dt, wl.D, wl.decay, precision=precision, device=device)
        me.set_dirichlet_activation(wl.dirichlet_active)
        if wl.uniform_faces():
            me.set_dirichlet_uniform(wl.face_values[0])
        else:
            for f, plane in enumerate(wl.face_planes()):
                me.set_dirichlet_face(f, plane)
        if upload:
            me.upload_field(wl.field0)
        if wl.n_agents and agents == "rates":
            me.set_agents_from_rates(wl.agent_voxel, wl.agent_volume, wl.secretion, wl.uptake, wl.saturation,
                                     wl.net_export)
        return me
