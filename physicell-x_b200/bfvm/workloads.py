"""Seeded synthetic microenvironment workloads.

Each workload is one BioFVM solve: a uniform Cartesian grid, S diffusing
substrates with constant coefficients, Dirichlet boundary data, an initial
field and a list of point agents with secretion/uptake/export rates.  The
shapes and value distributions follow the benchmark configurations of the
diffusion-decay path:

* ``cube50`` -- 50^3 voxels, dx=20 um, 2 substrates (oxygen-like Dirichlet
  38 on all faces; a zero-flux secreted substrate), 2,000 uniform agents,
  dt=0.01 min, 1000 steps.
* ``cube200`` -- 200^3, dx=10 um, 4 substrates with log-uniform D in
  [1e2,1e5] and decay in [1e-3,1]; substrate 0 Dirichlet 38; 100,000 uniform
  agents with per-agent uptake in [0,10] and secretion in [0,1]; 500 steps.
* ``cube640`` -- 640^3, dx=10 um, the two substrates of cube50, 1,000,000
  agents in a Gaussian ball (sigma 1500 um) clamped into the box; 1000 steps.
* ``uneven_env`` / ``serve_request`` -- the uneven environments of the
  batched and serving workloads (edges 24-128 / 32-256, 1-6 / 1-8 substrates,
  random Dirichlet activation and per-face values, 0-20k / 0-200k agents).

There is no public dataset behind these; the generators stand in for the
reference's PhysiCell settings files with seeded numpy ``Generator(PCG64)``
draws.  Layout conventions are the reference's: fields are flat float64
``[x][y][z][substrate]`` and voxel indices are ``(i*ny + j)*nz + k``
(BioFVM/BioFVM_mesh.cpp:1149-1158).

Dirichlet semantics follow the reference 3-D solvers: every voxel on the six
outer faces of an *activated* substrate is pinned to its own value
(Microenvironment::apply_dirichlet_boundaries_conditions,
BioFVM/BioFVM_microenvironment.cpp:348-446).  Per-face values are resolved
in the reference's setup order xmin, xmax, ymin, ymax, zmin, zmax, with
later faces overwriting shared edges (BioFVM_microenvironment.cpp:2647-2760),
and faces that nobody set keep 1.0 (:632).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

FACE_NAMES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


@dataclasses.dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    S: int
    dx: float
    dt: float
    steps: int
    D: np.ndarray               # [S]
    decay: np.ndarray           # [S]
    dirichlet_active: np.ndarray  # [S] uint8
    face_values: np.ndarray     # [6, S]: value per face (xmin..zmax) per substrate
    origin: tuple               # (x0, y0, z0) lower corner of the box
    seed: int
    # agents
    agent_pos: np.ndarray       # [n, 3]
    agent_volume: np.ndarray    # [n]
    secretion: np.ndarray       # [n, S]
    uptake: np.ndarray          # [n, S]
    saturation: np.ndarray      # [n, S]
    net_export: np.ndarray      # [n, S]
    init_kind: tuple = ()       # per substrate: ("const", v) or ("uniform", lo, hi)
    _field0: np.ndarray | None = None
    _voxel: np.ndarray | None = None

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz, self.S)

    @property
    def n_voxels(self):
        return self.nx * self.ny * self.nz

    @property
    def n_values(self):
        return self.n_voxels * self.S

    @property
    def n_agents(self):
        return int(self.agent_pos.shape[0])

    @property
    def voxel_volume(self):
        return self.dx * self.dx * self.dx

    @property
    def field0(self) -> np.ndarray:
        """Initial field, float64, reference layout (built on first use)."""
        if self._field0 is None:
            rng = np.random.Generator(np.random.PCG64(self.seed + 7))
            f = np.empty((self.n_voxels, self.S), np.float64)
            for d, kind in enumerate(self.init_kind):
                if kind[0] == "const":
                    f[:, d] = kind[1]
                else:
                    f[:, d] = rng.uniform(kind[1], kind[2], self.n_voxels)
            self._field0 = f.reshape(-1)
        return self._field0

    @property
    def agent_voxel(self) -> np.ndarray:
        """Reference voxel index of each agent (Cartesian_Mesh::nearest_voxel_index,
        BioFVM/BioFVM_mesh.cpp:1825-1843): floor((p - box_min)/dx), clamped."""
        if self._voxel is None:
            self._voxel = nearest_voxel(self.agent_pos, self.origin, self.dx, (self.nx, self.ny, self.nz))
        return self._voxel

    def face_planes(self):
        """The resolved Dirichlet value of every face voxel, as six planes in
        the reference orientation: x faces [ny, nz, S], y faces [nx, nz, S],
        z faces [nx, ny, S].  Shared edges carry the value of the face that the
        reference writes last (order xmin, xmax, ymin, ymax, zmin, zmax)."""
        nx, ny, nz, S = self.shape
        fv = self.face_values
        xm = np.broadcast_to(fv[0], (ny, nz, S)).copy()
        xp = np.broadcast_to(fv[1], (ny, nz, S)).copy()
        ym = np.broadcast_to(fv[2], (nx, nz, S)).copy()
        yp = np.broadcast_to(fv[3], (nx, nz, S)).copy()
        zm = np.broadcast_to(fv[4], (nx, ny, S)).copy()
        zp = np.broadcast_to(fv[5], (nx, ny, S)).copy()
        # y faces overwrite x-face edges; z faces overwrite both.
        xm[0, :, :] = fv[2]; xm[ny - 1, :, :] = fv[3]
        xp[0, :, :] = fv[2]; xp[ny - 1, :, :] = fv[3]
        for pl in (xm, xp):
            pl[:, 0, :] = fv[4]
            pl[:, nz - 1, :] = fv[5]
        for pl in (ym, yp):
            pl[:, 0, :] = fv[4]
            pl[:, nz - 1, :] = fv[5]
        # one-voxel-thick axes: the later face of the same axis wins.
        if nx == 1:
            xm[...] = xp
        if ny == 1:
            ym[...] = yp
        if nz == 1:
            zm[...] = zp
        return xm, xp, ym, yp, zm, zp

    @property
    def dirichlet_values(self) -> np.ndarray:
        """Full-grid Dirichlet value array in the reference layout (face voxels
        hold their resolved value; interior entries are 1.0 and unused)."""
        nx, ny, nz, S = self.shape
        dv = np.ones((nx, ny, nz, S), np.float64)
        xm, xp, ym, yp, zm, zp = self.face_planes()
        dv[0] = xm
        dv[nx - 1] = xp
        dv[:, 0] = ym
        dv[:, ny - 1] = yp
        dv[:, :, 0] = zm
        dv[:, :, nz - 1] = zp
        return dv.reshape(-1)

    def uniform_faces(self) -> bool:
        """True when every face of every substrate carries the same value."""
        return bool(np.all(self.face_values == self.face_values[0:1]))


def nearest_voxel(pos, origin, dx, dims):
    pos = np.asarray(pos, np.float64)
    nx, ny, nz = dims
    if pos.size == 0:
        return np.zeros(0, np.int32)
    idx = np.floor((pos - np.asarray(origin, np.float64)[None, :]) / dx).astype(np.int64)
    idx[:, 0] = np.clip(idx[:, 0], 0, nx - 1)
    idx[:, 1] = np.clip(idx[:, 1], 0, ny - 1)
    idx[:, 2] = np.clip(idx[:, 2], 0, nz - 1)
    return ((idx[:, 0] * ny + idx[:, 1]) * nz + idx[:, 2]).astype(np.int32)


def _loguniform(rng, lo, hi, n):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), n))


def _box(n, dx):
    # integer-valued corners keep the reference mesh's ceil((end-start)/dx) exact
    return -(n // 2) * dx


def make(name, nx, ny, nz, S, dx, dt, steps, D, decay, active, face_values, n_agents, seed,
         agent_mode="uniform", sigma=None, uptake=None, secretion=None, saturation=None, init_kind=None,
         agent_volume=2494.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    origin = (_box(nx, dx), _box(ny, dx), _box(nz, dx))
    ext = np.array([nx * dx, ny * dx, nz * dx])
    o = np.array(origin, np.float64)
    if agent_mode == "uniform":
        # strictly inside the box: the reference rejects positions outside it
        pos = o + rng.uniform(0.0, 1.0, (n_agents, 3)) * ext
    else:
        centre = o + ext / 2
        pos = centre + rng.normal(0.0, sigma, (n_agents, 3))
        pos = np.clip(pos, o + 1e-6 * dx, o + ext - 1e-6 * dx)
    sec = np.zeros((n_agents, S)) if secretion is None else secretion(rng, n_agents)
    upt = np.zeros((n_agents, S)) if uptake is None else uptake(rng, n_agents)
    sat = np.ones((n_agents, S)) if saturation is None else saturation(rng, n_agents)
    return Workload(name=name, nx=nx, ny=ny, nz=nz, S=S, dx=float(dx), dt=float(dt), steps=int(steps),
                    D=np.asarray(D, np.float64), decay=np.asarray(decay, np.float64),
                    dirichlet_active=np.asarray(active, np.uint8),
                    face_values=np.asarray(face_values, np.float64).reshape(6, S),
                    origin=origin, seed=seed, agent_pos=pos,
                    agent_volume=np.full(n_agents, agent_volume), secretion=sec, uptake=upt,
                    saturation=sat, net_export=np.zeros((n_agents, S)),
                    init_kind=tuple(init_kind))


def _two_substrate(name, n, dx, steps, n_agents, seed, agent_mode="uniform", sigma=None):
    """The two substrates of cube50 and cube640: oxygen-like (D=1e5, decay 0.1,
    Dirichlet 38 on all faces, initial 38) and a zero-flux secreted substrate
    (D=1e3, decay 0.01, initial noise in [0, 0.1)).  Agents take up substrate
    0 at 10/min and secrete substrate 1 at 1/min towards saturation 1."""
    fv = np.tile(np.array([38.0, 1.0]), (6, 1))

    def upt(rng, m):
        u = np.zeros((m, 2))
        u[:, 0] = 10.0
        return u

    def sec(rng, m):
        s = np.zeros((m, 2))
        s[:, 1] = 1.0
        return s

    return make(name, n, n, n, 2, dx, 0.01, steps, [1e5, 1e3], [0.1, 0.01], [1, 0], fv, n_agents, seed,
                agent_mode=agent_mode, sigma=sigma, uptake=upt, secretion=sec,
                init_kind=[("const", 38.0), ("uniform", 0.0, 0.1)])


def cube50(seed=1, steps=1000, n=50, n_agents=2000):
    return _two_substrate("cube50", n, 20.0, steps, n_agents, seed)


def cube640(seed=3, steps=1000, n=640, n_agents=1_000_000):
    return _two_substrate("cube640", n, 10.0, steps, n_agents, seed, agent_mode="gauss", sigma=1500.0 * n / 640)


def cube640_slab(axis, seed=3, steps=5, n=640, thickness=(12, 10), n_agents=20_000):
    """cube640's substrates, dx, dt and Gaussian agent ball (sigma 1500 um
    about the box centre, clamped into the box) on a slab that keeps the
    full 640-voxel lines along one axis and is thin across the other two
    (thickness voxels): every Thomas system of that axis has cube640's length
    and coefficients, at a size the reference runs in seconds."""
    dims = [thickness[0], thickness[1]]
    dims.insert(axis, n)
    nx, ny, nz = dims
    fv = np.tile(np.array([38.0, 1.0]), (6, 1))

    def upt(rng, m):
        u = np.zeros((m, 2))
        u[:, 0] = 10.0
        return u

    def sec(rng, m):
        s = np.zeros((m, 2))
        s[:, 1] = 1.0
        return s

    return make(f"cube640_slab{'xyz'[axis]}", nx, ny, nz, 2, 10.0, 0.01, steps, [1e5, 1e3], [0.1, 0.01], [1, 0],
                fv, n_agents, seed + 10 * (axis + 1), agent_mode="gauss", sigma=1500.0, uptake=upt, secretion=sec,
                init_kind=[("const", 38.0), ("uniform", 0.0, 0.1)])


def cube200(seed=2, steps=500, n=200, n_agents=100_000, S=4):
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    D = _loguniform(rng, 1e2, 1e5, S)
    decay = _loguniform(rng, 1e-3, 1.0, S)
    active = np.zeros(S, np.uint8)
    active[0] = 1
    fv = np.ones((6, S))
    fv[:, 0] = 38.0
    init = [("const", 38.0)] + [("uniform", 0.0, 1.0)] * (S - 1)
    return make("cube200", n, n, n, S, 10.0, 0.01, steps, D, decay, active, fv, n_agents, seed,
                uptake=lambda r, m: r.uniform(0.0, 10.0, (m, S)),
                secretion=lambda r, m: r.uniform(0.0, 1.0, (m, S)), init_kind=init)


def _random_env(name, rng, seed, edge_lo, edge_hi, s_lo, s_hi, agents_hi, steps, dx=20.0, steps_hi=None):
    nx, ny, nz = (int(v) for v in rng.integers(edge_lo, edge_hi + 1, 3))
    S = int(rng.integers(s_lo, s_hi + 1))
    D = _loguniform(rng, 1e2, 1e5, S)
    decay = _loguniform(rng, 1e-3, 1.0, S)
    active = (rng.uniform(0, 1, S) < 0.5).astype(np.uint8)
    # Faces: each substrate sets a random value on a random subset of faces;
    # the rest keep the reference default 1.0.
    fv = np.ones((6, S))
    on = rng.uniform(0, 1, (6, S)) < 0.6
    fv[on] = rng.uniform(0.0, 50.0, int(on.sum()))
    n_agents = int(rng.integers(0, agents_hi + 1))
    nsteps = steps if steps_hi is None else int(rng.integers(steps, steps_hi + 1))
    init = [("uniform", 0.0, 40.0)] * S
    return make(name, nx, ny, nz, S, dx, 0.01, nsteps, D, decay, active, fv, n_agents, seed,
                uptake=lambda r, m: r.uniform(0.0, 10.0, (m, S)),
                secretion=lambda r, m: r.uniform(0.0, 1.0, (m, S)), init_kind=init)


def uneven_env(index, seed=4, steps=200, agents_hi=20_000):
    rng = np.random.Generator(np.random.PCG64([seed, index]))
    return _random_env(f"uneven[{index}]", rng, seed * 100003 + index, 24, 128, 1, 6, agents_hi, steps)


def uneven_batch(n_envs=256, seed=4, steps=200, agents_hi=20_000):
    return [uneven_env(i, seed, steps, agents_hi) for i in range(n_envs)]


def serve_request(index, seed=5, steps_lo=100, steps_hi=10_000, agents_hi=200_000, edge_lo=32,
                    edge_hi=256):
    rng = np.random.Generator(np.random.PCG64([seed, index]))
    return _random_env(f"request[{index}]", rng, seed * 100003 + index, edge_lo, edge_hi, 1, 8, agents_hi,
                       steps_lo, dx=10.0, steps_hi=steps_hi)


def small_random(seed, nx=None, ny=None, nz=None, S=None, n_agents=None, steps=3, agent_mode="uniform",
                 stack=False):
    """Small random cases for parity tests (every shape feature the solver
    branches on: tiny and odd extents, several substrates, mixed Dirichlet
    activation, per-face values, agents stacked in one voxel)."""
    rng = np.random.Generator(np.random.PCG64([seed, 99]))
    nx = int(rng.integers(2, 19)) if nx is None else nx
    ny = int(rng.integers(2, 19)) if ny is None else ny
    nz = int(rng.integers(2, 19)) if nz is None else nz
    S = int(rng.integers(1, 5)) if S is None else S
    n_agents = int(rng.integers(0, 60)) if n_agents is None else n_agents
    D = _loguniform(rng, 1e2, 1e5, S)
    decay = _loguniform(rng, 1e-3, 1.0, S)
    active = (rng.uniform(0, 1, S) < 0.5).astype(np.uint8)
    fv = np.ones((6, S))
    on = rng.uniform(0, 1, (6, S)) < 0.7
    fv[on] = rng.uniform(0.0, 50.0, int(on.sum()))
    wl = make(f"small[{seed}]", nx, ny, nz, S, 20.0, 0.01, steps, D, decay, active, fv, n_agents, seed,
              agent_mode=agent_mode, sigma=20.0 * max(nx, ny, nz) / 6,
              uptake=lambda r, m: r.uniform(0.0, 10.0, (m, S)),
              secretion=lambda r, m: r.uniform(0.0, 1.0, (m, S)),
              saturation=lambda r, m: r.uniform(0.5, 2.0, (m, S)),
              init_kind=[("uniform", 0.0, 40.0)] * S)
    wl.net_export = rng.uniform(0.0, 5.0, (n_agents, S)) * (rng.uniform(0, 1, (n_agents, 1)) < 0.3)
    wl.agent_volume = rng.uniform(500.0, 5000.0, n_agents)
    if stack and n_agents:
        # pile a third of the agents into one voxel centre to exercise ordering
        c = np.array(wl.origin) + (np.array([nx, ny, nz]) // 2 + 0.5) * wl.dx
        wl.agent_pos[: max(1, n_agents // 3)] = c
    return wl
