"""ctypes access to the CPU oracles (test infrastructure only).

``Oracle``    -- the project's FP64 restatement (oracle/pic_oracle.c).
``Reference`` -- the reference program compiled by oracle/build.py
                 (oracle/_ref/libref3d_<name>.so), driven through
                 oracle/ref_harness.c.

Both exchange grids as the reference's 18-double Grid records in
grid[k][l][m] order and particles as rows (x, y, z, vx, vy, vz, n) + flag.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import build as _build

GRID_FIELDS = ["bx", "by", "bz", "b0x", "b0y", "b0z", "ex", "ey", "ez",
               "jix", "jiy", "jiz", "jex", "jey", "jez", "ni", "ne", "phi"]
F = {name: i for i, name in enumerate(GRID_FIELDS)}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_long)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def params_from_defines(d: dict) -> dict:
    """Run-time parameter dict from an oracle.build REF_CONFIGS entry."""
    alpha = d["ORACLE_ALPHA"]
    alpha = math.pi / 2 if alpha == "(Pi/2.)" else float(alpha)
    mp = d.get("ORACLE_MP", 1.672621637e-27)
    return dict(
        nx=d["ORACLE_NX"], ny=d["ORACLE_NY"], nz=d["ORACLE_NZ"], np=d["ORACLE_NP"],
        thread_n=d["ORACLE_THREADS"], dx=d["ORACLE_DX"], dt=d["ORACLE_DT"],
        q=d.get("ORACLE_Q", 1.602176487e-19), mi=mp, me=mp / d["ORACLE_MASS_RATIO"],
        mu0=d.get("ORACLE_MU0", 1.25663706144e-6), e0=d.get("ORACLE_E0", 8.854187817e-12),
        kb=d.get("ORACLE_KB", 1.3806504e-23), c=d.get("ORACLE_C", 2.99792458e8),
        V=d["ORACLE_V"], Nall=d["ORACLE_NALL"], Ti=d["ORACLE_TI"], Te=d["ORACLE_TE"],
        R=d["ORACLE_R"], I=d["ORACLE_I"], alpha=alpha, imf_x=0.0, imf_y=0.0, imf_z=0.0,
        absorb=d["ORACLE_ABSORB"], absorb2=d["ORACLE_ABSORB2"],
        sigma_a=d["ORACLE_SIGMA_A"], cutoff=210.0,
    )


_ORDER = ["nx", "ny", "nz", "np", "thread_n", "dx", "dt", "q", "mi", "me", "mu0", "e0",
          "kb", "c", "V", "Nall", "Ti", "Te", "R", "I", "alpha", "imf_x", "imf_y", "imf_z",
          "absorb", "absorb2", "sigma_a", "cutoff"]


class Oracle:
    """FP64 CPU restatement of the reference step (one domain, MPI size 1)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            path = _build.ORACLE_SO
            if not os.path.isfile(path):
                _build.build_oracle()
            L = C.CDLL(path)
            L.or_create.restype = C.c_void_p
            L.or_create.argtypes = [_dp]
            for name in ["or_destroy", "or_init_grid", "or_init_particle_flat", "or_add_flat",
                         "or_renew_grid", "or_renew_b", "or_renew_e", "or_sr_b", "or_sr_e",
                         "or_sr_current2", "or_push_j", "or_drift_n", "or_sr_particle",
                         "or_sort"]:
                getattr(L, name).argtypes = [C.c_void_p]
                getattr(L, name).restype = None
            L.or_grid_nodes.restype = C.c_long
            L.or_grid_nodes.argtypes = [C.c_void_p]
            L.or_get_grid.argtypes = [C.c_void_p, _dp]
            L.or_set_grid.argtypes = [C.c_void_p, _dp]
            L.or_get_sigma.argtypes = [C.c_void_p, _dp]
            L.or_count.restype = C.c_long
            L.or_count.argtypes = [C.c_void_p, C.c_int]
            L.or_set_particles.argtypes = [C.c_void_p, C.c_int, _dp, _ip, C.c_long]
            L.or_get_particles.restype = C.c_long
            L.or_get_particles.argtypes = [C.c_void_p, C.c_int, _dp, _ip, C.c_long]
            L.or_rng_counter.restype = C.c_longlong
            L.or_rng_counter.argtypes = [C.c_void_p, C.c_int, C.c_longlong]
            L.or_thrust.argtypes = [C.c_void_p, _dp]
            L.or_gauss_residual.argtypes = [C.c_void_p, _dp]
            L.or_gather.argtypes = [C.c_void_p, _dp, _dp]
            L.or_step.argtypes = [C.c_void_p, _ip, _ip, C.c_int, C.c_int]
            L.or_fdtd.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
            L.or_fave.argtypes = [C.c_void_p, _dp]
            L.or_oob_count.restype = C.c_long
            L.or_tl_create.restype = C.c_void_p
            L.or_tl_create.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double]
            L.or_tl_destroy.argtypes = [C.c_void_p]
            L.or_tl_result.argtypes = [C.c_void_p, _dp]
            L.or_tl_step.argtypes = [C.c_void_p, C.c_void_p, _ip, C.c_int]
            L.or_plain_step.restype = C.c_double
            L.or_plain_step.argtypes = [C.c_void_p, _ip, C.c_int]
            L.or_dipole_force.restype = C.c_double
            L.or_dipole_force.argtypes = [C.c_void_p]
            cls._lib = L
        return cls._lib

    def __init__(self, params: dict):
        self.p = dict(params)
        arr = np.array([float(self.p[k]) for k in _ORDER], dtype=np.float64)
        self.L = self.lib()
        self.h = self.L.or_create(_ptr(arr))
        self.shape = (self.p["nx"] + 4, self.p["ny"] + 4, self.p["nz"] + 4)
        self.c_add = C.c_int(0)
        self.c_thrust = C.c_int(0)

    def close(self):
        if self.h:
            self.L.or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def call(self, name):
        getattr(self.L, "or_" + name)(self.h)

    def grid(self) -> np.ndarray:
        g = np.zeros(self.shape + (18,), dtype=np.float64)
        self.L.or_get_grid(self.h, _ptr(g))
        return g

    def set_grid(self, g: np.ndarray):
        g = np.ascontiguousarray(g, dtype=np.float64)
        assert g.shape == self.shape + (18,)
        self.L.or_set_grid(self.h, _ptr(g))

    def sigma(self) -> np.ndarray:
        s = np.zeros(tuple(2 * n for n in self.shape), dtype=np.float64)
        self.L.or_get_sigma(self.h, _ptr(s))
        return s

    def particles(self, species: int):
        n = self.L.or_count(self.h, species)
        rows = np.zeros((max(n, 1), 7))
        flag = np.zeros(max(n, 1), dtype=np.int32)
        self.L.or_get_particles(self.h, species, _ptr(rows), _ptr(flag, _ip), n)
        return rows[:n], flag[:n]

    def set_particles(self, species: int, rows: np.ndarray, flag=None):
        rows = np.ascontiguousarray(rows, dtype=np.float64).reshape(-1, 7)
        f = None if flag is None else np.ascontiguousarray(flag, dtype=np.int32)
        self.L.or_set_particles(self.h, species, _ptr(rows), None if f is None else _ptr(f, _ip),
                                rows.shape[0])

    def rng_counter(self, which: int, set_to: int = -1) -> int:
        return int(self.L.or_rng_counter(self.h, which, set_to))

    def thrust(self) -> np.ndarray:
        out = np.zeros(33)
        self.L.or_thrust(self.h, _ptr(out))
        return out

    def gauss(self) -> np.ndarray:
        out = np.zeros(4)
        self.L.or_gauss_residual(self.h, _ptr(out))
        return out

    def gather(self, xyz) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        out = np.zeros(6)
        self.L.or_gather(self.h, _ptr(xyz), _ptr(out))
        return out

    def step(self, sort_every=500, add_every=5):
        self.L.or_step(self.h, C.byref(self.c_add), C.byref(self.c_thrust), sort_every, add_every)

    def fdtd(self, nsteps, sort_every=500, add_every=5):
        self.L.or_fdtd(self.h, nsteps, sort_every, add_every)

    def fave(self):
        out = np.zeros(27)
        self.L.or_fave(self.h, _ptr(out))
        return out

    def dipole_force(self) -> float:
        """F = -sum s q n dx^3 (v x B0(x))_z over the current particles."""
        return float(self.L.or_dipole_force(self.h))

    def plain_steps(self, nsteps, add_every=5) -> float:
        """nsteps loop bodies without sorting; returns sum of dt * F after each."""
        J = 0.0
        for _ in range(nsteps):
            J += self.L.or_plain_step(self.h, C.byref(self.c_add), add_every)
        return J

    def tangent_run(self, nsteps, dI, dV, add_every=5):
        """FP64 tangent-linear of nsteps loop bodies (no sorting) from the
        current state, seeded in direction (dI, dV); returns (J, dJ)."""
        arr = np.array([float(self.p[k]) for k in _ORDER], dtype=np.float64)
        t = self.L.or_tl_create(self.h, _ptr(arr), dI, dV)
        try:
            for _ in range(nsteps):
                self.L.or_tl_step(self.h, t, C.byref(self.c_add), add_every)
            out = np.zeros(2)
            self.L.or_tl_result(t, _ptr(out))
        finally:
            self.L.or_tl_destroy(t)
        return float(out[0]), float(out[1])


def sine_matrix(n: int) -> np.ndarray:
    """S[k][j] = sin(pi j k / n): the transform of the reference's sinft
    (PIC/3d_pic458_domain.c:8182-8210) on data[1..n] = rho[0..n-1], which
    sets data[1] = 0, so row and column 0 vanish."""
    j = np.arange(n, dtype=np.float64)
    return np.sin(np.pi * np.outer(j, j) / n)


def renew_phi3(grid: np.ndarray, dx: float, q: float, e0: float, absorb3: int) -> np.ndarray:
    """renew_phi3 + sr_phi + sr_e at MPI size 1 (PIC/3d_pic458_domain.c
    :8315-8665, :1389-1574, and the E wrap of sr_e), restated with numpy on a
    grid of records [x][y][z][18]; returns the new grid.

    - rho (:8338-8355): on interior cells (k, l, m) with 0 < k-2 < Nx - A3 ... the
      Gauss residual -( -q (ni - ne)/e0 + div4 E ), div4 the (27, -1)/24 stencil
      of E's forward differences; zero elsewhere (A3 = Absorb_grid3).
    - sine transforms along z, y, x (fft_z/y/x :7990-8084), division by
      A = -(sin^2(pi ky/2Ny) + sin^2(pi kz/2Nz) + sin^2(pi kx/2Nx)) / (dx/2)^2
      (zero where A = 0, :8502-8511), inverse transforms with 2/N (:8086-8180).
    - phi on the interior (:8655-8661); sr_phi wraps its two ghost planes in x,
      then in y over all x; E += the (27, -1)/24 backward gradient of phi on
      the interior (:1563-1572); sr_e wraps E's ghost planes in x, then y."""
    EX, EY, EZ, NI, NE, PHI = 6, 7, 8, 15, 16, 17
    g = grid.copy()
    gx, gy, gz = g.shape[:3]
    nx, ny, nz = gx - 4, gy - 4, gz - 4
    I = slice(2, nx + 2)
    Jy = slice(2, ny + 2)
    K = slice(2, nz + 2)

    def sh(a, dk=0, dl=0, dm=0):
        return a[2 + dk:nx + 2 + dk, 2 + dl:ny + 2 + dl, 2 + dm:nz + 2 + dm]

    ex, ey, ez = g[..., EX], g[..., EY], g[..., EZ]
    div = ((-sh(ex, 2) + 27 * sh(ex, 1) - 27 * sh(ex) + sh(ex, -1))
           + (-sh(ey, 0, 2) + 27 * sh(ey, 0, 1) - 27 * sh(ey) + sh(ey, 0, -1))
           + (-sh(ez, 0, 0, 2) + 27 * sh(ez, 0, 0, 1) - 27 * sh(ez) + sh(ez, 0, 0, -1))) / (24. * dx)
    rho = -(-q * (g[I, Jy, K, NI] - g[I, Jy, K, NE]) / e0 + div)
    kx = np.arange(nx)[:, None, None]
    ky = np.arange(ny)[None, :, None]
    kz = np.arange(nz)[None, None, :]
    mask = ((kx > absorb3) & (kx < nx - absorb3) & (ky > absorb3) & (ky < ny - absorb3)
            & (kz >= absorb3) & (kz < nz - absorb3))
    rho = np.where(mask, rho, 0.0)
    Sx, Sy, Sz = sine_matrix(nx), sine_matrix(ny), sine_matrix(nz)
    t = np.einsum("xyz,cz->xyc", rho, Sz)
    t = np.einsum("xyz,by->xbz", t, Sy)
    t = np.einsum("xyz,ax->ayz", t, Sx)
    A = -(np.sin(np.pi * ky / ny / 2.) ** 2 + np.sin(np.pi * kz / nz / 2.) ** 2
          + np.sin(np.pi * kx / nx / 2.) ** 2) / (dx / 2.) ** 2
    t = np.where(A == 0., 0.0, t / np.where(A == 0., 1.0, A))
    t = 2. * np.einsum("xyz,ax->ayz", t, Sx) / nx
    t = 2. * np.einsum("xyz,by->xbz", t, Sy) / ny
    t = 2. * np.einsum("xyz,cz->xyc", t, Sz) / nz
    g[I, Jy, K, PHI] = t
    # sr_phi at size 1: x planes (all y, z), then y planes (all x, z)
    g[0:2, :, :, PHI] = g[nx:nx + 2, :, :, PHI]
    g[nx + 2:nx + 4, :, :, PHI] = g[2:4, :, :, PHI]
    g[:, 0:2, :, PHI] = g[:, ny:ny + 2, :, PHI]
    g[:, ny + 2:ny + 4, :, PHI] = g[:, 2:4, :, PHI]
    phi = g[..., PHI]
    g[I, Jy, K, EX] += (-sh(phi, 1) + 27 * sh(phi) - 27 * sh(phi, -1) + sh(phi, -2)) / (24. * dx)
    g[I, Jy, K, EY] += (-sh(phi, 0, 1) + 27 * sh(phi) - 27 * sh(phi, 0, -1) + sh(phi, 0, -2)) / (24. * dx)
    g[I, Jy, K, EZ] += (-sh(phi, 0, 0, 1) + 27 * sh(phi) - 27 * sh(phi, 0, 0, -1) + sh(phi, 0, 0, -2)) / (24. * dx)
    for f in (EX, EY, EZ):
        g[0:2, :, :, f] = g[nx:nx + 2, :, :, f]
        g[nx + 2:nx + 4, :, :, f] = g[2:4, :, :, f]
        g[:, 0:2, :, f] = g[:, ny:ny + 2, :, f]
        g[:, ny + 2:ny + 4, :, f] = g[:, 2:4, :, f]
    return g


REF_OPS = dict(renew_grid=1, renew_b=2, sr_b=3, push_j=4, drift_n=5, reduce=6,
               sr_current=7, renew_e=8, sr_e=9, sr_particle=10, add_flat=11, sort=12,
               thrust_f=13)


class Reference:
    """The reference program itself, compiled at one geometry. Its state is
    process-global: use one instance per process."""

    def __init__(self, name: str):
        path = _build.ref_lib_path(name)
        if not os.path.isfile(path):
            _build.build_ref(name)
        L = C.CDLL(path)
        L.ref_grid_nodes.restype = C.c_long
        L.ref_get_grid.argtypes = [_dp]
        L.ref_set_grid.argtypes = [_dp]
        L.ref_get_sigma.argtypes = [_dp]
        L.ref_get_grid_thread.argtypes = [C.c_int, _dp]
        L.ref_count.restype = C.c_long
        L.ref_count.argtypes = [C.c_int]
        L.ref_get_particles.restype = C.c_long
        L.ref_get_particles.argtypes = [C.c_int, _dp, _ip, C.c_long]
        L.ref_set_particles.argtypes = [_dp, _ip, _lp, _dp, _ip, _lp]
        L.ref_rng_counter.restype = C.c_longlong
        L.ref_rng_counter.argtypes = [C.c_int, C.c_int, C.c_longlong]
        L.ref_thrust_sums.argtypes = [_dp, C.c_int]
        L.ref_gather.argtypes = [_dp, _dp]
        L.ref_fave.argtypes = [_dp]
        self.L = L
        self.name = name
        self.defines = _build.REF_CONFIGS[name]
        self.params = params_from_defines(self.defines)
        d = (C.c_int * 10)()
        L.ref_dims(d)
        self.dims = list(d)
        self.shape = (d[0] + 4, d[1] + 4, d[2] + 4)

    def op(self, name):
        self.L.ref_op(REF_OPS[name])

    def suspend(self):
        """suspend_job: the reference's checkpoint files in the working directory."""
        self.L.ref_suspend()

    def continue_job(self):
        """continue_job: the state from checkpoint files in the working directory."""
        self.L.ref_continue()

    def output(self, step: int):
        """output(): fdtd458-0-0-<step>.dat in the working directory."""
        self.L.ref_output(step)

    def renew_phi3(self):
        """renew_phi3 + sr_phi + sr_e (a geometry built with the PHI blocks)."""
        if self.L.ref_renew_phi3() != 0:
            raise RuntimeError(f"reference geometry {self.name} has no PHI blocks")

    def init_grid(self):
        self.L.ref_init_grid()

    def init_particle_flat(self):
        self.L.ref_init_particle_flat()

    def init_rng(self):
        self.L.ref_init_rng()

    def grid(self) -> np.ndarray:
        g = np.zeros(self.shape + (18,))
        self.L.ref_get_grid(_ptr(g))
        return g

    def set_grid(self, g):
        g = np.ascontiguousarray(g, dtype=np.float64)
        self.L.ref_set_grid(_ptr(g))

    def sigma(self):
        s = np.zeros(tuple(2 * n for n in self.shape))
        self.L.ref_get_sigma(_ptr(s))
        return s

    def particles(self, species: int):
        n = self.L.ref_count(species)
        rows = np.zeros((max(n, 1), 7))
        flag = np.zeros(max(n, 1), dtype=np.int32)
        self.L.ref_get_particles(species, _ptr(rows), _ptr(flag, _ip), n)
        return rows[:n], flag[:n]

    def set_particles(self, ion_rows, electron_rows, ion_flag=None, electron_flag=None):
        ir = np.ascontiguousarray(ion_rows, dtype=np.float64).reshape(-1, 7)
        er = np.ascontiguousarray(electron_rows, dtype=np.float64).reshape(-1, 7)
        ic = np.array([ir.shape[0]], dtype=np.int64)
        ec = np.array([er.shape[0]], dtype=np.int64)
        fi = None if ion_flag is None else np.ascontiguousarray(ion_flag, dtype=np.int32)
        fe = None if electron_flag is None else np.ascontiguousarray(electron_flag, dtype=np.int32)
        rc = self.L.ref_set_particles(_ptr(ir), None if fi is None else _ptr(fi, _ip), _ptr(ic, _lp),
                                      _ptr(er), None if fe is None else _ptr(fe, _ip), _ptr(ec, _lp))
        assert rc == 0

    def rng_counter(self, which: int, set_to: int = -1) -> int:
        return int(self.L.ref_rng_counter(0, which, set_to))

    def thrust(self, include_tail=True) -> np.ndarray:
        out = np.zeros(33)
        self.L.ref_thrust_sums(_ptr(out), 1 if include_tail else 0)
        return out

    def gather(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        out = np.zeros(6)
        self.L.ref_gather(_ptr(xyz), _ptr(out))
        return out

    def fdtd(self, nsteps: int):
        self.L.ref_fdtd(nsteps)

    def fave(self):
        out = np.zeros(27)
        self.L.ref_fave(_ptr(out))
        return out


GRID2D_FIELDS = ["b0x", "b0y", "b0z", "bx", "by", "bz", "ex", "ey", "ez",
                 "jix", "jiy", "jiz", "jex", "jey", "jez", "ni", "ne", "phi"]
F2 = {name: i for i, name in enumerate(GRID2D_FIELDS)}


class Reference2D:
    """The 2D reference program (PIC2D/2d_pic278_mpi.c) compiled at one
    geometry by oracle/build.py, driven through oracle/ref2d_harness.c. Its
    state is process-global: use one instance per process (or per test that
    re-initialises it). Particle rows: x, z, vx, vy, vz, n."""

    def __init__(self, name: str):
        path = _build.ref2d_lib_path(name)
        if not os.path.isfile(path):
            _build.build_ref2d(name)
        L = C.CDLL(path)
        L.ref2d_grid_nodes.restype = C.c_long
        L.ref2d_get_grid.argtypes = [_dp]
        L.ref2d_set_grid.argtypes = [_dp]
        L.ref2d_count.restype = C.c_long
        L.ref2d_count.argtypes = [C.c_int]
        L.ref2d_get_particles.restype = C.c_long
        L.ref2d_get_particles.argtypes = [C.c_int, _dp, _ip, C.c_long]
        L.ref2d_step.argtypes = [C.c_int]
        L.ref2d_thrust.argtypes = [_dp]
        L.ref2d_sinft.argtypes = [C.c_int, _dp]
        L.ref2d_dims.argtypes = [_ip]
        self.L = L
        d = np.zeros(10, dtype=np.int32)
        L.ref2d_dims(_ptr(d, _ip))
        self.nx, self.nz, self.np = int(d[0]), int(d[1]), int(d[2])
        self.shape = (self.nx + 4, self.nz + 4)
        self.params = dict(_build.REF2D_CONFIGS[name])

    def init(self):
        self.L.ref2d_init()

    def step(self, add_every=250):
        self.L.ref2d_step(add_every)

    def grid(self) -> np.ndarray:
        g = np.zeros(self.shape + (18,), dtype=np.float64)
        self.L.ref2d_get_grid(_ptr(g))
        return g

    def particles(self, species: int):
        n = self.L.ref2d_count(species)
        rows = np.zeros((max(n, 1), 6))
        flag = np.zeros(max(n, 1), dtype=np.int32)
        self.L.ref2d_get_particles(species, _ptr(rows), _ptr(flag, _ip), n)
        return rows[:n], flag[:n]

    def thrust(self) -> np.ndarray:
        out = np.zeros(3)
        self.L.ref2d_thrust(_ptr(out))
        return out

    def sinft(self, y) -> np.ndarray:
        y = np.array(y, dtype=np.float64)
        self.L.ref2d_sinft(len(y), _ptr(y))
        return y
