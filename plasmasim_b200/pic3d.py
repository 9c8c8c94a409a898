"""Host-side mirror of the reference's 3D PIC step over the C ABI.

``Pic3D`` exposes the step functions of PIC/3d_pic458_domain.c under the
reference's own names (init_grid, init_particle_flat, renew_grid, renew_b4_2,
renew_e4_2, the push/deposit loops, sr_current2, sr_particle, add_flat,
sorting, thrust_f, thrust_fave, fdtd) for one domain at MPI size 1, backed by
the CUDA library ``libplasmab200.so`` built from ``plasmasim_b200/csrc``.
Failures raise ``PicError`` instead of exiting the process as the reference
does. There is no CPU fallback: without the library or a GPU every call fails.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field, fields

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libplasmab200.so")

ION, ELECTRON, BOTH = 0, 1, -1
GRID_FIELDS = ["bx", "by", "bz", "b0x", "b0y", "b0z", "ex", "ey", "ez",
               "jix", "jiy", "jiz", "jex", "jey", "jez", "ni", "ne", "phi"]

ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "particle capacity exceeded",
          4: "call out of order", 5: "device counters report lost work",
          6: "input larger than the fixed-size scratch allows",
          7: "an exchange between ranks failed"}


class PicError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where}: {ERRORS.get(code, 'error')} (code {code})")
        self.code = code


class _CConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("np", C.c_int),
        ("precision", C.c_int), ("device", C.c_int),
        ("dx", C.c_double), ("dt", C.c_double),
        ("q", C.c_double), ("mi", C.c_double), ("me", C.c_double),
        ("mu0", C.c_double), ("e0", C.c_double), ("kb", C.c_double), ("c", C.c_double),
        ("v_drift", C.c_double), ("n_all", C.c_double), ("ti", C.c_double), ("te", C.c_double),
        ("coil_r", C.c_double), ("coil_i", C.c_double), ("alpha", C.c_double),
        ("imf_x", C.c_double), ("imf_y", C.c_double), ("imf_z", C.c_double),
        ("absorb_grid", C.c_int), ("absorb_grid2", C.c_int),
        ("sigma_a", C.c_double), ("dipole_cutoff", C.c_double),
        ("add_interval", C.c_int), ("sort_interval", C.c_int),
        ("diag_every_step", C.c_int), ("poisson_clean", C.c_int),
        ("capacity", C.c_longlong), ("seed_p", C.c_ulonglong), ("seed_v", C.c_ulonglong),
        ("absorb_grid3", C.c_int), ("procs_x", C.c_int), ("procs_y", C.c_int),
        ("rank_x", C.c_int), ("rank_y", C.c_int), ("plain_fields", C.c_int), ("slot_order", C.c_int),
    ]


@dataclass
class PicConfig:
    """Run-time form of the reference's #define block (PIC/3d_pic458_domain.c:52-103)."""
    nx: int = 32
    ny: int = 32
    nz: int = 32
    np: int = 16
    precision: int = 32
    device: int = 0
    dx: float = 1.5
    dt: float = 1.5e-9
    q: float = 1.602176487e-19
    mi: float = 1.672621637e-27
    me: float = 1.672621637e-29
    mu0: float = 1.25663706144e-6
    e0: float = 8.854187817e-12
    kb: float = 1.3806504e-23
    c: float = 2.99792458e8
    v_drift: float = 1.2e7
    n_all: float = 5e10
    ti: float = 1e9
    te: float = 1e9
    coil_r: float = 2.0
    coil_i: float = 6.8e7
    alpha: float = math.pi / 2
    imf_x: float = 0.0
    imf_y: float = 0.0
    imf_z: float = 0.0
    absorb_grid: int = 32
    absorb_grid2: int = 40
    sigma_a: float = 1e-6
    dipole_cutoff: float = 210.0
    add_interval: int = 5
    sort_interval: int = 500
    diag_every_step: int = 1
    poisson_clean: int = 0
    capacity: int = 0
    seed_p: int = 0
    seed_v: int = 50
    absorb_grid3: int = 40
    procs_x: int = 1
    procs_y: int = 1
    rank_x: int = 0
    rank_y: int = 0
    plain_fields: int = 0
    slot_order: int = 0

    @classmethod
    def normalized(cls, nx, ny, nz, np_, **kw) -> "PicConfig":
        """Solar-wind plasma in normalized units (c = e0 = mu0 = q = m_e = dx = 1,
        m_i = 100): drifting Maxwellian with v_th,e = 0.05 c and drift 0.1 c along
        +z, density 0.01, dipole |B| = 0.5 at 4 cells in its equatorial plane,
        dt at half of the 4th-order stencil's 3D stability limit, no damping
        layers (every particle pushed)."""
        base = dict(nx=nx, ny=ny, nz=nz, np=np_, dx=1.0, dt=0.5 * 6.0 / (7.0 * math.sqrt(3.0)),
                    q=1.0, mi=100.0, me=1.0, mu0=1.0, e0=1.0, kb=1.0, c=1.0, v_drift=0.1,
                    n_all=0.01, ti=0.0025, te=0.0025, coil_r=2.0, coil_i=32.0,
                    alpha=math.pi / 2, absorb_grid=0, absorb_grid2=0, sigma_a=1e-6)
        base.update(kw)
        return cls(**base)

    def to_c(self) -> _CConfig:
        c = _CConfig()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c


class _CTransport(C.Structure):
    """pic_transport: the exchange callbacks of a decomposed run (C function
    pointers, held opaque here)."""
    _fields_ = [("user", C.c_void_p), ("sendrecv", C.c_void_p), ("allreduce_sum_f64", C.c_void_p)]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_llp = C.POINTER(C.c_longlong)

EXPORTED = [
    "pic_config_default", "pic_create", "pic_destroy", "pic_init_grid", "pic_init_particle_flat",
    "pic_renew_grid", "pic_renew_b4_2", "pic_renew_e4_2", "pic_push_deposit_j",
    "pic_drift_deposit_n", "pic_reduce_current", "pic_sr_particle", "pic_add_flat", "pic_sort",
    "pic_thrust_f", "pic_thrust_fave", "pic_gauss_residual", "pic_step", "pic_fdtd",
    "pic_set_particles", "pic_get_particles", "pic_particle_count", "pic_get_grid",
    "pic_set_grid", "pic_rng_counters", "pic_status", "pic_field_path", "pic_synchronize", "pic_get_stream",
    "pic_error_string", "pic_set_timing", "pic_read_timing", "pic_gauss_residual_noalloc",
    "pic_objective", "pic_adjoint", "pic_save_checkpoint", "pic_load_checkpoint", "pic_write_output",
    "pic_append_thrust", "pic_append_thrust_ave", "pic_poisson_clean",
    "pic_set_transport", "pic_group_create", "pic_group_destroy", "pic_group_transport",
    "pic_group_set_timeout",
    "pic_nccl_unique_id", "pic_nccl_transport_create", "pic_nccl_transport_destroy",
    "pic2d_config_normalized", "pic2d_create", "pic2d_destroy", "pic2d_init", "pic2d_step",
    "pic2d_thrust", "pic2d_particle_count", "pic2d_get_particles", "pic2d_get_grid",
    "pic2d_autotune", "pic2d_set_push_shape", "pic2d_set_graph", "pic2d_status", "pic2d_get_stream",
]

PHASES = ["push", "field", "sort", "add", "diag"]

_lib = None


def load_library(path: str = ""):
    """Loads the CUDA library; raises if it has not been built. The path is
    the in-tree build unless PLASMA_B200_LIB names another build of the same
    sources (for comparing builds side by side)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("PLASMA_B200_LIB") or LIB_PATH
    if not os.path.isfile(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m plasmasim_b200.build` "
            "(there is no CPU fallback)")
    L = C.CDLL(path)
    vp = C.c_void_p
    L.pic_config_default.argtypes = [C.POINTER(_CConfig), C.c_int, C.c_int, C.c_int]
    L.pic_create.argtypes = [C.POINTER(_CConfig), C.POINTER(vp)]
    for name in ["pic_destroy", "pic_init_grid", "pic_init_particle_flat", "pic_renew_grid",
                 "pic_renew_b4_2", "pic_renew_e4_2", "pic_reduce_current", "pic_sr_particle",
                 "pic_add_flat", "pic_sort", "pic_synchronize"]:
        getattr(L, name).argtypes = [vp]
    L.pic_push_deposit_j.argtypes = [vp, C.c_int]
    L.pic_drift_deposit_n.argtypes = [vp, C.c_int]
    L.pic_thrust_f.argtypes = [vp, _dp, _dp]
    L.pic_thrust_fave.argtypes = [vp, _dp, C.c_int]
    L.pic_gauss_residual.argtypes = [vp, _dp]
    L.pic_poisson_clean.argtypes = [vp]
    L.pic_set_transport.argtypes = [vp, C.POINTER(_CTransport)]
    L.pic_group_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.pic_group_destroy.argtypes = [vp]
    L.pic_group_transport.argtypes = [vp, C.c_int, C.POINTER(_CTransport)]
    L.pic_group_set_timeout.argtypes = [vp, C.c_int]
    L.pic_nccl_unique_id.argtypes = [C.c_char_p]
    L.pic_nccl_transport_create.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(_CTransport)]
    L.pic_nccl_transport_destroy.argtypes = [C.POINTER(_CTransport)]
    L.pic_objective.argtypes = [vp, C.c_int, _dp]
    for name in ["pic_save_checkpoint", "pic_load_checkpoint"]:
        getattr(L, name).argtypes = [vp, C.c_char_p, C.c_int, C.c_int]
    for name in ["pic_write_output", "pic_append_thrust", "pic_append_thrust_ave"]:
        getattr(L, name).argtypes = [vp, C.c_char_p, C.c_int]
    L.pic_adjoint.argtypes = [vp, C.c_int, C.c_int, _dp]
    L.pic_step.argtypes = [vp, C.c_int]
    L.pic_fdtd.argtypes = [vp, C.c_int]
    L.pic_set_particles.argtypes = [vp, C.c_int, _dp, _ip, C.c_longlong]
    L.pic_get_particles.argtypes = [vp, C.c_int, _dp, _ip, C.c_longlong, _llp]
    L.pic_particle_count.argtypes = [vp, C.c_int, _llp]
    L.pic_get_grid.argtypes = [vp, _dp]
    L.pic_set_grid.argtypes = [vp, _dp]
    L.pic_rng_counters.argtypes = [vp, _llp, _llp, C.c_int]
    L.pic_status.argtypes = [vp, _llp]
    L.pic_field_path.argtypes = [vp, C.POINTER(C.c_int)]
    L.pic_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.pic_set_timing.argtypes = [vp, C.c_int]
    L.pic_read_timing.argtypes = [vp, _dp, _llp, _llp]
    L.pic_gauss_residual_noalloc.argtypes = [vp, vp, vp, vp, vp, C.c_int, C.c_int, C.c_int,
                                             C.c_double, C.c_double, C.c_double, vp, vp]
    L.pic_error_string.restype = C.c_char_p
    L.pic_error_string.argtypes = [C.c_int]
    _lib = L
    return L


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class Pic3D:
    """One simulation domain on one GPU (the reference at MPI size 1)."""

    def __init__(self, cfg: PicConfig):
        self.cfg = cfg
        self.L = load_library()
        self._c = cfg.to_c()
        h = C.c_void_p()
        self._check(self.L.pic_create(C.byref(self._c), C.byref(h)), "pic_create")
        self.h = h
        self.shape = (cfg.nx + 4, cfg.ny + 4, cfg.nz + 4)

    # -- plumbing
    def _check(self, rc: int, where: str):
        if rc != 0:
            raise PicError(rc, where)

    def close(self):
        if getattr(self, "h", None):
            self.L.pic_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _call(self, name: str, *args):
        self._check(getattr(self.L, name)(self.h, *args), name)

    # -- the reference's step functions
    def init_grid(self):
        self._call("pic_init_grid")

    def init_particle_flat(self):
        self._call("pic_init_particle_flat")

    def renew_grid(self):
        self._call("pic_renew_grid")

    def renew_b4_2(self):
        self._call("pic_renew_b4_2")

    def renew_e4_2(self):
        self._call("pic_renew_e4_2")

    def push_deposit_j(self, species: int = BOTH):
        self._call("pic_push_deposit_j", species)

    def drift_deposit_n(self, species: int = BOTH):
        self._call("pic_drift_deposit_n", species)

    def reduce_current(self):
        self._call("pic_reduce_current")

    def sr_particle(self):
        self._call("pic_sr_particle")

    def add_flat(self):
        self._call("pic_add_flat")

    def sorting(self):
        self._call("pic_sort")

    def thrust_f(self):
        F = np.zeros(27)
        E = np.zeros(6)
        self._call("pic_thrust_f", _ptr(F), _ptr(E))
        return F, E

    def thrust_fave(self, reset: bool = False):
        F = np.zeros(27)
        self._call("pic_thrust_fave", _ptr(F), 1 if reset else 0)
        return F

    def set_transport(self, transport: "_CTransport"):
        """Exchanges of a decomposed run go through `transport` (which must
        outlive this context's use of it)."""
        self._transport = transport
        self._call("pic_set_transport", C.byref(transport))

    def poisson_clean(self):
        """renew_phi3 + sr_phi + sr_e: the Poisson correction of E."""
        self._call("pic_poisson_clean")

    def gauss_residual(self):
        out = np.zeros(4)
        self._call("pic_gauss_residual", _ptr(out))
        return out

    def save_checkpoint(self, directory: str, rank: int = 0, nthreads: int = 1):
        """suspend_job's files (suspend-<rank>-field.dat, suspend-<rank>-<t>-{ion,electron}.dat)."""
        self._call("pic_save_checkpoint", directory.encode(), rank, nthreads)

    def load_checkpoint(self, directory: str, rank: int = 0, nthreads: int = 1):
        """continue_job: the state from suspend_job's files."""
        self._call("pic_load_checkpoint", directory.encode(), rank, nthreads)

    def write_output(self, directory: str, step: int):
        """output(): fdtd458-0-0-<step>.dat."""
        self._call("pic_write_output", directory.encode(), step)

    def append_thrust(self, directory: str, step: int):
        """thrust_f's line in thrust458.txt."""
        self._call("pic_append_thrust", directory.encode(), step)

    def append_thrust_ave(self, directory: str, step: int):
        """thrust_fave's line in thrust458_ave.txt (every 500 steps)."""
        self._call("pic_append_thrust_ave", directory.encode(), step)

    def objective(self, nsteps: int) -> float:
        """Impulse along z delivered to the dipole over nsteps slot-stable steps."""
        out = np.zeros(1)
        self._call("pic_objective", nsteps, _ptr(out))
        return float(out[0])

    def adjoint(self, nsteps: int, checkpoint_every: int = 20):
        """(J, dJ/dI, dJ/dV) over nsteps steps by the reverse pass."""
        out = np.zeros(3)
        self._call("pic_adjoint", nsteps, checkpoint_every, _ptr(out))
        return float(out[0]), float(out[1]), float(out[2])

    def step(self, nsteps: int = 1):
        self._call("pic_step", nsteps)

    def fdtd(self, nsteps: int):
        self._call("pic_fdtd", nsteps)

    # -- state import / export (reference units, FP64)
    def set_particles(self, species: int, rows, flag=None):
        rows = np.ascontiguousarray(rows, dtype=np.float64).reshape(-1, 7)
        f = None if flag is None else np.ascontiguousarray(flag, dtype=np.int32)
        self._call("pic_set_particles", species, _ptr(rows), None if f is None else _ptr(f, _ip),
                   rows.shape[0])

    def particle_count(self, species: int) -> int:
        n = C.c_longlong()
        self._call("pic_particle_count", species, C.byref(n))
        return n.value

    def particles(self, species: int, out=None):
        """Live particles as rows (x, y, z, vx, vy, vz, n); `out` may be a
        caller-owned (e.g. pinned) float64 array with at least as many rows."""
        if out is None:
            n = self.particle_count(species)
            rows = np.zeros((max(n, 1), 7))
        else:
            rows = out
            n = rows.shape[0]
            assert rows.dtype == np.float64 and rows.flags.c_contiguous and rows.shape[1] == 7
        got = C.c_longlong()
        self._call("pic_get_particles", species, _ptr(rows), None, n, C.byref(got))
        return rows[: min(n, got.value)]

    def grid(self) -> np.ndarray:
        g = np.zeros(self.shape + (18,))
        self._call("pic_get_grid", _ptr(g))
        return g

    def set_grid(self, g):
        g = np.ascontiguousarray(g, dtype=np.float64)
        if g.shape != self.shape + (18,):
            raise ValueError(f"grid shape {g.shape} != {self.shape + (18,)}")
        self._call("pic_set_grid", _ptr(g))

    def rng_counters(self, set_to=None):
        p, v = C.c_longlong(), C.c_longlong()
        if set_to is not None:
            p.value, v.value = set_to
            self._call("pic_rng_counters", C.byref(p), C.byref(v), 1)
        else:
            self._call("pic_rng_counters", C.byref(p), C.byref(v), 0)
        return p.value, v.value

    def status(self):
        out = np.zeros(8, dtype=np.int64)
        rc = self.L.pic_status(self.h, _ptr(out, _llp))
        return rc, out

    def staged_fields(self) -> bool:
        """True when renew_b4_2 / renew_e4_2 run the TMA-staged stencil kernels."""
        v = C.c_int()
        self._call("pic_field_path", C.byref(v))
        return bool(v.value)

    def synchronize(self):
        self._call("pic_synchronize")

    def stream_handle(self) -> int:
        s = C.c_void_p()
        self._call("pic_get_stream", C.byref(s))
        return s.value or 0

    def set_timing(self, enable: bool):
        self._call("pic_set_timing", 1 if enable else 0)

    def read_timing(self):
        """(ms per phase dict, event pairs per phase dict, launches since creation)."""
        ms = np.zeros(8)
        pairs = np.zeros(8, dtype=np.int64)
        launches = C.c_longlong()
        self._call("pic_read_timing", _ptr(ms), _ptr(pairs, _llp), C.byref(launches))
        return ({p: float(ms[i]) for i, p in enumerate(PHASES)},
                {p: int(pairs[i]) for i, p in enumerate(PHASES)}, launches.value)
