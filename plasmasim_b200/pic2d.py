"""ctypes mirror of the batched 2D API (pic2d_* in include/plasma_b200.h):
many independent runs of PIC2D/2d_pic278_mpi.c advanced together on one GPU."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, fields

import numpy as np

from .pic3d import PicError, load_library

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_llp = C.POINTER(C.c_longlong)

GRID2D_FIELDS = ["b0x", "b0y", "b0z", "bx", "by", "bz", "ex", "ey", "ez",
                 "jix", "jiy", "jiz", "jex", "jey", "jez", "ni", "ne", "phi"]


class _C2Config(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("nz", C.c_int), ("np", C.c_int), ("add_interval", C.c_int),
        ("dx", C.c_double), ("dt", C.c_double), ("q", C.c_double), ("mi", C.c_double),
        ("me", C.c_double), ("mu0", C.c_double), ("e0", C.c_double), ("kb", C.c_double),
        ("c", C.c_double), ("v_drift", C.c_double), ("n_all", C.c_double), ("ti", C.c_double),
        ("te", C.c_double), ("coil_i", C.c_double), ("imf_x", C.c_double), ("imf_y", C.c_double),
        ("imf_z", C.c_double), ("absorb_grid", C.c_int), ("absorb_grid2", C.c_int),
        ("absorb_grid3", C.c_int), ("sort_interval", C.c_int), ("sigma_a", C.c_double),
        ("seed_p", C.c_ulonglong), ("seed_v", C.c_ulonglong), ("capacity", C.c_longlong),
    ]


@dataclass
class Pic2DConfig:
    nx: int
    nz: int
    np: int
    add_interval: int = 250
    dx: float = 1.0
    dt: float = 0.5 * 6.0 / (7.0 * math.sqrt(2.0))
    q: float = 1.0
    mi: float = 100.0
    me: float = 1.0
    mu0: float = 1.0
    e0: float = 1.0
    kb: float = 1.0
    c: float = 1.0
    v_drift: float = 0.1
    n_all: float = 0.01
    ti: float = 0.0025
    te: float = 0.0025
    coil_i: float = 12.0
    imf_x: float = 0.0
    imf_y: float = 0.0
    imf_z: float = 0.0
    absorb_grid: int = 32
    absorb_grid2: int = 16
    absorb_grid3: int = 32
    sort_interval: int = 12
    sigma_a: float = 1e-6
    seed_p: int = 0
    seed_v: int = 50
    capacity: int = 0

    def to_c(self) -> _C2Config:
        c = _C2Config()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c


_bound = False


def _bind(L):
    global _bound
    if _bound:
        return
    vp = C.c_void_p
    L.pic2d_create.argtypes = [C.POINTER(_C2Config), C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
    for name in ["pic2d_destroy", "pic2d_init"]:
        getattr(L, name).argtypes = [vp]
    L.pic2d_step.argtypes = [vp, C.c_int]
    L.pic2d_thrust.argtypes = [vp, _dp]
    L.pic2d_particle_count.argtypes = [vp, C.c_int, C.c_int, _llp]
    L.pic2d_get_particles.argtypes = [vp, C.c_int, C.c_int, _dp, C.c_longlong, _llp]
    L.pic2d_get_grid.argtypes = [vp, C.c_int, _dp]
    L.pic2d_autotune.argtypes = [vp, _ip]
    L.pic2d_set_graph.argtypes = [vp, C.c_int]
    L.pic2d_set_push_shape.argtypes = [vp, C.c_int, C.c_int]
    L.pic2d_status.argtypes = [vp, _llp]
    L.pic2d_get_stream.argtypes = [vp, C.POINTER(vp)]
    _bound = True


class Pic2DBatch:
    """A batch of independent 2D runs (each the reference at MPI size 1)."""

    def __init__(self, cfgs, precision: int = 32, device: int = 0):
        self.L = load_library()
        _bind(self.L)
        self.cfgs = list(cfgs)
        arr = (_C2Config * len(self.cfgs))(*[c.to_c() for c in self.cfgs])
        h = C.c_void_p()
        self._check(self.L.pic2d_create(arr, len(self.cfgs), precision, device, C.byref(h)), "pic2d_create")
        self.h = h

    def _check(self, rc, where):
        if rc != 0:
            raise PicError(rc, where)

    def close(self):
        if getattr(self, "h", None):
            self.L.pic2d_destroy(self.h)
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

    def init(self):
        self._check(self.L.pic2d_init(self.h), "pic2d_init")

    def step(self, nsteps: int = 1):
        self._check(self.L.pic2d_step(self.h, nsteps), "pic2d_step")

    def thrust(self) -> np.ndarray:
        out = np.zeros(3 * len(self.cfgs))
        self._check(self.L.pic2d_thrust(self.h, out.ctypes.data_as(_dp)), "pic2d_thrust")
        return out.reshape(-1, 3)

    def count(self, run: int, species: int) -> int:
        n = C.c_longlong()
        self._check(self.L.pic2d_particle_count(self.h, run, species, C.byref(n)), "pic2d_particle_count")
        return int(n.value)

    def particles(self, run: int, species: int) -> np.ndarray:
        n = self.count(run, species)
        rows = np.zeros((max(n, 1), 6))
        got = C.c_longlong()
        self._check(self.L.pic2d_get_particles(self.h, run, species, rows.ctypes.data_as(_dp), n,
                                               C.byref(got)), "pic2d_get_particles")
        return rows[: got.value]

    def grid(self, run: int) -> np.ndarray:
        c = self.cfgs[run]
        g = np.zeros((c.nx + 4, c.nz + 4, 18))
        self._check(self.L.pic2d_get_grid(self.h, run, g.ctypes.data_as(_dp)), "pic2d_get_grid")
        return g

    def autotune(self):
        out = np.zeros(2, dtype=np.int32)
        self._check(self.L.pic2d_autotune(self.h, out.ctypes.data_as(_ip)), "pic2d_autotune")
        return int(out[0]), int(out[1])

    def set_push_shape(self, tile_rows: int, blocks: int):
        self._check(self.L.pic2d_set_push_shape(self.h, tile_rows, blocks), "pic2d_set_push_shape")

    def set_graph(self, enable: bool):
        self._check(self.L.pic2d_set_graph(self.h, int(enable)), "pic2d_set_graph")

    def status(self):
        out = np.zeros(8, dtype=np.int64)
        rc = self.L.pic2d_status(self.h, out.ctypes.data_as(_llp))
        return rc, out

    def stream_handle(self) -> int:
        s = C.c_void_p()
        self._check(self.L.pic2d_get_stream(self.h, C.byref(s)), "pic2d_get_stream")
        return s.value or 0
