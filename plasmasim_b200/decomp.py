"""Domain decomposition of the 3D step over PROCESS_Nx x PROCESS_Ny ranks
(PIC/3d_pic458_domain.c:100-101, :194-211): every rank is a Pic3D context of
Grid_Nx x Grid_Ny x Grid_Nz cells whose exchanges -- sr_b, sr_e, sr_current2,
sr_particle and thrust_f's MPI_Allreduce -- go through a transport.

- `LocalGroup` / `DecomposedPic3D`: all ranks in one process, one host thread
  per rank, on one GPU or several (an in-process transport: device-to-device
  copies ordered by CUDA events, rendezvous on the host).
- `NcclTransport`: one process per GPU, NCCL send/recv and all-reduce; the
  unique id travels through a torch.distributed store.

Each rank's random streams are keyed as the reference keys them:
(myrank_y PROCESS_Nx + myrank_x) * 10000 + the single-rank keys (:442-443).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .pic3d import Pic3D, PicConfig, PicError, _CTransport, load_library


def rank_config(cfg: PicConfig, procs_x: int, procs_y: int, rank: int, device: int | None = None) -> PicConfig:
    """The configuration of rank `rank` (myrank_y * procs_x + myrank_x) of a
    procs_x x procs_y decomposition whose ranks hold cfg.nx x cfg.ny x cfg.nz cells each."""
    rx, ry = rank % procs_x, rank // procs_x
    kw = dict(procs_x=procs_x, procs_y=procs_y, rank_x=rx, rank_y=ry,
              seed_p=cfg.seed_p + 10000 * rank, seed_v=cfg.seed_v + 10000 * rank)
    if device is not None:
        kw["device"] = device
    return dataclasses.replace(cfg, **kw)


class LocalGroup:
    """pic_group: an in-process transport for `nranks` ranks."""

    def __init__(self, nranks: int):
        self.L = load_library()
        h = C.c_void_p()
        rc = self.L.pic_group_create(nranks, C.byref(h))
        if rc:
            raise PicError(rc, "pic_group_create")
        self.h = h
        self.n = nranks
        self._transports = []
        for r in range(nranks):
            t = _CTransport()
            rc = self.L.pic_group_transport(self.h, r, C.byref(t))
            if rc:
                raise PicError(rc, "pic_group_transport")
            self._transports.append(t)

    def transport(self, rank: int) -> _CTransport:
        return self._transports[rank]

    def set_timeout(self, ms: int):
        """pic_group_set_timeout: the host rendezvous limit of every exchange."""
        rc = self.L.pic_group_set_timeout(self.h, int(ms))
        if rc:
            raise PicError(rc, "pic_group_set_timeout")

    def close(self):
        if self.h:
            self.L.pic_group_destroy(self.h)
            self.h = None


class NcclTransport:
    """pic_nccl_transport_create for this process's rank; rank 0 creates the
    NCCL unique id and publishes it in `store` (a torch.distributed Store)."""

    @staticmethod
    def share_unique_id(store, rank: int, key: str = "plasma_b200_nccl_id") -> bytes:
        """Rank 0 makes the NCCL unique id and sets it in the store; every
        rank returns it from the store."""
        if rank == 0:
            buf = C.create_string_buffer(128)
            rc = load_library().pic_nccl_unique_id(buf)
            if rc:
                raise PicError(rc, "pic_nccl_unique_id")
            store.set(key, bytes(buf.raw))
        return bytes(store.get(key))

    def __init__(self, store, nranks: int, rank: int, device: int, key: str = "plasma_b200_nccl_id"):
        self.L = load_library()
        uid = self.share_unique_id(store, rank, key)
        self.t = _CTransport()
        rc = self.L.pic_nccl_transport_create(uid, nranks, rank, device, C.byref(self.t))
        if rc:
            raise PicError(rc, "pic_nccl_transport_create")

    def transport(self) -> _CTransport:
        return self.t

    def close(self):
        if self.t.user:
            self.L.pic_nccl_transport_destroy(C.byref(self.t))


class DecomposedPic3D:
    """procs_x x procs_y ranks of Pic3D in this process, each driven by its own
    thread (every call runs on all ranks at once and returns the per-rank
    results in rank order)."""

    def __init__(self, cfg: PicConfig, procs_x: int, procs_y: int, devices=None):
        self.px, self.py = procs_x, procs_y
        self.n = procs_x * procs_y
        self.group = LocalGroup(self.n)
        devs = list(devices) if devices else [cfg.device]
        self.ranks = [Pic3D(rank_config(cfg, procs_x, procs_y, r, devs[r % len(devs)])) for r in range(self.n)]
        for r, P in enumerate(self.ranks):
            P.set_transport(self.group.transport(r))
        self.pool = ThreadPoolExecutor(max_workers=self.n)

    def all(self, name: str, *args):
        futures = [self.pool.submit(getattr(P, name), *args) for P in self.ranks]
        return [f.result() for f in futures]

    def each(self, fn):
        """fn(rank, Pic3D) on every rank at once."""
        futures = [self.pool.submit(fn, r, P) for r, P in enumerate(self.ranks)]
        return [f.result() for f in futures]

    def __getattr__(self, name):
        if name.startswith("_") or name in ("ranks", "pool", "group"):
            raise AttributeError(name)
        return lambda *args: self.all(name, *args)

    def thrust_f(self):
        """The summed thrust (thrust_f's MPI_Allreduce): every rank returns the same."""
        return self.all("thrust_f")[0]

    def close(self):
        for P in self.ranks:
            P.close()
        self.group.close()
        self.pool.shutdown()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def global_particles(parts_per_rank, procs_x: int, nx: int, ny: int, dx: float):
    """Particle rows of every rank in global coordinates (x + myrank_x Nx dx,
    y + myrank_y Ny dx), stacked in rank order."""
    out = []
    for r, rows in enumerate(parts_per_rank):
        rows = np.array(rows, dtype=np.float64, copy=True)
        rows[:, 0] += (r % procs_x) * nx * dx
        rows[:, 1] += (r // procs_x) * ny * dx
        out.append(rows)
    return np.concatenate(out) if out else np.zeros((0, 7))
