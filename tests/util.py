"""Shared helpers of the test suite: configurations in both the product's form
(PicConfig) and the oracle's form, seeded states, and comparison metrics."""
from __future__ import annotations

import math
import os

import numpy as np

from oracle import build as obuild
from oracle.pyoracle import Oracle, params_from_defines
from plasmasim_b200.pic3d import PicConfig

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# grid record fields
BX, BY, BZ, B0X, B0Y, B0Z, EX, EY, EZ, JIX, JIY, JIZ, JEX, JEY, JEZ, NI, NE, PHI = range(18)


def config_from_oracle_params(p: dict, precision: int = 32, **kw) -> PicConfig:
    cfg = PicConfig(nx=p["nx"], ny=p["ny"], nz=p["nz"], np=p["np"], precision=precision,
                    dx=p["dx"], dt=p["dt"], q=p["q"], mi=p["mi"], me=p["me"], mu0=p["mu0"],
                    e0=p["e0"], kb=p["kb"], c=p["c"], v_drift=p["V"], n_all=p["Nall"],
                    ti=p["Ti"], te=p["Te"], coil_r=p["R"], coil_i=p["I"], alpha=p["alpha"],
                    imf_x=p["imf_x"], imf_y=p["imf_y"], imf_z=p["imf_z"],
                    absorb_grid=p["absorb"], absorb_grid2=p["absorb2"],
                    sigma_a=p["sigma_a"], dipole_cutoff=p["cutoff"])
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def oracle_params(name: str) -> dict:
    return params_from_defines(obuild.REF_CONFIGS[name])


def make_oracle(name: str) -> Oracle:
    return Oracle(oracle_params(name))


def load_golden(tag: str, name: str = "tiny"):
    return dict(np.load(os.path.join(GOLDEN, f"ref_{name}_{tag}.npz")))


def rel_norm(a, b) -> float:
    """||a - b|| / ||b|| over all entries (0 when both vanish)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    if den == 0.0:
        return float(num)
    return float(num / den)


def field_rel_err(g1, g2, fields) -> dict:
    """Per-field max |difference| relative to the field's max magnitude."""
    out = {}
    for f in fields:
        scale = max(np.abs(g2[..., f]).max(), 1e-300)
        out[f] = float(np.abs(g1[..., f] - g2[..., f]).max() / scale)
    return out


def sort_rows(rows: np.ndarray) -> np.ndarray:
    """Particle rows in a canonical order (lexicographic on x, y, z, vx)."""
    if rows.shape[0] == 0:
        return rows
    idx = np.lexsort((rows[:, 3], rows[:, 2], rows[:, 1], rows[:, 0]))
    return rows[idx]


def random_fields(shape, rng, scale_e=1e-2, scale_b=0.1, smooth=True):
    """Smooth random E and induced-B perturbations (added to B0 by the caller)."""
    gx, gy, gz = shape
    x = np.arange(gx)[:, None, None]
    y = np.arange(gy)[None, :, None]
    z = np.arange(gz)[None, None, :]
    out = []
    for _ in range(6):
        kx, ky, kz = rng.uniform(0.2, 0.9, size=3)
        ph = rng.uniform(0, 2 * math.pi, size=3)
        f = np.sin(kx * x + ph[0]) * np.cos(ky * y + ph[1]) * np.sin(kz * z + ph[2])
        f = f + 0.1 * rng.standard_normal(shape) if not smooth else f
        out.append(f)
    e = [scale_e * f for f in out[:3]]
    b = [scale_b * f for f in out[3:]]
    return e, b


def match_rows(mine: np.ndarray, ref: np.ndarray):
    """Pairs each row of `mine` with the row of `ref` nearest in position.

    Rows of the two sides come in different orders (the GPU keeps particles in
    its tiled cell order). One step moves a particle about 0.025 cells and the
    FP32 path places it within a few 1e-7 cells of the FP64 oracle, while
    neighbouring particles lie tenths of a cell apart, so the nearest position
    identifies the particle. Returns (mine, ref[idx]) after checking that the
    pairing is one to one."""
    from scipy.spatial import cKDTree

    assert mine.shape == ref.shape, (mine.shape, ref.shape)
    if mine.shape[0] == 0:
        return mine, ref
    tree = cKDTree(ref[:, :3])
    dist, idx = tree.query(mine[:, :3], k=1)
    assert np.bincount(idx, minlength=ref.shape[0]).max() == 1, "position matching is not one to one"
    return mine, ref[idx]


def step_errors(mine: np.ndarray, ref: np.ndarray, dt: float, dx: float) -> dict:
    """Per-particle errors of one step, rows already paired (match_rows).

    disp: ||x_mine - x_ref|| / ||v_ref dt|| over all particles, i.e. the error
          of the displacement relative to the displacement (a step moves each
          particle by v^{n+1/2} dt, so x_mine - x_ref is the displacement error)
    vel:  ||v_mine - v_ref|| / ||v_ref||
    max_dx_cells: the largest position difference of one particle, in cells
    max_dv_rel:   the largest |v_mine - v_ref| / |v_ref| of one particle"""
    dxv = mine[:, :3] - ref[:, :3]
    dvv = mine[:, 3:6] - ref[:, 3:6]
    vref = ref[:, 3:6]
    vn = np.linalg.norm(vref, axis=1)
    return dict(
        disp=float(np.linalg.norm(dxv) / max(np.linalg.norm(vref) * dt, 1e-300)),
        vel=float(np.linalg.norm(dvv) / max(np.linalg.norm(vref), 1e-300)),
        max_dx_cells=float(np.abs(dxv).max() / dx) if len(dxv) else 0.0,
        max_dv_rel=float((np.linalg.norm(dvv, axis=1) / np.maximum(vn, 1e-300)).max()) if len(dvv) else 0.0,
    )


def oracle_params_for(nx: int, ny: int, nz: int, np_: int, base: str = "tiny") -> dict:
    """Run-time oracle parameters of the normalized plasma on an nx x ny x nz
    grid with np_ particles per cell per species (the restatement takes its
    geometry at run time; no compiled reference is needed)."""
    p = dict(oracle_params(base))
    p.update(nx=nx, ny=ny, nz=nz, np=np_)
    return p


def density_moments(grid: np.ndarray) -> np.ndarray:
    """Sum n and the first moments sum n x, n y, n z of both species' density
    planes (node indices as coordinates): 8 numbers."""
    gx, gy, gz = grid.shape[:3]
    ax = [np.arange(gx, dtype=np.float64), np.arange(gy, dtype=np.float64), np.arange(gz, dtype=np.float64)]
    out = []
    for f in (NI, NE):
        n = grid[..., f]
        out.append(n.sum())
        out.append((n.sum(axis=(1, 2)) * ax[0]).sum())
        out.append((n.sum(axis=(0, 2)) * ax[1]).sum())
        out.append((n.sum(axis=(0, 1)) * ax[2]).sum())
    return np.array(out)
