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
