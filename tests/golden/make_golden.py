"""Generates the golden fixtures in tests/golden/ by running the reference
program PIC/3d_pic458_domain.c itself, compiled by oracle/build.py into
oracle/_ref/libref3d_tiny.so (8x8x8 cells, 4 particles/cell/species, normalized
units). Needs the reference checkout; run from the repository root:

    python tests/golden/make_golden.py

Each scenario runs in a fresh process (the reference keeps its state in
process globals) inside a temporary working directory (fdtd writes files).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# grid fields kept in the fixtures: B, B0, E, J_i, J_e, n_i, n_e (phi is unused)
KEEP = list(range(17))


def _init(name):
    from oracle.pyoracle import Reference
    R = Reference(name)
    R.init_grid()
    R.init_particle_flat()
    return R


def scenario_init(name, q):
    R = _init(name)
    ion, fi = R.particles(0)
    el, fe = R.particles(1)
    q.put(dict(grid=R.grid()[..., KEEP], ion=ion, electron=el,
               rng=np.array([R.rng_counter(0), R.rng_counter(1)], dtype=np.int64)))


def scenario_step(name, q):
    """One loop body of fdtd (:688-911 without output) from the initial state."""
    R = _init(name)
    n0 = (R.particles(0)[0].shape[0], R.particles(1)[0].shape[0])
    for op in ["renew_grid", "renew_b", "sr_b", "push_j", "renew_b", "sr_b", "drift_n",
               "reduce", "sr_current", "renew_e", "sr_e"]:
        R.op(op)
    grid_pre = R.grid()[..., KEEP]
    pre_ion, _ = R.particles(0)
    pre_el, _ = R.particles(1)
    R.op("sr_particle")
    ion, _ = R.particles(0)
    el, _ = R.particles(1)
    q.put(dict(grid=grid_pre, ion_pre=pre_ion, electron_pre=pre_el, ion=ion, electron=el,
               thrust=R.thrust(include_tail=True), n0=np.array(n0)))


def scenario_add(name, q):
    """add_ion_flat + add_electron_flat from the initial state."""
    R = _init(name)
    R.op("add_flat")
    after = [R.particles(s)[0] for s in (0, 1)]
    q.put(dict(ion_after=after[0], electron_after=after[1],
               rng=np.array([R.rng_counter(0), R.rng_counter(1)], dtype=np.int64)))


def scenario_fdtd(name, q):
    """fdtd for 10 steps from the initial state (add_flat at 0 and 5)."""
    R = _init(name)
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        R.fdtd(10)
    q.put(dict(grid=R.grid()[..., KEEP], thrust=R.thrust(include_tail=True), fave=R.fave(),
               counts=np.array([R.particles(0)[0].shape[0], R.particles(1)[0].shape[0]])))


def run(fn, name):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=fn, args=(name, q))
    p.start()
    res = q.get()
    p.join()
    return res


def main():
    name = "tiny"
    for tag, fn in [("init", scenario_init), ("step", scenario_step), ("add", scenario_add),
                    ("fdtd10", scenario_fdtd)]:
        res = run(fn, name)
        path = os.path.join(OUT, f"ref_{name}_{tag}.npz")
        np.savez_compressed(path, **res)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
