"""Poisson cleaning (renew_phi3 + sr_phi + sr_e) through the C ABI.

Three references:
- the compiled reference itself, built with its PHI blocks (oracle/_ref
  libref3d_tiny_phi*.so), on its own state;
- the numpy restatement oracle.pyoracle.renew_phi3, which
  tests/test_poisson_oracle.py pins to the compiled reference, on random
  fields of a non-cubic grid;
- the oracle's loop body followed by the restatement, against pic_step with
  poisson_clean = 1.

Tolerances: FP64 1e-12 of each field's maximum (the transforms sum in another
order than the reference's FFT); FP32 2e-6 of each field's maximum for E (E
itself is stored in FP32) and 1e-5 for phi, whose transforms run in FP32.
"""
import os

import numpy as np
import pytest

from oracle import build as obuild
from oracle.pyoracle import Reference, renew_phi3
from plasmasim_b200 import ELECTRON, ION, Pic3D
from tests.util import (config_from_oracle_params, field_rel_err, make_oracle, oracle_params,
                        random_fields, rel_norm, sort_rows)

pytestmark = pytest.mark.gpu

EX, EY, EZ, PHI = 6, 7, 8, 17
TOL = {64: {EX: 1e-12, EY: 1e-12, EZ: 1e-12, PHI: 1e-12},
       32: {EX: 2e-6, EY: 2e-6, EZ: 2e-6, PHI: 1e-5}}


def check(mine, ref, precision, what):
    err = field_rel_err(mine, ref, (EX, EY, EZ, PHI))
    bad = {f: e for f, e in err.items() if e > TOL[precision][f]}
    assert not bad, (what, bad)
    others = [f for f in range(17) if f not in (EX, EY, EZ)]
    scale = max(np.abs(ref[..., others]).max(), 1e-300)
    lim = 1e-15 if precision == 64 else 1e-7
    assert np.abs(mine[..., others] - ref[..., others]).max() <= lim * scale, what


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("name", ["tiny_phi", "tiny_phi1"])
def test_matches_compiled_reference(name, precision):
    if not os.path.isfile(obuild.ref_lib_path(name)):
        pytest.skip("the compiled reference (oracle/_ref) is not built")
    R = Reference(name)
    R.init_grid()
    R.init_particle_flat()
    R.L.ref_loop(4, 500, 5)
    before = R.grid()
    R.renew_phi3()
    after = R.grid()
    a3 = int(R.defines["ORACLE_ABSORB3"])
    cfg = config_from_oracle_params(R.params, precision=precision, absorb_grid3=a3)
    with Pic3D(cfg) as P:
        P.set_grid(before)
        P.poisson_clean()
        check(P.grid(), after, precision, name)
        assert P.status()[0] == 0


@pytest.mark.parametrize("precision", [64, 32])
def test_matches_restatement_on_random_fields(precision):
    """A non-cubic grid (8 x 16 x 32) with smooth random E and densities."""
    p = dict(oracle_params("tiny"), nx=8, ny=16, nz=32)
    rng = np.random.default_rng(7)
    shape = (p["nx"] + 4, p["ny"] + 4, p["nz"] + 4)
    g = np.zeros(shape + (18,))
    (ex, ey, ez), _ = random_fields(shape, rng)
    g[..., EX], g[..., EY], g[..., EZ] = ex, ey, ez
    g[..., 15] = 0.01 * (1 + 0.2 * rng.random(shape))
    g[..., 16] = 0.01 * (1 + 0.2 * rng.random(shape))
    g[..., PHI] = rng.random(shape)  # only the z ghosts survive the cleaning
    if precision == 32:
        g = g.astype(np.float32).astype(np.float64)
    ref = renew_phi3(g, p["dx"], p["q"], p["e0"], 2)
    with Pic3D(config_from_oracle_params(p, precision=precision, absorb_grid3=2)) as P:
        P.set_grid(g)
        P.poisson_clean()
        check(P.grid(), ref, precision, "random")


@pytest.mark.parametrize("precision", [64, 32])
def test_step_with_cleaning(precision):
    """pic_step with poisson_clean = 1 = the oracle's loop body followed by
    renew_phi3 (the PHI block after renew_e4_2 / sr_e, :901-907); the cleaning
    changes E and phi only, so the particles match the plain step."""
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    nx = O.p["nx"]
    rows = [O.particles(s)[0] for s in (0, 1)]
    rows = [r[r[:, 0] < nx + 2] for r in rows]
    for s in (0, 1):
        O.set_particles(s, rows[s])
    O.step()
    ref = renew_phi3(O.grid(), O.p["dx"], O.p["q"], O.p["e0"], 0)
    cfg = config_from_oracle_params(oracle_params("tiny"), precision=precision, diag_every_step=0,
                                    poisson_clean=1, absorb_grid3=0)
    with Pic3D(cfg) as P:
        P.init_grid()
        P.set_particles(ION, rows[0])
        P.set_particles(ELECTRON, rows[1])
        P.step(1)
        tol = 1e-13 if precision == 64 else 1e-6
        for s in (ION, ELECTRON):
            assert rel_norm(sort_rows(P.particles(s))[:, :6], sort_rows(O.particles(s)[0])[:, :6]) <= tol
        mine = P.grid()
        err = field_rel_err(mine, ref, (EX, EY, EZ, PHI))
        lim = {64: 1e-11, 32: 2e-5}[precision]
        assert all(e <= lim for e in err.values()), err
        assert P.status()[0] == 0


def test_cleaning_reduces_gauss_residual():
    """The correction halves the Gauss-law residual of a reference state
    (renew_phi3's spectral Laplacian is not the inverse of the 4th-order
    div-grad pair, and the first line of every axis stays out, so it does not
    remove it)."""
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    for _ in range(6):
        O.step()
    with Pic3D(config_from_oracle_params(oracle_params("tiny"), precision=64, absorb_grid3=0)) as P:
        P.set_grid(O.grid())
        before = P.gauss_residual()
        P.poisson_clean()
        after = P.gauss_residual()
        assert after[0] < 0.6 * before[0], (before, after)
