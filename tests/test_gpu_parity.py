"""Parity of the CUDA path with the reference on identical inputs.

The reference side is either a golden fixture written by the reference program
itself (tests/golden) or the FP64 oracle restatement (oracle/pic_oracle.c),
which tests/test_oracle_golden.py pins bit for bit to the reference. Every
call goes through the C ABI (plasmasim_b200.Pic3D over libplasmab200.so).

Tolerances (stated per test): FP64 path to 1e-11..1e-13 relative (summation
order of the atomics and libm ulps differ); FP32 path to 1e-6 relative for the
particle state after one step and to 1e-5 of each field's
maximum for grid quantities.
"""
import numpy as np
import pytest

from plasmasim_b200 import BOTH, ELECTRON, ION, Pic3D
from tests.util import (config_from_oracle_params, field_rel_err, load_golden, make_oracle,
                        oracle_params, rel_norm, sort_rows)

pytestmark = pytest.mark.gpu

PRECISIONS = [64, 32]
PART_TOL = {64: 1e-13, 32: 1e-6}
GRID_TOL = {64: 1e-11, 32: 1e-5}


def new_pic(name="tiny", precision=32, **kw):
    return Pic3D(config_from_oracle_params(oracle_params(name), precision=precision, **kw))


def check_rows(mine, ref, precision, what):
    assert mine.shape == ref.shape, what
    ex = rel_norm(mine[:, :3], ref[:, :3])
    ev = rel_norm(mine[:, 3:6], ref[:, 3:6])
    assert ex <= PART_TOL[precision], (what, "x", ex)
    assert ev <= PART_TOL[precision] * (10 if precision == 64 else 1), (what, "v", ev)
    assert np.all(mine[:, 6] == ref[:, 6])


def check_grid(mine, ref, fields, precision, what, tol=None):
    err = field_rel_err(mine, ref, fields)
    bad = {f: e for f, e in err.items() if e > (tol or GRID_TOL[precision])}
    assert not bad, (what, bad)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_init_matches_reference(precision):
    """init_grid + init_particle_flat against the reference's own output."""
    g = load_golden("init")
    with new_pic(precision=precision) as P:
        P.init_grid()
        P.init_particle_flat()
        grid = P.grid()
        check_grid(grid, g["grid"], range(6), precision, "B/B0", tol=1e-13 if precision == 64 else 1e-7)
        assert np.all(grid[..., 6:17] == 0)
        check_rows(P.particles(ION), g["ion"], precision, "ions")
        check_rows(P.particles(ELECTRON), g["electron"], precision, "electrons")
        assert list(P.rng_counters()) == list(g["rng"])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_step_pieces_match_reference(precision):
    """The reference's step functions one by one (:688-911) from its initial state."""
    g = load_golden("step")
    with new_pic(precision=precision) as P:
        P.init_grid()
        P.init_particle_flat()
        P.renew_grid()
        P.renew_b4_2()
        P.push_deposit_j(BOTH)
        P.renew_b4_2()
        P.drift_deposit_n(BOTH)
        P.reduce_current()
        P.renew_e4_2()
        check_rows(P.particles(ION), g["ion_pre"], precision, "ions")
        check_rows(P.particles(ELECTRON), g["electron_pre"], precision, "electrons")
        check_grid(P.grid(), g["grid"], range(17), precision, "grid")
        P.sr_particle()
        check_rows(sort_rows(P.particles(ION)), sort_rows(g["ion"]), precision, "ions after sr_particle")
        check_rows(sort_rows(P.particles(ELECTRON)), sort_rows(g["electron"]), precision,
                   "electrons after sr_particle")
        assert P.status()[0] == 0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_fused_step_matches_reference(precision):
    """pic_step (tiled sort, then the fused particle kernel) against one
    reference loop body. The reference's initial state holds one particle per
    species in ghost cell x = N+2 (init_particle_flat's extra particle, which
    fdtd's first add_*_flat deletes); pic_step sorts before its first push and
    the sort drops ghost-cell particles as sorting() does, so that particle is
    removed from the input of both sides."""
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    nx = O.p["nx"]
    rows = [O.particles(s)[0] for s in (0, 1)]
    rows = [r[r[:, 0] < nx + 2] for r in rows]
    for s in (0, 1):
        O.set_particles(s, rows[s])
    O.step()
    with new_pic(precision=precision, diag_every_step=0) as P:
        P.init_grid()
        P.set_particles(ION, rows[0])
        P.set_particles(ELECTRON, rows[1])
        P.step(1)
        check_rows(sort_rows(P.particles(ION)), sort_rows(O.particles(0)[0]), precision, "ions")
        check_rows(sort_rows(P.particles(ELECTRON)), sort_rows(O.particles(1)[0]), precision, "electrons")
        check_grid(P.grid(), O.grid(), range(17), precision, "grid")
        F, E = P.thrust_f()
        t = np.concatenate([F, E])
        ref = O.thrust()
        scale = np.maximum(np.abs(ref), 1e-300)
        tol = 1e-10 if precision == 64 else 2e-4
        for q in [0, 1, 2, 3, 4, 5, 9, 10, 11, 27, 28, 29, 30]:
            assert abs(t[q] - ref[q]) <= tol * max(abs(ref[q]), np.abs(ref[:3]).max() if q < 27 else 0), q
        assert P.status()[0] == 0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_add_flat_matches_oracle(precision):
    """add_*_flat: shell deletion and refill draws (same streams as the reference)."""
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    O.call("add_flat")
    with new_pic(precision=precision) as P:
        P.init_grid()
        P.init_particle_flat()
        P.add_flat()
        assert list(P.rng_counters()) == [O.rng_counter(0), O.rng_counter(1)]
        for s in (ION, ELECTRON):
            check_rows(sort_rows(P.particles(s)), sort_rows(O.particles(s)[0]), precision, f"species {s}")


@pytest.mark.parametrize("precision", PRECISIONS)
def test_add_flat_into_tiled_layout_matches_oracle(precision):
    """add_*_flat after a sort, then a second sort: the refill, appended after
    the tiled layout, is moved into the holes the shell deletion left (the
    in-place re-layout) and holds the same particles as the reference's."""
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    O.call("sort")
    O.call("add_flat")
    with new_pic(precision=precision) as P:
        P.init_grid()
        P.init_particle_flat()
        P.sorting()
        P.add_flat()
        P.sorting()
        assert list(P.rng_counters()) == [O.rng_counter(0), O.rng_counter(1)]
        for s in (ION, ELECTRON):
            check_rows(sort_rows(P.particles(s)), sort_rows(O.particles(s)[0]), precision, f"species {s}")


@pytest.mark.parametrize("precision", PRECISIONS)
def test_sort_matches_oracle(precision):
    """sorting: the same particle set in cell order (ghost-cell particles dropped)."""
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    O.call("sort")
    with new_pic(precision=precision) as P:
        P.init_grid()
        P.init_particle_flat()
        P.sorting()
        for s in (ION, ELECTRON):
            mine = P.particles(s)
            ref = O.particles(s)[0]
            assert mine.shape == ref.shape
            # slots are grouped by tile (2 x 4 x 32 interior cells) in tile order
            cells = np.floor(mine[:, :3]).astype(np.int64) - 2
            p = P.cfg
            nty, ntz = -(-p.ny // 4), -(-p.nz // 32)
            tile = ((cells[:, 0] // 2) * nty + cells[:, 1] // 4) * ntz + cells[:, 2] // 32
            assert np.all(np.diff(tile) >= 0)
            check_rows(sort_rows(mine), sort_rows(ref), precision, f"species {s}")


@pytest.mark.parametrize("name", ["damped", "mksa"])
@pytest.mark.parametrize("precision", PRECISIONS)
def test_geometries_one_step(name, precision):
    """Non-cubic grid with damping layers and ballistic particles, and the
    reference's MKSA constants: fdtd's first iteration (refill then a step)."""
    O = make_oracle(name)
    O.call("init_grid")
    O.call("init_particle_flat")
    O.fdtd(1)
    with new_pic(name, precision=precision, diag_every_step=0) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(1)
        for s in (ION, ELECTRON):
            check_rows(sort_rows(P.particles(s)), sort_rows(O.particles(s)[0]), precision, f"{name} {s}")
        check_grid(P.grid(), O.grid(), range(17), precision, name,
                   tol=(1e-10 if precision == 64 else 2e-5))
        assert P.status()[0] == 0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_thrust_and_gauss_match_oracle(precision):
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    O.fdtd(3)
    with new_pic(precision=precision, diag_every_step=0) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(3)
        # compare on the oracle's own state so only the reductions differ
        P.set_grid(O.grid())
        for s in (ION, ELECTRON):
            P.set_particles(s, O.particles(s)[0])
        F, E = P.thrust_f()
        ref = O.thrust()
        tol = 1e-12 if precision == 64 else 1e-5
        fscale = np.abs(ref[:27]).max()
        assert np.abs(F - ref[:27]).max() <= tol * fscale
        assert np.all(np.abs(E - ref[27:]) <= tol * np.abs(ref[27:]) + 1e-300)
        gr = P.gauss_residual()
        go = O.gauss()
        assert gr[3] == go[3]
        assert abs(gr[0] - go[0]) <= (1e-10 if precision == 64 else 1e-4) * go[0]
        assert abs(gr[1] - go[1]) <= (1e-10 if precision == 64 else 1e-5) * go[1]


@pytest.mark.parametrize("precision", PRECISIONS)
def test_twenty_steps_statistics(precision):
    """fdtd over 20 steps with refills every 5 and a sort every 10: field
    energy, densities and thrust against the FP64 oracle. Atomics make the
    deposit order differ, so agreement is statistical (stated tolerances)."""
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    O.fdtd(20, 10, 5)
    with new_pic(precision=precision, diag_every_step=0, sort_interval=10) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(20)
        for s in (ION, ELECTRON):
            n_ref = O.particles(s)[0].shape[0]
            assert abs(P.particle_count(s) - n_ref) <= (2 if precision == 64 else 0.005 * n_ref)
        g1, g2 = P.grid(), O.grid()
        tol = 1e-9 if precision == 64 else 1e-3
        for f in (15, 16):
            assert abs(g1[..., f].sum() / g2[..., f].sum() - 1) < tol
        e1 = (g1[..., 6:9] ** 2).sum()
        e2 = (g2[..., 6:9] ** 2).sum()
        assert abs(e1 / e2 - 1) < (1e-8 if precision == 64 else 2e-2)
        F, E = P.thrust_f()
        ref = O.thrust()
        assert abs(E[2] / ref[29] - 1) < tol
        assert abs(E[3] / ref[30] - 1) < tol


def test_fp32_within_thrust_tolerance_of_fp64():
    """FP32 step against the FP64 step from the same seed: thrust and energies
    within 1e-3 relative after 20 steps (the precision bar of the FP32 path)."""
    res = {}
    for precision in (64, 32):
        with new_pic("tiny", precision=precision, diag_every_step=0) as P:
            P.init_grid()
            P.init_particle_flat()
            P.fdtd(20)
            F, E = P.thrust_f()
            res[precision] = (F, E)
    F64, E64 = res[64]
    F32, E32 = res[32]
    for q in (2, 3):
        assert abs(E32[q] / E64[q] - 1) < 1e-3
    assert abs(E32[1] / E64[1] - 1) < 1e-3


@pytest.mark.parametrize("precision", PRECISIONS)
def test_edge_cases(precision):
    """Empty species, particles on cell faces and box edges, the ghost-cell
    deposit that would leave the array, capacity and argument errors."""
    with new_pic(precision=precision, diag_every_step=0, capacity=65536) as P:
        P.init_grid()
        P.set_particles(ION, np.zeros((0, 7)))
        P.set_particles(ELECTRON, np.zeros((0, 7)))
        P.step(2)
        assert P.particle_count(ION) == 0
        w = 0.01 / 4
        rows = np.array([
            [2.0, 2.0, 2.0, 0.0, 0.0, 0.05, w],      # on the lower interior faces
            [9.999999, 5.5, 5.5, 0.01, 0.0, 0.0, w],  # just below (N+2) dx in x
            [5.5, 5.5, 9.9999, 0.0, 0.0, 0.1, w],     # leaves through z
            [5.5, 5.5, 5.5, 0.0, 0.0, 0.0, w],        # at rest in the centre
            [11.5, 5.5, 5.5, 0.0, 0.0, 0.0, w],       # last ghost cell: stencil leaves the array
        ])
        P.set_particles(ION, rows)
        P.push_deposit_j(ION)
        rc, counters = P.status()
        assert rc == 5 and counters[0] >= 1   # the out-of-array deposit was counted
        O = make_oracle("tiny")
        O.call("init_grid")
        O.set_particles(0, np.zeros((0, 7)))
        O.set_particles(1, np.zeros((0, 7)))
        O.step()
        O.step()
        O.set_particles(0, rows)
        O.call("renew_grid")
        O.call("push_j")
        check_rows(P.particles(ION), O.particles(0)[0], precision, "edge push")
        with pytest.raises(Exception):
            P.set_particles(ION, np.zeros((65537, 7)) + w)  # over capacity
        bad = rows.copy()
        bad[0, 6] = 2 * w
        with pytest.raises(Exception):
            P.set_particles(ION, bad)                        # weight is per species
