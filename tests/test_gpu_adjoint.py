"""The GPU adjoint (pic_adjoint) of the slot-stable step, checked against the
FP64 tangent-linear of the oracle step (oracle/tangent.c, itself checked
against central differences in tests/test_adjoint_oracle.py) and against
central differences of the GPU forward (pic_objective).

Objective: the impulse along z delivered to the dipole over NSTEPS steps;
parameters: the coil current I and the drift V. Tolerances: FP64 gradient to
1e-6 relative of the tangent-linear (the GPU forward sums J in 64-bit fixed
point, the oracle in FP64); FP32 gradient to 1e-3."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from plasmasim_b200 import ELECTRON, ION, Pic3D
from tests.util import config_from_oracle_params, oracle_params

pytestmark = pytest.mark.gpu

NSTEPS = 8  # includes the refill of step 5


def gpu_ctx(p, precision, I=None, V=None):
    q = dict(p)
    if I is not None:
        q["I"] = I
    if V is not None:
        q["V"] = V
    P = Pic3D(config_from_oracle_params(q, precision=precision, diag_every_step=0))
    P.init_grid()
    P.init_particle_flat()
    P.fdtd(0)
    return P


def cpu_tangent(p, seed, nsteps=NSTEPS):
    O = Oracle(p)
    O.call("init_grid")
    O.call("init_particle_flat")
    O.call("add_flat")
    return O.tangent_run(nsteps, *seed)


@pytest.fixture(scope="module")
def tangent_tiny():
    p = oracle_params("tiny")
    J, dI = cpu_tangent(p, (1.0, 0.0))
    _, dV = cpu_tangent(p, (0.0, 1.0))
    return J, dI, dV


@pytest.mark.parametrize("every", [NSTEPS, 3, 1])
def test_fp64_adjoint_matches_cpu_tangent_linear(tangent_tiny, every):
    J_ref, dI_ref, dV_ref = tangent_tiny
    with gpu_ctx(oracle_params("tiny"), 64) as P:
        J, dI, dV = P.adjoint(NSTEPS, every)
        assert P.status()[0] == 0
    assert abs(J / J_ref - 1) < 1e-9, (J, J_ref)
    assert abs(dI / dI_ref - 1) < 1e-6, (dI, dI_ref)
    assert abs(dV / dV_ref - 1) < 1e-6, (dV, dV_ref)


def test_fp32_adjoint_within_north_star_tolerance(tangent_tiny):
    J_ref, dI_ref, dV_ref = tangent_tiny
    with gpu_ctx(oracle_params("tiny"), 32) as P:
        J, dI, dV = P.adjoint(NSTEPS, 4)
        assert P.status()[0] == 0
    assert abs(J / J_ref - 1) < 1e-4, (J, J_ref)
    assert abs(dI / dI_ref - 1) < 1e-3, (dI, dI_ref)
    assert abs(dV / dV_ref - 1) < 1e-3, (dV, dV_ref)


def test_adjoint_matches_gpu_central_differences():
    """FP64 GPU forward at I(1 +- h), V(1 +- h), h = 1e-4."""
    p = oracle_params("tiny")
    I0, V0, h = p["I"], p["V"], 1e-4

    def J(I=None, V=None):
        with gpu_ctx(p, 64, I=I, V=V) as P:
            return P.objective(NSTEPS)

    fd_I = (J(I=I0 * (1 + h)) - J(I=I0 * (1 - h))) / (2 * h * I0)
    fd_V = (J(V=V0 * (1 + h)) - J(V=V0 * (1 - h))) / (2 * h * V0)
    with gpu_ctx(p, 64) as P:
        J0, dI, dV = P.adjoint(NSTEPS, 4)
    # the trajectory replays bit for bit; the FP64 sum of the objective is
    # formed with atomics, so its last bit may differ
    assert abs(J0 / J() - 1) < 1e-14
    assert abs(dI / fd_I - 1) < 1e-4, (dI, fd_I)
    assert abs(dV / fd_V - 1) < 1e-4, (dV, fd_V)


def test_adjoint_leaves_the_forward_end_state():
    p = oracle_params("tiny")
    with gpu_ctx(p, 64) as A, gpu_ctx(p, 64) as B:
        A.adjoint(NSTEPS, 3)
        B.objective(NSTEPS)
        for s in (ION, ELECTRON):
            a, b = A.particles(s), B.particles(s)
            assert a.shape == b.shape
            assert np.array_equal(a, b)
        assert np.array_equal(A.grid()[..., :9], B.grid()[..., :9])


def test_adjoint_argument_errors():
    with gpu_ctx(oracle_params("tiny"), 32) as P:
        for bad in [(0, 1), (4, 0)]:
            with pytest.raises(Exception):
                P.adjoint(*bad)


def restore(P, rows, grid, ctr):
    for s in (ION, ELECTRON):
        P.set_particles(s, rows[s])
    P.set_grid(grid)
    P.rng_counters(set_to=ctr)


def test_adjoint_reuses_context_memory():
    """pic_adjoint keeps its snapshot and work memory with the context. A second
    call that starts from an imported state must give what a context that never
    ran an adjoint gives from the same state. That context first runs the same
    number of production steps, so that its refill counter is in the same
    phase as the first context's after its first adjoint."""
    p = oracle_params("tiny")
    with gpu_ctx(p, 64) as P:
        rows = {s: P.particles(s) for s in (ION, ELECTRON)}
        grid, ctr = P.grid(), tuple(P.rng_counters())
        P.adjoint(10, 3)
        restore(P, rows, grid, ctr)
        second = P.adjoint(10, 3)
        assert P.status()[0] == 0
    with gpu_ctx(p, 64) as Q:
        Q.step(10)
        restore(Q, rows, grid, ctr)
        fresh = Q.adjoint(10, 3)
    np.testing.assert_allclose(second, fresh, rtol=1e-10)
