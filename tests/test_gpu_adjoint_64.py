"""The adjoint (pic_adjoint) at the differentiable run's geometry: 64^3 cells x
16 particles per cell per species, FP32, against central differences of the
GPU forward (pic_objective, relative step 1e-3) for the three drifts the run
sweeps, V = 0.05, 0.1 and 0.2 c.

The adjoint is exact for the discrete trajectory it differentiates, but that
trajectory is chaotic: the pathwise derivative and the finite difference part
ways as the horizon grows, the sooner the faster the drift (measured on a
B200 at h = 1e-3: within 1e-3 up to 15 steps at 0.05 c, 12 at 0.1 c, 5 at
0.2 c; at 20 steps 1.1e-3, 1.1e-2 and 7.5e-2 for dJ/dI). Each drift is checked
at a horizon inside its range, with a checkpoint every 5 steps so that the
reverse pass recomputes segments; a second test checks that the checkpoint
interval does not change the gradient. Tolerance: 1e-3 relative, the bar of
the north star."""
import pytest

from plasmasim_b200 import Pic3D, PicConfig

pytestmark = pytest.mark.gpu

H = 1e-3
HORIZON = {0.05: 10, 0.1: 10, 0.2: 5}


def ctx(I=32.0, V=0.1):
    cfg = PicConfig.normalized(64, 64, 64, 16, precision=32, diag_every_step=0, sort_interval=20, add_interval=5)
    cfg.coil_i, cfg.v_drift = I, V
    P = Pic3D(cfg)
    P.init_grid()
    P.init_particle_flat()
    P.fdtd(0)
    return P


@pytest.mark.parametrize("V", sorted(HORIZON))
def test_adjoint_against_central_differences(V, record):
    T = HORIZON[V]
    with ctx(V=V) as P:
        J, dI, dV = P.adjoint(T, 5)
        assert P.status()[0] == 0
    vals = []
    for I, v in ((32 * (1 + H), V), (32 * (1 - H), V), (32, V * (1 + H)), (32, V * (1 - H))):
        with ctx(I, v) as P:
            vals.append(P.objective(T))
    fdI = (vals[0] - vals[1]) / (2 * H * 32)
    fdV = (vals[2] - vals[3]) / (2 * H * V)
    errs = dict(V=V, steps=T, dI=dI, fdI=fdI, dV=dV, fdV=fdV, eI=abs(dI / fdI - 1), eV=abs(dV / fdV - 1))
    record.update(errs)
    assert errs["eI"] <= 1e-3, errs
    assert errs["eV"] <= 1e-3, errs


def test_checkpoint_interval_leaves_gradient_unchanged(record):
    """10 steps reversed from checkpoints every 5 steps and from one
    checkpoint: the recomputed segments replay the forward bit for bit in its
    fixed-point currents, so the gradients agree to rounding of the reverse
    sums (measured 1e-8)."""
    res = []
    for every in (5, 10):
        with ctx() as P:
            res.append(P.adjoint(10, every))
    J5, I5, V5 = res[0]
    J10, I10, V10 = res[1]
    record.update(J=[J5, J10], dI=[I5, I10], dV=[V5, V10])
    assert abs(J5 / J10 - 1) <= 1e-12
    assert abs(I5 / I10 - 1) <= 1e-6
    assert abs(V5 / V10 - 1) <= 1e-6
