"""The FP64 tangent-linear of the oracle step (oracle/tangent.c), which the GPU
adjoint is checked against, checked itself against central differences of the
oracle's own forward run: the difference must shrink as h^2 (second-order
agreement), to 1e-6 relative at h = 1e-5."""
import pytest

from oracle.pyoracle import Oracle
from tests.util import oracle_params

NSTEPS = 8  # includes the refill of step 5


def _run(p, I, V, tangent=None):
    q = dict(p)
    q["I"], q["V"] = I, V
    O = Oracle(q)
    O.call("init_grid")
    O.call("init_particle_flat")
    O.call("add_flat")
    if tangent is not None:
        return O.tangent_run(NSTEPS, *tangent)
    return O.plain_steps(NSTEPS)


@pytest.mark.parametrize("which", ["I", "V"])
def test_tangent_linear_matches_central_differences(which):
    p = oracle_params("tiny")
    I0, V0 = p["I"], p["V"]
    seed = (1.0, 0.0) if which == "I" else (0.0, 1.0)
    J, dJ = _run(p, I0, V0, tangent=seed)
    assert J == _run(p, I0, V0)  # the dual-number step computes the same values
    errs = []
    for h in (1e-3, 1e-4, 1e-5):
        if which == "I":
            fd = (_run(p, I0 * (1 + h), V0) - _run(p, I0 * (1 - h), V0)) / (2 * h * I0)
        else:
            fd = (_run(p, I0, V0 * (1 + h)) - _run(p, I0, V0 * (1 - h))) / (2 * h * V0)
        errs.append(abs(dJ / fd - 1))
    assert errs[2] < 1e-6, errs
    assert errs[1] < 0.05 * errs[0] and errs[2] < 0.05 * errs[1], errs  # O(h^2)
