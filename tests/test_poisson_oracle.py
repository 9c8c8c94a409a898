"""The numpy restatement of renew_phi3 + sr_phi + sr_e
(oracle.pyoracle.renew_phi3) against the reference compiled with its PHI
blocks, on the reference's own state after a few loop bodies."""
import os

import numpy as np
import pytest

from oracle import build as obuild
from oracle.pyoracle import Reference, renew_phi3, sine_matrix


@pytest.mark.parametrize("name", ["tiny_phi", "tiny_phi1"])
def test_restatement_matches_compiled_reference(name):
    if not obuild.reference_available() and not os.path.isfile(obuild.ref_lib_path(name)):
        pytest.skip("reference source not available")
    obuild.build_ref(name)
    R = Reference(name)
    R.init_grid()
    R.init_particle_flat()
    R.L.ref_loop(4, 500, 5)
    before = R.grid()
    R.renew_phi3()
    after = R.grid()
    p = R.params
    mine = renew_phi3(before, p["dx"], p["q"], p["e0"], int(R.defines["ORACLE_ABSORB3"]))
    for f in (6, 7, 8, 17):
        scale = np.abs(after[..., f]).max()
        assert np.abs(mine[..., f] - after[..., f]).max() <= 1e-14 * scale, f
    assert np.abs(after[..., 17]).max() > 0  # the cleaning did something
    others = [f for f in range(18) if f not in (6, 7, 8, 17)]
    assert np.array_equal(mine[..., others], after[..., others])


def test_sine_matrix_is_sinft():
    """S applied to a vector = the reference's sinft on data[1..n] with data[1]
    dropped, checked against the direct sum of its definition."""
    n = 16
    rng = np.random.default_rng(3)
    y = rng.standard_normal(n)
    S = sine_matrix(n)
    want = np.array([sum(y[j] * np.sin(np.pi * j * k / n) for j in range(1, n)) for k in range(n)])
    assert np.allclose(S @ y, want, rtol=0, atol=1e-13)
    assert np.allclose(S @ S, n / 2 * np.diag([0] + [1] * (n - 1)), atol=1e-12)
