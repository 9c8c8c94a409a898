"""The TMA-staged field kernels (renew_b4_2 / renew_e4_2, PIC/3d_pic458_domain.c
:2580-2652) against the per-node kernels on the same random fields.

Both kernels evaluate the same expression for every node, so the staged path
must reproduce the per-node path bit for bit; the per-node path is itself held
to the reference by tests/test_gpu_parity.py. The sizes leave partial tiles on
every axis (nx, ny not multiples of the 4 x 8 tile, nz not a multiple of 32),
and the damped cases put the sigma ramps under part of the tiles.
"""
import numpy as np
import pytest

from plasmasim_b200 import Pic3D, PicConfig

pytestmark = pytest.mark.gpu

# (nx, ny, nz, absorb_grid): nz + 4 is a multiple of 4, so both precisions stage
SIZES = [(8, 8, 8, 0), (18, 21, 76, 0), (37, 13, 28, 5), (64, 64, 124, 16)]


def random_grid(P, seed):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal(P.shape + (18,))
    g[..., 17] = 0.0
    return g


def run(cfg, grid, steps):
    with Pic3D(cfg) as P:
        P.set_grid(grid)
        for _ in range(steps):
            P.renew_b4_2()
            P.renew_e4_2()
            P.renew_b4_2()
        out = P.grid()
        rc, counters = P.status()
        staged = P.staged_fields()
    assert rc == 0 and counters[5] == 0
    return out, staged


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("size", SIZES)
def test_staged_matches_per_node(precision, size):
    nx, ny, nz, absorb = size
    cfg = PicConfig.normalized(nx, ny, nz, 1, precision=precision, absorb_grid=absorb,
                               sigma_a=0.05 if absorb else 1e-6)
    with Pic3D(cfg) as P:
        grid = random_grid(P, seed=nx * 1000 + nz)
    staged, used = run(cfg, grid, steps=3)
    assert used, "the staged kernels were not chosen"
    cfg.plain_fields = 1
    plain, used = run(cfg, grid, steps=3)
    assert not used
    assert np.array_equal(staged, plain), np.max(np.abs(staged - plain))


def test_unaligned_pitch_takes_the_per_node_kernels():
    """FP32 with nz + 4 = 50 values per row (200 bytes): no TMA boxes."""
    with Pic3D(PicConfig.normalized(8, 8, 46, 1, precision=32)) as P:
        assert not P.staged_fields()
    with Pic3D(PicConfig.normalized(8, 8, 46, 1, precision=64)) as P:
        assert P.staged_fields()
