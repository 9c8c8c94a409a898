"""The allocation-free Gauss-law residual (pic_gauss_residual_noalloc).

It serves callers that may not allocate device memory themselves, such as a
plugin inside a host application that owns every device allocation: the
caller hands in its own device buffers, and the entry point's only scratch is
a fixed-size device array built into the library. Here it is called through
the C ABI on FP32 planes held in caller-owned torch tensors, twice in a row
(the second call runs on the scratch the first one left behind), and its
result is checked against pic_gauss_residual on the same state, to 1e-9
relative (both reduce in FP64, in a different order).

The cases: a grid of one reduction block (8^3 cells), a grid of several
blocks with sides that are not multiples of anything (64 x 40 x 33 = 84,480
cells, six blocks of 16,384 cells), the largest input the scratch covers
(33,554,432 cells, accepted) and one cell more (rejected before any launch).
"""
import math

import numpy as np
import pytest

from plasmasim_b200 import Pic3D, PicConfig
from plasmasim_b200.pic3d import load_library
from tests.util import config_from_oracle_params, oracle_params

pytestmark = pytest.mark.gpu

EX, EY, EZ, NI, NE = 6, 7, 8, 15, 16
MAX_CELLS = 2048 * 256 * 64  # blocks x threads x cells per thread of the static scratch
PIC_ERR_ARG, PIC_ERR_TOO_LARGE = 1, 6


def _call(L, planes, nx, ny, nz, dx, q, e0, out, stream):
    return L.pic_gauss_residual_noalloc(
        planes[EX].data_ptr(), planes[EY].data_ptr(), planes[EZ].data_ptr(),
        planes[NI].data_ptr(), planes[NE].data_ptr(), nx, ny, nz, dx, q, e0, stream, out.data_ptr())


def _check_against_context(cfg: PicConfig, steps: int):
    import torch

    with Pic3D(cfg) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(steps)
        ref = P.gauss_residual()
        grid = P.grid()
    assert ref[3] == cfg.nx * cfg.ny * cfg.nz and ref[1] > 0

    dev = torch.device("cuda", 0)
    planes = {f: torch.tensor(np.ascontiguousarray(grid[..., f]), dtype=torch.float32, device=dev)
              for f in (EX, EY, EZ, NI, NE)}
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    L = load_library()
    stream = torch.cuda.current_stream(dev).cuda_stream
    results = []
    for _ in range(2):
        out.fill_(-1.0)
        assert _call(L, planes, cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.q, cfg.e0, out, stream) == 0
        torch.cuda.synchronize(dev)
        results.append(out.cpu().numpy().copy())
    for got in results:
        assert got[3] == ref[3]
        for q in (0, 1, 2):
            assert abs(got[q] - ref[q]) <= 1e-9 * abs(ref[q]), (q, got[q], ref[q])
    assert np.array_equal(results[0], results[1])


def test_noalloc_residual_matches_context_residual():
    """8^3 cells: one block of the reduction."""
    cfg = config_from_oracle_params(oracle_params("tiny"), precision=32, diag_every_step=0)
    _check_against_context(cfg, 4)


def test_noalloc_residual_several_blocks():
    """64 x 40 x 33 cells: six blocks, so the grid-stride partials and the final
    sum over several partial slots both run."""
    cfg = PicConfig.normalized(64, 40, 33, 2, precision=32, diag_every_step=0)
    _check_against_context(cfg, 3)


def test_noalloc_accepts_the_largest_input():
    """256 x 256 x 512 cells, exactly the scratch's maximum, on zero planes:
    accepted, every cell counted, residual zero."""
    import torch

    L = load_library()
    nx, ny, nz = 256, 256, 512
    assert nx * ny * nz == MAX_CELLS
    zero = torch.zeros((nx + 4) * (ny + 4) * (nz + 4), dtype=torch.float32, device="cuda")
    planes = {f: zero for f in (EX, EY, EZ, NI, NE)}
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    for _ in range(2):
        assert _call(L, planes, nx, ny, nz, 1.0, 1.0, 1.0, out, None) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[3] == MAX_CELLS and got[0] == 0.0 and got[1] == 0.0 and got[2] == 0.0


def test_noalloc_rejects_inputs_beyond_its_scratch():
    """One cell over the maximum (and a far larger grid) return
    PIC_ERR_TOO_LARGE before any launch; non-finite constants PIC_ERR_ARG.
    The output is left as it was."""
    import torch

    L = load_library()
    t = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    planes = {f: t for f in (EX, EY, EZ, NI, NE)}
    # the planes are far too small for these shapes: only the size check,
    # which comes before any launch, keeps the kernels from reading them
    assert _call(L, planes, MAX_CELLS + 1, 1, 1, 1.0, 1.0, 1.0, out, None) == PIC_ERR_TOO_LARGE
    assert _call(L, planes, 400, 400, 400, 1.0, 1.0, 1.0, out, None) == PIC_ERR_TOO_LARGE
    for dx, q, e0 in ((math.inf, 1.0, 1.0), (1.0, math.nan, 1.0), (1.0, 1.0, math.nan), (0.0, 1.0, 1.0)):
        assert _call(L, planes, 2, 2, 2, dx, q, e0, out, None) == PIC_ERR_ARG
    torch.cuda.synchronize()
    assert np.all(out.cpu().numpy() == -1.0)
    assert L.pic_error_string(PIC_ERR_TOO_LARGE) == b"input larger than the fixed-size scratch allows"
