"""The allocation-free Gauss-law residual (pic_gauss_residual_noalloc).

It serves callers that may not allocate device memory themselves, such as a
plugin inside a host application that owns every device allocation: the
caller hands in its own device buffers, and the entry point's only scratch is
a fixed-size device array built into the library. Here it is called through
the C ABI on FP32 planes held in caller-owned torch tensors, twice in a row
(the second call runs on the scratch the first one left behind), and its
result is checked against pic_gauss_residual on the same state, to 1e-9
relative (both reduce in FP64, in a different order).
"""
import ctypes as C

import numpy as np
import pytest

from plasmasim_b200 import Pic3D
from plasmasim_b200.pic3d import load_library
from tests.util import config_from_oracle_params, oracle_params

pytestmark = pytest.mark.gpu

EX, EY, EZ, NI, NE = 6, 7, 8, 15, 16


def test_noalloc_residual_matches_context_residual():
    import torch

    p = oracle_params("tiny")
    cfg = config_from_oracle_params(p, precision=32, diag_every_step=0)
    with Pic3D(cfg) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(4)
        ref = P.gauss_residual()
        grid = P.grid()
    assert ref[3] == p["nx"] * p["ny"] * p["nz"] and ref[1] > 0

    dev = torch.device("cuda", 0)
    planes = {f: torch.tensor(np.ascontiguousarray(grid[..., f]), dtype=torch.float32, device=dev)
              for f in (EX, EY, EZ, NI, NE)}
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    L = load_library()
    stream = torch.cuda.current_stream(dev).cuda_stream
    results = []
    for _ in range(2):
        out.fill_(-1.0)
        rc = L.pic_gauss_residual_noalloc(
            planes[EX].data_ptr(), planes[EY].data_ptr(), planes[EZ].data_ptr(),
            planes[NI].data_ptr(), planes[NE].data_ptr(), p["nx"], p["ny"], p["nz"],
            p["dx"], p["q"], p["e0"], stream, out.data_ptr())
        assert rc == 0
        torch.cuda.synchronize(dev)
        results.append(out.cpu().numpy().copy())
    for got in results:
        assert got[3] == ref[3]
        for q in (0, 1, 2):
            assert abs(got[q] - ref[q]) <= 1e-9 * abs(ref[q]), (q, got[q], ref[q])
    assert np.array_equal(results[0], results[1])


def test_noalloc_rejects_inputs_beyond_its_scratch():
    import torch

    L = load_library()
    t = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    ptr = t.data_ptr()
    # 400^3 cells exceed the 2048 x 256 x 64 cells the static scratch covers;
    # the size check comes before any launch
    rc = L.pic_gauss_residual_noalloc(ptr, ptr, ptr, ptr, ptr, 400, 400, 400, 1.0, 1.0, 1.0,
                                      None, out.data_ptr())
    assert rc == 6
    assert L.pic_error_string(rc) == b"input larger than the fixed-size scratch allows"
