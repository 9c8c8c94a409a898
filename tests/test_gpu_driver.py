"""The C host driver (plasmasim_b200/driver/pic3d_main.c), the reference's
main/fdtd loop written against the C ABI, run as its own process: 32^3 cells
x 8 particles per cell per species, 5 steps, FP64, a thrust line after every
step. Its printed thrust lines and the files it writes (thrust458.txt, and
thrust458_ave.txt at step 0, a multiple of 500) are checked against the same
run made through the Python binding: F to the printed three decimals
(4 significant digits), E to the printed eight."""
import os
import subprocess

import numpy as np
import pytest

from plasmasim_b200 import Pic3D, PicConfig
from plasmasim_b200 import build as pbuild

pytestmark = pytest.mark.gpu


def test_c_driver_runs_the_loop(tmp_path):
    exe = pbuild.DRIVER
    if not os.path.isfile(exe):
        pbuild.build_driver()
    steps = 5
    res = subprocess.run([exe, "32", "32", "32", "8", str(steps), "64", "20", "1", str(tmp_path)],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    lines = [l.split() for l in res.stdout.splitlines() if l.strip()]
    assert [int(l[0]) for l in lines] == list(range(steps))
    assert all(len(l) == 34 for l in lines)
    printed = np.array([[float(x) for x in l[1:]] for l in lines])

    cfg = PicConfig.normalized(32, 32, 32, 8, precision=64, sort_interval=20, diag_every_step=1)
    ours = []
    with Pic3D(cfg) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(0)
        for _ in range(steps):
            P.step(1)
            F, E = P.thrust_f()
            ours.append(np.concatenate([F, E]))
    ours = np.array(ours)
    for c in range(steps):
        F, Fp = ours[c, :27], printed[c, :27]
        scale = np.abs(F).max()
        assert np.all(np.abs(Fp - F) <= 5e-4 * np.abs(F) + 1e-12 * scale), c
        E, Ep = ours[c, 27:], printed[c, 27:]
        assert np.all(np.abs(Ep - E) <= 1e-8 * np.abs(E) + 1e-300), c

    thrust = (tmp_path / "thrust458.txt").read_text().splitlines()
    assert [int(l.split()[0]) for l in thrust] == list(range(steps))
    ave = (tmp_path / "thrust458_ave.txt").read_text().splitlines()
    assert len(ave) == 1 and ave[0].split()[0] == "0" and len(ave[0].split()) == 28
    assert "steps 5" in res.stderr and not np.isnan(printed).any()
