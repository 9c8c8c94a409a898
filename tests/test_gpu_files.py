"""The reference's files through the C ABI (pic_save_checkpoint,
pic_load_checkpoint, pic_write_output, pic_append_thrust,
pic_append_thrust_ave), checked against the reference compiled from its own
source (oracle/_ref, suspend_job / continue_job / output run by the harness)
and, for the thrust lines, against the oracle's sums in the reference's
printf formats."""
import os

import numpy as np
import pytest

from oracle import build as obuild
from oracle.pyoracle import Reference
from plasmasim_b200 import ELECTRON, ION, Pic3D
from tests.util import config_from_oracle_params, make_oracle, oracle_params, sort_rows

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not os.path.isfile(obuild.ref_lib_path("tiny")),
                       reason="the compiled reference (oracle/_ref) is not built"),
]


def gpu_ctx(precision=64, **kw):
    return Pic3D(config_from_oracle_params(oracle_params("tiny"), precision=precision, **kw))


def reference_state(nsteps=3):
    R = Reference("tiny")
    R.init_grid()
    R.init_particle_flat()
    R.L.ref_loop(nsteps, 500, 5)
    return R


def test_reference_checkpoint_loads(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    R = reference_state()
    R.suspend()
    assert os.path.isfile("suspend-0-field.dat") and os.path.isfile("suspend-0-0-ion.dat")
    with gpu_ctx() as P:
        P.load_checkpoint(str(tmp_path))
        for s in (ION, ELECTRON):
            a, b = sort_rows(P.particles(s)), sort_rows(R.particles(s)[0])
            assert a.shape == b.shape
            assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
        g, rg = P.grid(), R.grid()
        assert np.abs(g[..., :17] - rg[..., :17]).max() <= 1e-15 * np.abs(rg).max()
        assert list(P.rng_counters()) == [0, 0]  # continue_job restarts the streams


def test_engine_checkpoint_continues_in_reference(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    with gpu_ctx(diag_every_step=0) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(3)
        P.save_checkpoint(str(tmp_path))
        R = Reference("tiny")
        R.continue_job()
        for s in (ION, ELECTRON):
            a, b = sort_rows(P.particles(s)), sort_rows(R.particles(s)[0])
            assert a.shape == b.shape
            assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
        g, rg = P.grid(), R.grid()
        assert np.abs(g[..., :17] - rg[..., :17]).max() <= 1e-15 * np.abs(g).max()


def test_output_file_is_byte_identical(tmp_path, monkeypatch):
    ref_dir, mine_dir = tmp_path / "ref", tmp_path / "mine"
    ref_dir.mkdir()
    mine_dir.mkdir()
    monkeypatch.chdir(ref_dir)
    R = reference_state(4)
    R.output(7)
    with gpu_ctx() as P:
        P.set_grid(R.grid())
        P.write_output(str(mine_dir), 7)
    name = "fdtd458-0-0-7.dat"
    a = (ref_dir / name).read_bytes()
    b = (mine_dir / name).read_bytes()
    assert len(a) > 0 and a == b


def test_thrust_lines(tmp_path):
    O = make_oracle("tiny")
    O.call("init_grid")
    O.call("init_particle_flat")
    O.call("add_flat")
    for _ in range(3):
        O.step()
    ref = O.thrust()
    with gpu_ctx(diag_every_step=1) as P:
        P.set_grid(O.grid())
        for s in (ION, ELECTRON):
            rows, flag = O.particles(s)
            P.set_particles(s, rows, flag)
        P.append_thrust(str(tmp_path), 12)
        P.append_thrust(str(tmp_path), 13)
        line = (tmp_path / "thrust458.txt").read_text().splitlines()
        assert len(line) == 2 and line[0].split()[0] == "12" and line[1].split()[0] == "13"
        expect = "12" + "".join(f" {v:.3E}" for v in ref[:27]) + "".join(f" {v:.8E}" for v in ref[27:])
        got = [float(x) for x in line[0].split()[1:]]
        want = [float(x) for x in expect.split()[1:]]
        assert len(got) == 33
        # three significant digits for F, nine for E (the reference's formats)
        assert np.allclose(got[:27], want[:27], rtol=2e-3, atol=1e-300)
        assert np.allclose(got[27:], want[27:], rtol=1e-8)
        P.step(2)
        Fave = P.thrust_fave()
        P.append_thrust_ave(str(tmp_path), 499)  # not a multiple of 500: nothing written
        assert not (tmp_path / "thrust458_ave.txt").exists()
        P.append_thrust_ave(str(tmp_path), 500)
        ave = (tmp_path / "thrust458_ave.txt").read_text().split()
        assert ave[0] == "500" and len(ave) == 28
        assert np.allclose([float(x) for x in ave[1:]], Fave, rtol=2e-3, atol=1e-300)
        assert np.all(P.thrust_fave() == 0)  # the running mean restarted
