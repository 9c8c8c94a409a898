"""Failure paths of the C ABI, each made on the host: an allocation the device
cannot satisfy, checkpoint files cut short or of the wrong size, and an
exchange partner that never arrives. Every failure returns a status code,
leaves the device usable and faults nothing on the GPU.
"""
import os
import shutil
import time

import numpy as np
import pytest

from oracle import build as obuild
from oracle.pyoracle import params_from_defines
from plasmasim_b200 import ELECTRON, ION, DecomposedPic3D, Pic3D, PicError
from tests.util import config_from_oracle_params, oracle_params

pytestmark = pytest.mark.gpu

PIC_ERR_ARG, PIC_ERR_CUDA, PIC_ERR_COMM = 1, 2, 7


def tiny(**kw):
    return config_from_oracle_params(oracle_params("tiny"), precision=32, diag_every_step=0, **kw)


def test_allocation_failure_leaves_the_device_usable():
    """2e9 particle slots per species (four 64 GB record buffers in FP32)
    exceed the device: pic_create fails with PIC_ERR_CUDA, frees what it had
    allocated, and a context created afterwards steps normally."""
    with pytest.raises(PicError) as e:
        Pic3D(tiny(capacity=2_000_000_000))
    assert e.value.code == PIC_ERR_CUDA
    with Pic3D(tiny()) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(2)
        assert P.status()[0] == 0
        assert P.particle_count(ION) > 0


def _cut(path, nbytes):
    with open(path, "r+b") as f:
        f.truncate(nbytes)


def test_truncated_checkpoints_are_rejected(tmp_path):
    """continue_job's files (:7676-7911) as suspend_job writes them load back;
    a field file one record short or one byte long, and a particle file cut
    inside a record, return PIC_ERR_ARG before the context's state changes."""
    good = tmp_path / "good"
    good.mkdir()
    with Pic3D(tiny()) as P:
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(2)
        P.save_checkpoint(str(good))
        counts = [P.particle_count(s) for s in (ION, ELECTRON)]
    field = "suspend-0-field.dat"
    ion = "suspend-0-0-ion.dat"
    rec = 18 * 8
    cases = {
        "field short": (field, os.path.getsize(good / field) - rec),
        "field long": (field, os.path.getsize(good / field) + 1),
        "particles cut": (ion, os.path.getsize(good / ion) - 40),
    }
    for what, (name, size) in cases.items():
        d = tmp_path / what.replace(" ", "_")
        shutil.copytree(good, d)
        _cut(d / name, size)
        with Pic3D(tiny()) as Q:
            Q.init_grid()
            with pytest.raises(PicError) as e:
                Q.load_checkpoint(str(d))
            assert e.value.code == PIC_ERR_ARG, what
            assert Q.particle_count(ION) == 0 and Q.particle_count(ELECTRON) == 0, what
    with Pic3D(tiny()) as Q:
        Q.init_grid()
        Q.load_checkpoint(str(good))
        assert [Q.particle_count(s) for s in (ION, ELECTRON)] == counts


def _decomposed():
    p = params_from_defines(obuild.REF_CONFIGS["tiny_2x1"])
    D = DecomposedPic3D(config_from_oracle_params(p, precision=32, diag_every_step=0), 2, 1)
    D.group.set_timeout(300)
    D.init_grid()
    D.init_particle_flat()
    return D


@pytest.mark.parametrize("call", ["thrust_f", "step"])
def test_exchange_partner_never_arrives(call):
    """Two ranks of an in-process group with a 300 ms rendezvous limit; rank 1
    stops making calls. Rank 0's all-reduce (thrust_f's MPI_Allreduce) or its
    first ghost exchange (sr_b inside the step) returns PIC_ERR_COMM after the
    limit instead of blocking; no kernel waits on the other rank."""
    with _decomposed() as D:
        t0 = time.monotonic()
        with pytest.raises(PicError) as e:
            getattr(D.ranks[0], call)()
        waited = time.monotonic() - t0
        assert e.value.code == PIC_ERR_COMM
        assert 0.25 <= waited < 10.0
        D.ranks[0].synchronize()  # the context's stream still completes
