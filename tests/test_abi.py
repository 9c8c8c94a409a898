"""The C-ABI library: it loads without a GPU, exports every function that
include/plasma_b200.h declares, and its config struct matches the ctypes
mirror field for field. CPU only (no compute calls)."""
import ctypes as C
import os
import re
import subprocess

import pytest

import plasmasim_b200 as pb
from plasmasim_b200 import build as pbuild
from plasmasim_b200.pic2d import _C2Config
from plasmasim_b200.pic3d import _CConfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "plasma_b200.h")


@pytest.fixture(scope="module")
def lib():
    pbuild.build()
    return pb.load_library()


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(pic(?:2d)?_\w+)\(", text, re.M)))


def test_exports_every_declared_function(lib):
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    assert sorted(pb.pic3d.EXPORTED) == names


@pytest.mark.parametrize("struct,mirror", [("pic_config", _CConfig), ("pic2d_config", _C2Config)])
def test_config_layout_matches_header(tmp_path, struct, mirror):
    fields = [f[0] for f in mirror._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void){',
           f'printf("%zu\\n", sizeof({struct}));']
    src += [f'printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    src += ['return 0;}']
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(c), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == C.sizeof(mirror)
    for f, off in zip(fields, out[1:]):
        assert getattr(mirror, f).offset == off, f


def test_error_strings(lib):
    for code in range(0, 6):
        assert lib.pic_error_string(code)


def test_config_default_is_reference_block(lib):
    cfg = _CConfig()
    assert lib.pic_config_default(C.byref(cfg), 8, 8, 512) == 0
    # PIC/3d_pic458_domain.c:61-103
    assert (cfg.dx, cfg.dt, cfg.np, cfg.v_drift, cfg.n_all) == (1.5, 1.5e-9, 16, 1.2e7, 5e10)
    assert (cfg.ti, cfg.te, cfg.coil_r, cfg.coil_i) == (1e9, 1e9, 2.0, 6.8e7)
    assert (cfg.absorb_grid, cfg.absorb_grid2, cfg.add_interval, cfg.sort_interval) == (32, 40, 5, 500)
    assert cfg.me == cfg.mi / 100.0


def test_invalid_config_rejected_without_device(lib):
    cfg = _CConfig()
    lib.pic_config_default(C.byref(cfg), 8, 8, 8)
    cfg.precision = 16
    h = C.c_void_p()
    assert lib.pic_create(C.byref(cfg), C.byref(h)) == 1  # PIC_ERR_ARG before touching CUDA
    cfg.precision = 32
    cfg.nx = 2000
    assert lib.pic_create(C.byref(cfg), C.byref(h)) == 1


def test_null_arguments(lib):
    assert lib.pic_create(None, None) == 1
    assert lib.pic_destroy(None) == 0
    assert lib.pic_step(None, 1) == 1
