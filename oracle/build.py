"""Build recipes for the CPU oracles (test infrastructure only).

Two things are built here:

* ``oracle/liboracle3d.so`` -- the project's own FP64 CPU restatement of the
  reference time step (``oracle/pic_oracle.c``), parameterised at run time.
* ``oracle/_ref/libref3d_<name>.so`` -- the reference program
  ``PIC/3d_pic458_domain.c`` itself, compiled from where it lies under the
  reference checkout, with its compile-time ``#define`` values replaced per
  geometry by ``oracle/ref_patch.sed`` (the patched text is piped straight into
  gcc; no copy of the reference source is written anywhere), the project-written
  size-1 MPI and GSL-subset shims under ``oracle/shim``, and the harness
  ``oracle/ref_harness.c`` appended to the same translation unit.

The reference is only present in the development container; on a machine
without it the prebuilt ``oracle/_ref`` libraries (if any) are used as they are.
"""
from __future__ import annotations

import math
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: PLASMA_REFERENCE_ROOT, else a "reference" directory
# beside this repository's root.
REF_ROOT = os.environ.get("PLASMA_REFERENCE_ROOT",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
REF_SRC = os.path.join(REF_ROOT, "PIC", "3d_pic458_domain.c")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(HERE, "liboracle3d.so")

# Normalized units: c = e0 = mu0 = 1, q = 1, m_e = 1, m_i = 100 m_e, dx = 1.
# dt is half of the 3D stability limit of the reference's 4th-order
# (27/24, -1/24) curl stencil, dt_max = 6/(7*sqrt(3)) dx/c.
DT_NORM = 0.5 * 6.0 / (7.0 * math.sqrt(3.0))
NORMALIZED = dict(
    ORACLE_Q=1.0, ORACLE_MP=100.0, ORACLE_ME=1.0, ORACLE_MU0=1.0, ORACLE_E0=1.0,
    ORACLE_KB=1.0, ORACLE_C=1.0, ORACLE_MASS_RATIO=100.0,
    ORACLE_DX=1.0, ORACLE_DT=DT_NORM,
    # drifting Maxwellian: v_th,e = 0.05 c (kT = 0.0025 m_e c^2), drift 0.1 c
    ORACLE_V=0.1, ORACLE_NALL=0.01, ORACLE_TI=0.0025, ORACLE_TE=0.0025,
    # dipole moment I*pi*R^2 with mu0*I*R^2/(4*4^3) = 0.5: |B| = 0.5 at 4 cells
    # in the equatorial plane; moment along the reference's y (alpha = pi/2)
    ORACLE_R=2.0, ORACLE_I=32.0, ORACLE_ALPHA="(Pi/2.)",
    ORACLE_SIGMA_A=1e-6,
)
# The reference's own MKSA parameters (PIC/3d_pic458_domain.c:52-75).
MKSA = dict(
    ORACLE_MASS_RATIO=100.0, ORACLE_DX=1.5, ORACLE_DT=1.5e-9, ORACLE_V=1.2e7,
    ORACLE_NALL=5e10, ORACLE_TI=1e9, ORACLE_TE=1e9, ORACLE_R=2.0, ORACLE_I=6.8e7,
    ORACLE_ALPHA="(Pi/2.)", ORACLE_SIGMA_A=1e-6,
)


def _geom(nx, ny, nz, np_, absorb=0, absorb2=0, threads=1, pack=20000, absorb3=40, phi=0, pnx=1, pny=1):
    return dict(ORACLE_NX=nx, ORACLE_NY=ny, ORACLE_NZ=nz, ORACLE_NP=np_,
                ORACLE_ABSORB=absorb, ORACLE_ABSORB2=absorb2,
                ORACLE_THREADS=threads, ORACLE_PACK_N=pack,
                ORACLE_ABSORB3=absorb3, ORACLE_PHI=phi, ORACLE_PNX=pnx, ORACLE_PNY=pny)


REF_CONFIGS = {
    # small cube used by most parity tests
    "tiny": {**NORMALIZED, **_geom(8, 8, 8, 4)},
    # non-cubic grid, absorbing layers and a strong damping amplitude
    "damped": {**NORMALIZED, **_geom(10, 12, 14, 2, absorb=3, absorb2=3), "ORACLE_SIGMA_A": 0.05},
    # the reference's own MKSA constants on a small grid
    "mksa": {**MKSA, **_geom(8, 8, 12, 4, absorb=2, absorb2=2)},
    # 32^3 cells, 8 particles/cell/species: the CPU-runnable configuration
    "cube32": {**NORMALIZED, **_geom(32, 32, 32, 8, pack=80000)},
    # 64^3 cells, 16 particles/cell/species: CPU throughput sample
    "cube64": {**NORMALIZED, **_geom(64, 64, 64, 16, pack=400000)},
    # the tiny cube with the reference's PHI blocks compiled in (renew_phi3,
    # sr_phi, sr_e after each renew_e4_2 and after the first add_*_flat);
    # Absorb_grid3 = 0 and 1 (the reference ships 40, which leaves no cell of
    # an 8^3 grid)
    "tiny_phi": {**NORMALIZED, **_geom(8, 8, 8, 4, absorb3=0, phi=1)},
    "tiny_phi1": {**NORMALIZED, **_geom(8, 8, 8, 4, absorb3=1, phi=1)},
    # the reference as an MPI job of 2 x 1 and 2 x 2 ranks of 8^3 cells each
    # (oracle/shim/mpi_shim.c runs the ranks as processes; oracle/multirank.py
    # drives them); absorbing layers 2 and 3 cells wide on the global domain
    "tiny_2x1": {**NORMALIZED, **_geom(8, 8, 8, 4, pnx=2, pny=1)},
    # one rank over the 2 x 1 job's global grid (16 x 8 x 8)
    "wide16": {**NORMALIZED, **_geom(16, 8, 8, 4)},
    "tiny_2x2": {**NORMALIZED, **_geom(8, 8, 8, 4, pnx=2, pny=2)},
    "damped_2x2": {**NORMALIZED, **_geom(8, 8, 10, 2, absorb=2, absorb2=3, pnx=2, pny=2), "ORACLE_SIGMA_A": 0.05},
    # the benchmark workload, 128^3 cells x 64 particles/cell/species, with
    # OpenMP on: THREAD_N = active_thread = 64 particle lists and threads (the
    # reference ships THREAD_N 4 and active_thread 1 and is built with -h omp);
    # ref_set_threads picks the threads of a run, 1 for the shipped setting
    "cube128_t64": {**NORMALIZED, **_geom(128, 128, 128, 64, threads=64, pack=20000),
                    "ORACLE_ACTIVE_THREADS": 64},
}

# a quarter of that volume, 64 x 64 x 128 cells x 64 particles/cell/species:
# a bounded CPU sample of the same workload
REF_CONFIGS["quarter128_t64"] = {**NORMALIZED, **_geom(64, 64, 128, 64, threads=64, pack=20000),
                                 "ORACLE_ACTIVE_THREADS": 64}

# geometries that are large to build or run and are built only on request
ON_REQUEST = {"cube128_t64", "quarter128_t64"}


# The 2D reference (PIC2D/2d_pic278_mpi.c) in normalized units: c = e0 = mu0 =
# q = m_e = dx = 1, m_i = 100; dt at half of the 2D stability limit of the
# (27/24, -1/24) stencil, 6/(7 sqrt 2) dx/c; drift 0.1 c, v_th,e = 0.05 c.
REF2D_SRC = os.path.join(REF_ROOT, "PIC2D", "2d_pic278_mpi.c")
DT2D_NORM = 0.5 * 6.0 / (7.0 * math.sqrt(2.0))
NORMALIZED_2D = dict(
    ORACLE_Q=1.0, ORACLE_MI=100.0, ORACLE_ME=1.0, ORACLE_MU0=1.0, ORACLE_E0=1.0, ORACLE_KB=1.0,
    ORACLE_C=1.0, ORACLE_DX=1.0, ORACLE_DT=DT2D_NORM, ORACLE_V=0.1, ORACLE_NALL=0.01,
    ORACLE_TI=0.0025, ORACLE_TE=0.0025, ORACLE_R=2.0, ORACLE_I=12.0, ORACLE_ALPHA=0.0,
    ORACLE_SIGMA_A=1e-6,
)


def _geom2d(nx, nz, np_, absorb, absorb2, absorb3, pack=20000):
    return dict(ORACLE_NX=nx, ORACLE_NZ=nz, ORACLE_NP=np_, ORACLE_ABSORB=absorb,
                ORACLE_ABSORB2=absorb2, ORACLE_ABSORB3=absorb3, ORACLE_PACK_N=pack)


REF2D_CONFIGS = {
    # a small strip: 16 x 32 cells, 2 x 2 particles per cell per species
    "strip": {**NORMALIZED_2D, **_geom2d(16, 32, 2, 4, 2, 4)},
    # 64 x 64 cells, 4 x 4 particles per cell: a batch run of the smallest size
    "sq64": {**NORMALIZED_2D, **_geom2d(64, 64, 4, 8, 4, 8)},
    # 32 x 128 cells, 3 x 3 particles per cell, a different current and drift
    "rect": {**NORMALIZED_2D, **_geom2d(32, 128, 3, 6, 3, 6), "ORACLE_I": 20.0, "ORACLE_V": 0.15},
    # 32 x 16 cells, 3 x 3 particles per cell: half of a 32-cell z tile of the
    # batched push (the reference's sine transform needs power-of-two sides)
    "half": {**NORMALIZED_2D, **_geom2d(32, 16, 3, 4, 2, 4), "ORACLE_I": 12.0, "ORACLE_V": 0.2},
}


def ref2d_lib_path(name: str) -> str:
    return os.path.join(REF_OUT, f"libref2d_{name}.so")


def build_ref2d(name: str, force: bool = False) -> str:
    """Compile the 2D reference at geometry ``name`` (size-1 MPI and GSL-subset
    shims, harness oracle/ref2d_harness.c); returns the library path."""
    out = ref2d_lib_path(name)
    if os.path.isfile(out) and not force:
        return out
    if not os.path.isfile(REF2D_SRC):
        raise FileNotFoundError(f"2D reference source not found at {REF2D_SRC}")
    os.makedirs(REF_OUT, exist_ok=True)
    defs = [f"-D{k}={_fmt(v)}" for k, v in REF2D_CONFIGS[name].items()]
    sed = subprocess.run(["sed", "-f", os.path.join(HERE, "ref2d_patch.sed"), REF2D_SRC],
                         check=True, capture_output=True)
    with open(os.path.join(HERE, "ref2d_harness.c"), "rb") as f:
        tu = sed.stdout + b"\n" + f.read()
    cmd = ["gcc", "-x", "c", "-", "-x", "none",
           os.path.join(HERE, "shim", "gsl_shim.c"), os.path.join(HERE, "shim", "mpi_shim.c"),
           "-std=gnu11", "-O2", "-ffp-contract=off", "-fgnu89-inline", "-fPIC", "-shared", "-w",
           "-I", os.path.join(HERE, "shim"), "-include", os.path.join(HERE, "ref_pre.h"),
           *defs, "-lm", "-o", out]
    subprocess.run(cmd, input=tu, check=True)
    return out


def ref_lib_path(name: str) -> str:
    return os.path.join(REF_OUT, f"libref3d_{name}.so")


def reference_available() -> bool:
    return os.path.isfile(REF_SRC)


def _fmt(v) -> str:
    if isinstance(v, float):
        return repr(v)
    return str(v)


def build_ref(name: str, force: bool = False) -> str:
    """Compile the reference at geometry ``name``; returns the library path."""
    out = ref_lib_path(name)
    if os.path.isfile(out) and not force:
        return out
    if not reference_available():
        raise FileNotFoundError(f"reference source not found at {REF_SRC}")
    os.makedirs(REF_OUT, exist_ok=True)
    defs = [f"-D{k}={_fmt(v)}" for k, v in REF_CONFIGS[name].items()]
    sed = subprocess.run(["sed", "-f", os.path.join(HERE, "ref_patch.sed"), REF_SRC],
                         check=True, capture_output=True)
    with open(os.path.join(HERE, "ref_harness.c"), "rb") as f:
        tu = sed.stdout + b"\n" + f.read()
    # OpenMP for the threaded configurations; their static per-thread grids
    # (grid_thread[THREAD_N][...], :149) pass 2 GB, beyond the small code model
    omp = (["-fopenmp", "-mcmodel=medium"] if REF_CONFIGS[name].get("ORACLE_ACTIVE_THREADS", 1) > 1 else [])
    cmd = ["gcc", "-x", "c", "-", "-x", "none",
           os.path.join(HERE, "shim", "gsl_shim.c"), os.path.join(HERE, "shim", "mpi_shim.c"),
           "-std=gnu11", "-O2", "-ffp-contract=off", "-fgnu89-inline", "-fPIC", "-shared", "-w", *omp,
           "-I", os.path.join(HERE, "shim"), "-include", os.path.join(HERE, "ref_pre.h"),
           *defs, "-lm", "-lpthread", "-o", out]
    subprocess.run(cmd, input=tu, check=True)
    return out


def build_oracle(force: bool = False) -> str:
    """Compile the project's FP64 restatement of the step (oracle/pic_oracle.c)
    together with its tangent-linear (oracle/tangent.c, which includes it)."""
    srcs = [os.path.join(HERE, "pic_oracle.c"), os.path.join(HERE, "tangent.c")]
    src = srcs[1]
    if (os.path.isfile(ORACLE_SO) and not force
            and os.path.getmtime(ORACLE_SO) >= max(os.path.getmtime(f) for f in srcs)):
        return ORACLE_SO
    cmd = ["gcc", "-std=gnu11", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-Wall",
           "-Wno-unused-function", "-I", HERE, src, os.path.join(HERE, "shim", "gsl_shim.c"),
           "-lm", "-o", ORACLE_SO]
    subprocess.run(cmd, check=True)
    return ORACLE_SO


def build_all(force: bool = False) -> None:
    build_oracle(force)
    if reference_available():
        for name in REF_CONFIGS:
            build_ref(name, force and name not in ON_REQUEST)
    if os.path.isfile(REF2D_SRC):
        for name in REF2D_CONFIGS:
            build_ref2d(name, force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
