"""Domain decomposition (PROCESS_Nx x PROCESS_Ny ranks) against the reference
run as an MPI job of the same ranks (oracle/multirank.py: the reference
compiled with PROCESS_Nx, PROCESS_Ny > 1 over a multi-process MPI stand-in).
The engine's ranks are contexts of one process exchanging through the
in-process transport (plasmasim_b200.decomp), all on the test's one GPU; no
kernel of one rank waits for another.

Tolerances as the single-domain parity tests: FP64 particle state 1e-13
relative (velocities 1e-12), grid quantities 1e-11 of each field's maximum.
"""
import os

import numpy as np
import pytest

from oracle import build as obuild
from oracle.multirank import grid_of, run_ranks, scenario_refill, scenario_steps
from oracle.pyoracle import params_from_defines
from plasmasim_b200 import ELECTRON, ION, DecomposedPic3D, Pic3D, PicError
from plasmasim_b200.decomp import LocalGroup, NcclTransport
from tests.util import config_from_oracle_params, field_rel_err, rel_norm, sort_rows

pytestmark = pytest.mark.gpu

NAMES = ["tiny_2x1", "tiny_2x2", "damped_2x2"]


def need(name):
    if not os.path.isfile(obuild.ref_lib_path(name)):
        pytest.skip("the compiled reference (oracle/_ref) is not built")


def config(name, **kw):
    return config_from_oracle_params(params_from_defines(obuild.REF_CONFIGS[name]), precision=64, **kw)


def check_rows(mine, ref, what, tol=1e-13):
    mine, ref = sort_rows(mine), sort_rows(ref)
    assert mine.shape == ref.shape, (what, mine.shape, ref.shape)
    assert rel_norm(mine[:, :3], ref[:, :3]) <= tol, what
    assert rel_norm(mine[:, 3:6], ref[:, 3:6]) <= 10 * tol, what


@pytest.mark.parametrize("name", NAMES)
def test_init_matches_reference(name):
    """init_grid (B0 of the global dipole on each rank) and init_particle_flat
    (each rank's own random streams)."""
    need(name)
    ref = run_ranks(name, scenario_steps, (0,))
    px, py = grid_of(name)
    with DecomposedPic3D(config(name), px, py) as D:
        D.init_grid()
        D.init_particle_flat()
        for r, P in enumerate(D.ranks):
            err = field_rel_err(P.grid(), ref[r]["grid"], range(6))
            assert all(e <= 1e-13 for e in err.values()), (r, err)
            # the extra ghost particle is still in the engine's store here
            nx = P.cfg.nx
            for s, key in ((ION, "start_ion"), (ELECTRON, "start_electron")):
                rows = P.particles(s)
                check_rows(rows[rows[:, 0] < (nx + 2) * P.cfg.dx], ref[r][key], (r, key))
            assert list(P.rng_counters()) == list(ref[r]["rng"])


@pytest.mark.parametrize("name", NAMES)
def test_steps_match_reference(name):
    """Eight loop bodies: pushes with particles crossing between ranks, the
    ghost exchanges of B and E, the current folds and the rank-0 / last-rank
    particle losses of sr_particle."""
    need(name)
    nsteps = 8
    ref = run_ranks(name, scenario_steps, (nsteps,))
    px, py = grid_of(name)
    cfg = config(name, add_interval=1000000, sort_interval=1000000, diag_every_step=0)
    with DecomposedPic3D(cfg, px, py) as D:
        D.init_grid()

        def load(r, P):
            P.set_particles(ION, ref[r]["start_ion"])
            P.set_particles(ELECTRON, ref[r]["start_electron"])

        D.each(load)
        D.step(nsteps)
        F, E = D.thrust_f()
        for r, P in enumerate(D.ranks):
            check_rows(P.particles(ION), ref[r]["ion"], (r, "ion"))
            check_rows(P.particles(ELECTRON), ref[r]["electron"], (r, "electron"))
            err = field_rel_err(P.grid(), ref[r]["grid"], range(17))
            bad = {f: e for f, e in err.items() if e > 1e-11}
            assert not bad, (r, bad)
            assert P.status()[0] == 0
        # thrust_f's sums over every rank (MPI_Allreduce)
        t = np.concatenate([F, E])
        want = sum(x["thrust"] for x in ref)
        for q in [0, 1, 2, 3, 4, 5, 9, 10, 11, 27, 28, 29, 30]:
            scale = max(abs(want[q]), np.abs(want[:3]).max() if q < 27 else 0)
            assert abs(t[q] - want[q]) <= 1e-10 * scale, (q, t[q], want[q])


@pytest.mark.parametrize("name", NAMES)
def test_refill_matches_reference(name):
    """add_*_flat on every rank: the shells each rank deletes and the slabs it
    refills depend on where it sits in the process grid (:6015-6401). The
    refill is bit-exact; the deletion differs from the reference only by the
    node its list code skips after a deleted head."""
    need(name)
    ref = run_ranks(name, scenario_refill)
    px, py = grid_of(name)
    with DecomposedPic3D(config(name), px, py) as D:
        D.init_grid()
        D.init_particle_flat()  # draws what the reference's init draws on each rank's streams

        def load(r, P):
            P.set_particles(ION, ref[r]["ion_before"])
            P.set_particles(ELECTRON, ref[r]["electron_before"])

        D.each(load)
        D.add_flat()
        for r, P in enumerate(D.ranks):
            assert list(P.rng_counters()) == list(ref[r]["rng"]), r
            for s, key in ((ION, "ion"), (ELECTRON, "electron")):
                mine = P.particles(s)
                want = ref[r][key]
                before = ref[r][key + "_before"]
                n_inj = int(want.shape[0] - np.sum(np.isin(want[:, 0], before[:, 0])))
                # the injected particles come last on both sides, in the same order
                if n_inj:
                    assert rel_norm(mine[-n_inj:, :6], want[-n_inj:, :6]) <= 1e-13, (r, key)
                    assert np.all(mine[-n_inj:, 6] == want[-n_inj:, 6])
                sm = sort_rows(mine[:mine.shape[0] - n_inj])
                sr = sort_rows(want[:want.shape[0] - n_inj])
                # the reference keeps at most one extra survivor (the skipped node)
                assert 0 <= sr.shape[0] - sm.shape[0] <= 1, (r, key, sr.shape, sm.shape)
                if sr.shape[0] > sm.shape[0]:
                    scale = np.abs(sr).max(axis=0)
                    hit = [np.any(np.all(np.abs(sm - row) <= 1e-12 * scale, axis=1)) for row in sr]
                    assert hit.count(False) == 1, (r, key)
                    sr = sr[np.array(hit)]
                check_rows(sm, sr, (r, key, "survivors"))


@pytest.mark.parametrize("transport", ["local", "nccl"])
def test_single_rank_transport_matches_single_domain(transport):
    """A 1 x 1 decomposition that exchanges through a transport (its own
    ghosts and packets sent to itself) gives the single domain's result."""
    name = "tiny"
    cfg = config(name, add_interval=5, sort_interval=20)
    with Pic3D(cfg) as A:
        A.init_grid()
        A.init_particle_flat()
        A.fdtd(8)
        ga, ia, ea = A.grid(), A.particles(ION), A.particles(ELECTRON)
    if transport == "local":
        owner = LocalGroup(1)
        t = owner.transport(0)
    else:
        class _Store(dict):
            def set(self, k, v):
                self[k] = v

            def get(self, k):
                return self[k]
        try:
            owner = NcclTransport(_Store(), 1, 0, 0)
        except PicError as e:
            pytest.skip(f"NCCL unavailable: {e}")
        t = owner.transport()
    try:
        with Pic3D(cfg) as B:
            B.set_transport(t)
            B.init_grid()
            B.init_particle_flat()
            B.fdtd(8)
            err = field_rel_err(B.grid(), ga, range(17))
            assert all(e <= 1e-12 for e in err.values()), err
            check_rows(B.particles(ION), ia, "ion", 1e-12)
            check_rows(B.particles(ELECTRON), ea, "electron", 1e-12)
            assert B.status()[0] == 0
    finally:
        owner.close()
