"""The reference run as an MPI job of several ranks (oracle/multirank.py over
the multi-process MPI stand-in), pinned to the reference run as one rank on
the job's global grid where the two must agree bit for bit: the dipole field
B0 of init_grid, evaluated at global coordinates (:4588-4614), and the
damping-free initial state's field record elsewhere."""
import numpy as np
import pytest

from oracle import build as obuild
from oracle.multirank import run_ranks, scenario_state
from oracle.pyoracle import Reference


def _global_b0(q):
    R = Reference("wide16")
    R.init_grid()
    q.put(R.grid()[..., 3:6])


def test_two_rank_b0_is_the_global_dipole():
    if not obuild.reference_available():
        pytest.skip("reference source not available")
    for name in ("tiny_2x1", "wide16"):
        obuild.build_ref(name)
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_global_b0, args=(q,))
    p.start()
    glob = q.get(timeout=120)
    p.join()
    ranks = run_ranks("tiny_2x1", scenario_state, (0,))
    for r, res in enumerate(ranks):
        window = glob[8 * r: 8 * r + 12]
        assert np.array_equal(res["grid"][..., 3:6], window), r
    # the two ranks' streams differ (keys 0 and 10000)
    assert not np.array_equal(ranks[0]["ion"][:8], ranks[1]["ion"][:8])
