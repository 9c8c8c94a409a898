"""The compiled reference as an MPI job of several ranks (test infrastructure).

A geometry of oracle.build.REF_CONFIGS with ORACLE_PNX x ORACLE_PNY > 1 is
compiled against the multi-process MPI stand-in (oracle/shim/mpi_shim.c).
`run_ranks` starts one process per rank (spawned, so that each holds its own
copy of the reference's globals), points the stand-in at a rendezvous
directory, and runs a scenario function in every rank. The scenario receives
the rank's `oracle.pyoracle.Reference` and returns a picklable result; the
call returns the results in rank order (rank = myrank_y * PROCESS_Nx +
myrank_x, as main() numbers them, PIC/3d_pic458_domain.c:205-206).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import queue
import tempfile
import traceback

from . import build as _build


def grid_of(name: str):
    d = _build.REF_CONFIGS[name]
    return int(d.get("ORACLE_PNX", 1)), int(d.get("ORACLE_PNY", 1))


def _rank_main(name, rank, size, sockdir, workdir, scenario, args, q):
    os.environ["ORACLE_MPI_RANK"] = str(rank)
    os.environ["ORACLE_MPI_SIZE"] = str(size)
    os.environ["ORACLE_MPI_DIR"] = sockdir
    os.chdir(workdir)
    try:
        from oracle.pyoracle import Reference

        R = Reference(name)
        q.put((rank, scenario(R, *args), None))
    except Exception:  # reported to the parent, which raises
        q.put((rank, None, traceback.format_exc()))


def run_ranks(name: str, scenario, args=(), timeout: float = 300.0):
    """Runs scenario(R, *args) on every rank of geometry `name`."""
    pnx, pny = grid_of(name)
    size = pnx * pny
    path = _build.ref_lib_path(name)
    if not os.path.isfile(path):
        _build.build_ref(name)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with tempfile.TemporaryDirectory(prefix="ormpi", dir="/tmp") as sockdir, \
            tempfile.TemporaryDirectory(prefix="orwork") as workdir:
        procs = [ctx.Process(target=_rank_main, args=(name, r, size, sockdir, workdir, scenario, args, q))
                 for r in range(size)]
        for p in procs:
            p.start()
        results, errors = {}, []
        try:
            for _ in range(size):
                rank, out, err = q.get(timeout=timeout)
                if err:
                    errors.append(f"rank {rank}:\n{err}")
                results[rank] = out
        except queue.Empty:
            errors.append(f"ranks did not finish within {timeout} s")
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
                p.join()
        if errors:
            raise RuntimeError("\n".join(errors))
    return [results[r] for r in range(size)]


# ----------------------------------------------------------- scenarios
def scenario_state(R, nsteps: int = 0, sort_every: int = 500, add_every: int = 5):
    """init_grid, init_particle_flat, then nsteps loop bodies of fdtd
    (oracle/ref_harness.c ref_loop); returns the rank's grid, particles, RNG
    counters and its part of the thrust sums."""
    import numpy as np

    R.init_grid()
    R.init_particle_flat()
    if nsteps:
        R.L.ref_loop(nsteps, sort_every, add_every)
    return dict(grid=R.grid(), ion=R.particles(0)[0], electron=R.particles(1)[0],
                rng=np.array([R.rng_counter(0), R.rng_counter(1)], dtype=np.int64),
                thrust=R.thrust(include_tail=True))


def _drop_ghost_particle(R):
    """Removes init_particle_flat's extra particle, which the loop leaves in
    ghost cell x = Nx + 2 (a sort before the first push drops it; the engine
    sorts before its first push, the reference loop does not)."""
    nx = R.params["nx"]
    rows = [R.particles(s)[0] for s in (0, 1)]
    rows = [r[r[:, 0] < (nx + 2) * R.params["dx"]] for r in rows]
    R.set_particles(rows[0], rows[1])
    return rows


def scenario_steps(R, nsteps: int):
    """init, the extra particle removed, nsteps loop bodies without a refill
    (add every 10^6 steps) and without a sort; the rank's state and its part
    of the thrust sums."""
    import numpy as np

    R.init_grid()
    R.init_particle_flat()
    start = _drop_ghost_particle(R)
    R.L.ref_loop(nsteps, 1000000, 1000000)
    return dict(start_ion=start[0], start_electron=start[1], grid=R.grid(), ion=R.particles(0)[0],
                electron=R.particles(1)[0], thrust=R.thrust(include_tail=True),
                rng=np.array([R.rng_counter(0), R.rng_counter(1)], dtype=np.int64))


def scenario_refill(R):
    """init, the extra particle removed, then add_ion_flat + add_electron_flat
    on this rank: the particles before and after, and the RNG counters."""
    import numpy as np

    R.init_grid()
    R.init_particle_flat()
    before = _drop_ghost_particle(R)
    R.op("add_flat")
    return dict(ion_before=before[0], electron_before=before[1], ion=R.particles(0)[0],
                electron=R.particles(1)[0],
                rng=np.array([R.rng_counter(0), R.rng_counter(1)], dtype=np.int64))

