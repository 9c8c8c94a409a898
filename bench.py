"""Benchmark of the B200 PIC step: particle-steps/s of push + deposit + FDTD
(with boundary refill every 5 steps and a cell sort every 20) on the 3D
solar-wind/dipole plasma of 128^3 cells x 64 particles/cell/species
(268,435,456 particles), FP32 path, with the FP64 path timed on the same seed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU (torchrun, one process per GPU): every rank advances an independent
replica of the workload (the single-domain path has no data exchange between
runs); value = all ranks' particle-steps / max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s (push+deposit+FDTD)"
UNIT = "particle-steps/s"
NX = NY = NZ = 128
PPC = 64
SORT_EVERY = 20
ADD_EVERY = 5


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle-reason samples while the timed region runs: NVML
    read every 10 ms from a thread (reads only), else nvidia-smi at its
    200 ms floor."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []  # (sm MHz, max sm MHz, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap)
        self.proc = None
        self.stop = threading.Event()
        self.thread = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = None
            try:  # the CUDA device by its PCI address (NVML numbers all GPUs, CUDA the visible ones)
                import torch

                pr = torch.cuda.get_device_properties(self.index)
                h = pynvml.nvmlDeviceGetHandleByPciBusId(
                    f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0")
            except Exception:
                h = None
            if h is None:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            bits = [pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap]
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def poll():
                while not self.stop.is_set():
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.rows.append((float(sm), float(mx), *[bool(r & b) for b in bits]))
                    self.stop.wait(0.01)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 6 and parts[0].replace(".", "").isdigit() and parts[1].replace(".", "").isdigit():
                self.rows.append((float(parts[0]), float(parts[1]), *[p == "Active" for p in parts[2:6]]))

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[2 + i]})
        return {"sm_mhz": statistics.median(r[0] for r in self.rows),
                "sm_max_mhz": max(r[1] for r in self.rows), "reasons": reasons,
                "samples": len(self.rows), "source": "nvml" if self.proc is None else "nvidia-smi"}


# ------------------------------------------------------------------ CPU side
def _reference_threaded_worker(name, phases, warm, budget_s, q):
    from oracle.pyoracle import Reference

    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        R = Reference(name)
        lists = R.L.ref_set_threads(phases[0][0])
        t0 = time.perf_counter()
        R.init_grid()
        R.init_particle_flat()
        R.op("add_flat")              # fdtd's refill before its loop
        init_s = time.perf_counter() - t0
        if warm:
            R.L.ref_loop(warm, SORT_EVERY, ADD_EVERY)
        out = []
        for threads, steps in phases:
            R.L.ref_set_threads(threads)
            n0 = R.L.ref_count(0) + R.L.ref_count(1)
            done, secs = 0, 0.0
            while done < steps and (done == 0 or secs < budget_s):
                t1 = time.perf_counter()
                R.L.ref_loop(1, SORT_EVERY, ADD_EVERY)
                secs += time.perf_counter() - t1
                done += 1
            n1 = R.L.ref_count(0) + R.L.ref_count(1)
            out.append({"psteps": 0.5 * (n0 + n1) * done, "secs": secs, "steps": done, "particles": n0,
                        "init_s": init_s, "lists": lists, "threads": threads})
        q.put(out)


def reference_threaded(name: str, phases, warm: int, budget_s: float = 150.0):
    """The reference program compiled with OpenMP (oracle/_ref, THREAD_N = 64
    particle lists) at geometry `name`, in a spawned process: init, the
    initial refill and `warm` untimed loop bodies on the first phase's
    threads, then for each (threads, steps) of `phases` up to `steps` timed
    loop bodies on that many host threads (fewer when they pass `budget_s`).
    Its loop is fdtd's body (:687-949): the particle loops run one list per
    thread (:731, :818), the field loops split over x. One result per phase."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_reference_threaded_worker, args=(name, list(phases), warm, budget_s, q))
    p.start()
    res = q.get()
    p.join()
    return res


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def ensure_reference_lib(name: str) -> bool:
    from oracle import build as obuild

    if os.path.isfile(obuild.ref_lib_path(name)):
        return True
    if obuild.reference_available():
        obuild.build_ref(name)
        return True
    return False


# ------------------------------------------------------------------ GPU side
def make_config(precision: int, seed: int):
    from plasmasim_b200 import PicConfig

    return PicConfig.normalized(NX, NY, NZ, PPC, precision=precision, sort_interval=SORT_EVERY,
                                add_interval=ADD_EVERY, diag_every_step=0, seed_p=seed,
                                seed_v=seed + 50)


def run_gpu(precision: int, steps: int, warmup: int, seed: int, dist=None, clocks_index=0):
    """Device-resident timing of `steps` pic_step calls after `warmup` steps."""
    import torch
    from plasmasim_b200 import Pic3D

    P = Pic3D(make_config(precision, seed))
    P.init_grid()
    P.init_particle_flat()
    P.fdtd(0)                      # fdtd's refill before its loop
    P.step(warmup)
    P.synchronize()
    stream = torch.cuda.ExternalStream(P.stream_handle())
    _, c0 = P.status()
    P.set_timing(True)
    _, _, launches0 = P.read_timing()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(clocks_index) as clk:
        start.record(stream)
        P.step(steps)
        stop.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    phase_ms, phase_pairs, launches1 = P.read_timing()
    P.set_timing(False)
    rc, c1 = P.status()
    pushed = int(c1[3] - c0[3])
    out = dict(ms=ms, pushed=pushed, phase_ms=phase_ms, phase_pairs=phase_pairs,
               launches=launches1 - launches0, clocks=clk.summary(), status=int(rc),
               errors=[int(x) for x in c1[:3]])
    return P, out


def run_e2e(P, steps: int):
    """The same step through the public API with host buffers: upload of the
    particle and grid state from pinned host memory, `steps` steps each
    followed by the thrust/energy read-back (thrust_f), download of the final
    particle state. Returns (particle-steps/s, h2d bytes/step, d2h bytes/step)."""
    import numpy as np
    import torch

    from plasmasim_b200 import ELECTRON, ION

    rows = {}
    for s in (ION, ELECTRON):
        n = P.particle_count(s)
        buf = torch.empty((n, 7), dtype=torch.float64, pin_memory=True)
        rows[s] = buf.numpy()
        rows[s][:] = P.particles(s)
    g = torch.empty(P.shape + (18,), dtype=torch.float64, pin_memory=True).numpy()
    g[:] = P.grid()
    _, c0 = P.status()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    P.set_grid(g)
    for s in (ION, ELECTRON):
        P.set_particles(s, rows[s])
    for _ in range(steps):
        P.step(1)
        P.thrust_f()
    outn = 0
    for s in (ION, ELECTRON):
        got = P.particles(s, out=rows[s])
        outn += got.size
    dt = time.perf_counter() - t0
    _, c1 = P.status()
    pushed = int(c1[3] - c0[3])
    h2d = g.nbytes + sum(r.nbytes for r in rows.values())
    d2h = outn * 8 + steps * 33 * 8
    return pushed / dt, h2d / steps, d2h / steps


# DRAM bytes (read + write) per pushed particle of push_tiled_kernel<float>,
# from the ncu capture of a 64^3 x 64 ppc launch
# (profiles/push_tiled_kernel_grid64_64ppc.md); at a fixed number of particles
# per cell the traffic of a launch grows with its particles.
PUSH_TRAFFIC_PER_PARTICLE = 73.0


def roofline(out, npart_species, cells, rsize):
    """Push kernel: algorithmic bytes per launch = particles x (read + write of
    the SoA state: 4 + 6 rsize bytes each way) + cells x rsize x (6 gathered
    field components + 4 deposited quantities)."""
    pushes = out["pushed"]
    launches = out["phase_pairs"]["push"] * 2
    per_particle = 2 * (4 + 6 * rsize)
    bytes_total = pushes * per_particle + launches * cells * rsize * 10
    secs = out["phase_ms"]["push"] / 1e3
    return bytes_total / secs / 1e9, bytes_total / max(launches, 1), secs / max(launches, 1)


def batch2d_configs(nruns: int, seed: int = 7):
    """The batched 2D workload: nruns x-z runs with grid sides uniform in
    [64, 256] (even), Np uniform in [4, 8] (16-64 particles per cell per
    species), coil current uniform in [6, 25] (x0.5-x2 of the current giving
    |B| = 0.5 at 4 cells) and drift uniform in [0.05, 0.2] c; absorb widths
    8 / 4 / 8 cells; each run its own random streams."""
    import numpy as np

    from plasmasim_b200 import Pic2DConfig

    rng = np.random.default_rng(seed)
    cfgs = []
    for r in range(nruns):
        nx, nz = (int(v) // 2 * 2 for v in rng.integers(64, 257, size=2))
        cfgs.append(Pic2DConfig(nx=nx, nz=nz, np=int(rng.integers(4, 9)), coil_i=float(rng.uniform(6, 25)),
                                v_drift=float(rng.uniform(0.05, 0.2)), absorb_grid=8, absorb_grid2=4,
                                absorb_grid3=8, seed_p=1000 * r, seed_v=1000 * r + 50))
    return cfgs


def run_batch2d(nruns: int, steps: int, warmup: int):
    """Device-timed steps of the batched 2D workload (FP32), after init, the
    online launch tuning and at least `warmup` further steps: at least `steps`
    steps, rounded up to whole sort cycles."""
    import torch

    from plasmasim_b200 import Pic2DBatch

    cfgs = batch2d_configs(nruns)
    B = Pic2DBatch(cfgs, precision=32)
    B.init()
    choice = B.autotune()  # 16 steps of the runs themselves
    # the timed window starts with a sort step and covers whole sort cycles,
    # so that it holds each step of the cycle equally often
    si = cfgs[0].sort_interval
    if si > 0:
        B.step(warmup + (-(16 + warmup)) % si)
        steps = -(-steps // si) * si
    else:  # sorts at refills only
        B.step(warmup)
    stream = torch.cuda.ExternalStream(B.stream_handle())
    _, c0 = B.status()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    B.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    rc, c1 = B.status()
    pushed = int(c1[3] - c0[3])
    B.close()
    # algorithmic bytes: every particle's cell and five FP32 values read and written
    peak, kind = measured_peaks()
    gbs = pushed * 48 / (ms / 1e3) / 1e9
    return {"workload": f"{nruns} independent x-z runs (PIC2D), grid sides uniform in [64, 256], "
                        "16-64 particles/cell/species, coil current and drift seeded-random",
            "value": pushed / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "particles": pushed // max(steps, 1),
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "bytes": "particles x 48 (cell + 5 FP32 values, read and written)", "peak_kind": kind},
            "launch_shape": list(choice), "graph": True,
            "kernels_per_step": int(c1[5] - c0[5]) // max(steps, 1), "device_errors": [int(x) for x in c1[:3]]}


def step_batch2d(nruns: int, steps: int, tile_rows: int = 2, blocks: int = 2368):
    """The batched 2D workload stepped with a fixed push shape (no tuning, no
    timing), for profiling the kernels of its steps."""
    from plasmasim_b200 import Pic2DBatch

    B = Pic2DBatch(batch2d_configs(nruns), precision=32)
    B.init()
    B.set_push_shape(tile_rows, blocks)
    B.step(steps)
    rc, counters = B.status()
    B.close()
    return rc, [int(x) for x in counters]


def batch2d_cpu_sample(steps: int = 3):
    """The 2D reference compiled at 64 x 64 cells x 16 ppc (oracle/_ref), one core."""
    from oracle import build as obuild
    from oracle.pyoracle import Reference2D

    if not os.path.isfile(obuild.ref2d_lib_path("sq64")):
        if not os.path.isfile(obuild.REF2D_SRC):
            return None
        obuild.build_ref2d("sq64")
    R = Reference2D("sq64")
    R.init()
    n0 = len(R.particles(0)[0]) + len(R.particles(1)[0])
    t0 = time.perf_counter()
    for _ in range(steps):
        R.step(250)
    dt = time.perf_counter() - t0
    return {"value": n0 * steps / dt, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"2D reference loop body, 64 x 64 cells x 16 ppc/species ({n0} particles), {steps} steps"}


def run_adjoint(nsteps: int = 200, every: int = 20):
    """The adjoint of configs' differentiable run: 64^3 cells x 16 ppc/species,
    nsteps steps with a checkpoint every `every` steps (FP32): wall times of
    the production step, the slot-stable forward and the adjoint, and the
    adjoint against central differences (h = 1e-3 relative) at growing
    horizons."""
    import torch

    from plasmasim_b200 import Pic3D, PicConfig

    def ctx(I=32.0, V=0.1):
        cfg = PicConfig.normalized(64, 64, 64, 16, precision=32, diag_every_step=0, sort_interval=20,
                                   add_interval=5)
        cfg.coil_i, cfg.v_drift = I, V
        P = Pic3D(cfg)
        P.init_grid()
        P.init_particle_flat()
        P.fdtd(0)
        P.synchronize()
        return P

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    def best_of(reps, run, prep=None):
        """Wall time of `run` on a fresh context, the fastest of `reps` runs
        (single wall-clock runs of the adjoint, which reads the particle
        counts back at every refill, varied by up to 2x on one box)."""
        best, res = None, None
        for _ in range(reps):
            P = ctx()
            if prep:
                prep(P)
            r, t = timed(lambda: run(P))
            P.close()
            if best is None or t < best:
                best, res = t, r
        return res, best

    _, t_step = best_of(3, lambda P: P.step(nsteps), prep=lambda P: P.step(3))
    _, t_fwd = best_of(3, lambda P: P.objective(nsteps))
    # each timed adjoint follows one on the same context, whose snapshot and work memory it reuses
    out, t_adj = best_of(3, lambda P: P.adjoint(nsteps, every), prep=lambda P: P.adjoint(nsteps, every))
    checks = []
    h = 1e-3
    for T in sorted({T for T in (5, 20, 50, nsteps) if T <= nsteps}):
        P = ctx()
        J, dI, dV = P.adjoint(T, min(every, T))
        P.close()
        vals = []
        for I, V in ((32 * (1 + h), 0.1), (32 * (1 - h), 0.1), (32, 0.1 * (1 + h)), (32, 0.1 * (1 - h))):
            P = ctx(I, V)
            vals.append(P.objective(T))
            P.close()
        fdI = (vals[0] - vals[1]) / (2 * h * 32)
        fdV = (vals[2] - vals[3]) / (2 * h * 0.1)
        checks.append({"steps": T, "dJ_dI": dI, "fd_dJ_dI": fdI, "rel_err_I": abs(dI / fdI - 1),
                       "dJ_dV": dV, "fd_dJ_dV": fdV, "rel_err_V": abs(dV / fdV - 1)})
    return {"workload": f"64^3 cells x 16 ppc/species, {nsteps} steps, checkpoint every {every}, FP32",
            "timing": "wall clock, fastest of 3 runs on fresh contexts; the adjoint after a first adjoint on its context",
            "objective": "impulse along z delivered to the dipole",
            "timed_run": {"J": out[0], "dJ_dI": out[1], "dJ_dV": out[2],
                          "start": f"the state after a first {nsteps}-step adjoint"},
            "step_ms": t_step / nsteps * 1e3, "forward_ms": t_fwd / nsteps * 1e3, "adjoint_ms": t_adj / nsteps * 1e3,
            "adjoint_over_step": t_adj / t_step, "adjoint_over_forward": t_adj / t_fwd,
            "fd_checks": checks}


def run_thrust_error(steps: int = 200, seed: int = 0):
    """The thrust error the metric is quoted at: the FP32 path against the FP64
    path on the same seed and the benchmark grid, after `steps` steps of fdtd
    (refill every 5, sort every 20). Compares thrust_f's F[27] after the last
    step and thrust_fave's running mean over all steps (27 components each,
    normwise), and the total force (F[0..2]). A second FP32 run from another
    seed gives the sampling noise of the same quantities: the spread between
    two equally valid runs of the plasma."""
    import numpy as np

    from plasmasim_b200 import Pic3D

    def run(precision, s):
        cfg = make_config(precision, s)
        cfg.diag_every_step = 1
        with Pic3D(cfg) as P:
            P.init_grid()
            P.init_particle_flat()
            P.fdtd(steps)
            F, E = P.thrust_f()
            return np.asarray(F), np.asarray(E), np.asarray(P.thrust_fave())

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    t0 = time.perf_counter()
    F64, E64, A64 = run(64, seed)
    F32, E32, A32 = run(32, seed)
    G32, _, B32 = run(32, seed + 1)
    return {"workload": f"{NX}x{NY}x{NZ} cells x {PPC} ppc/species, {steps} steps, FP32 vs FP64 from the same seed",
            "thrust_rel_err": rel(F32, F64), "thrust_total_rel_err": rel(F32[:3], F64[:3]),
            "fave_rel_err": rel(A32, A64), "fave_total_rel_err": rel(A32[:3], A64[:3]),
            "energy_rel_err": [abs(E32[q] / E64[q] - 1) for q in range(4)],
            "seed_spread": {"thrust": rel(G32, F32), "thrust_total": rel(G32[:3], F32[:3]),
                            "fave": rel(B32, A32), "fave_total": rel(B32[:3], A32[:3])},
            "F64_total": [float(x) for x in F64[:3]], "fave64_total": [float(x) for x in A64[:3]],
            "wall_s": time.perf_counter() - t0}


def run_configs2(steps: int = 100, grid: int = 256, ppc: int = 32):
    """The large-grid workload: `grid`^3 cells x `ppc` particles/cell/species
    (256^3 x 32: 1.07 G particles), the dipole moment at 0.5, 1 and 2 times
    the benchmark's (coil current I = 16, 32, 64). For each, the FP32 path
    (tiled layout) and the FP64 path from the same seed -- in slot order, one
    record buffer per species, which is what lets 1.07 G FP64 particles fit
    next to nothing else -- advance `steps` steps of fdtd; their thrust_f
    F[27] and E[6], thrust_fave's running mean and the Gauss-law residual are
    compared (the FP64 run as the reference), and the FP32 steps are timed
    with CUDA events."""
    import numpy as np
    import torch

    from plasmasim_b200 import Pic3D, PicConfig

    def run(precision, coil_i, slot_order):
        cfg = PicConfig.normalized(grid, grid, grid, ppc, precision=precision, sort_interval=SORT_EVERY,
                                   add_interval=ADD_EVERY, diag_every_step=1, slot_order=slot_order)
        cfg.coil_i = coil_i
        with Pic3D(cfg) as P:
            P.init_grid()
            P.init_particle_flat()
            P.fdtd(0)
            stream = torch.cuda.ExternalStream(P.stream_handle())
            _, c0 = P.status()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            P.synchronize()
            e0.record(stream)
            P.step(steps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            rc, c1 = P.status()
            F, E = P.thrust_f()
            return dict(F=np.asarray(F), E=np.asarray(E), fave=np.asarray(P.thrust_fave()),
                        gauss=np.asarray(P.gauss_residual()), ms=ms, pushed=int(c1[3] - c0[3]), rc=int(rc))

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    out = []
    for mult in (0.5, 1.0, 2.0):
        r64 = run(64, 32.0 * mult, 1)
        r32 = run(32, 32.0 * mult, 0)
        out.append({"dipole": mult, "coil_i": 32.0 * mult,
                    "F_rel_err": rel(r32["F"], r64["F"]), "F_total_rel_err": rel(r32["F"][:3], r64["F"][:3]),
                    "fave_rel_err": rel(r32["fave"], r64["fave"]),
                    "E_rel_err": [abs(r32["E"][q] / r64["E"][q] - 1) for q in range(4)],
                    "gauss_rel_err": [abs(r32["gauss"][q] / r64["gauss"][q] - 1) for q in range(3)],
                    "fp32": {"value": r32["pushed"] / (r32["ms"] / 1e3), "ms_per_step": r32["ms"] / steps,
                             "status": r32["rc"]},
                    "fp64_slot_order": {"value": r64["pushed"] / (r64["ms"] / 1e3), "ms_per_step": r64["ms"] / steps,
                                        "status": r64["rc"]},
                    "particles": r32["pushed"] // max(steps, 1)})
        log(json.dumps(out[-1]))
    return {"workload": f"{grid}^3 cells x {ppc} ppc/species, {steps} steps, dipole x0.5 / x1 / x2, "
                        "FP32 (tiled) against FP64 (slot order) from the same seed", "runs": out}


def combine_over_ranks(ms: float, pushed: float, dist=None, device: str = "cuda"):
    """Whole-job numbers of the replicas: the slowest rank's time and the
    particle pushes of all ranks (max and sum over the process group)."""
    if dist is None:
        return ms, float(pushed)
    import torch

    tmax = torch.tensor([ms], dtype=torch.float64, device=device)
    tsum = torch.tensor([float(pushed)], dtype=torch.float64, device=device)
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(tsum[0])


def run_poisson(reps: int = 10):
    """Poisson cleaning (pic_poisson_clean: renew_phi3 + sr_phi + sr_e) on the
    bench grid, FP32, timed with CUDA events on the context's stream. FLOPs:
    the six sine-transform GEMMs, 2 * 2 * N * (nx + ny + nz) for N interior
    cells (forward and inverse along each axis)."""
    import torch

    from plasmasim_b200 import Pic3D

    cfg = make_config(32, 0)
    cfg.absorb_grid3 = 0
    P = Pic3D(cfg)
    P.init_grid()
    P.init_particle_flat()
    P.fdtd(0)
    P.step(2)
    P.poisson_clean()
    P.synchronize()
    stream = torch.cuda.ExternalStream(P.stream_handle())
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(reps):
        P.poisson_clean()
    stop.record(stream)
    stop.synchronize()
    ms = start.elapsed_time(stop) / reps
    P.close()
    n = NX * NY * NZ
    flop = 4.0 * n * (NX + NY + NZ)
    # nominal FP32 CUDA-core peak: 148 SMs x 128 FMA/clock x 2 x 1.965 GHz
    fp32_peak = 148 * 128 * 2 * 1.965e9
    return {"workload": f"{NX}x{NY}x{NZ} interior cells, FP32, Absorb_grid3 = 0", "ms": ms,
            "gflop": flop / 1e9, "tflops": flop / ms / 1e9, "fp32_simt_peak_tflops": fp32_peak / 1e12,
            "frac_of_fp32_simt_peak": flop / (ms * 1e-3) / fp32_peak}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--grid", type=int, default=128,
                    help="cells per axis (128 for the benchmark; smaller cases for profiling)")
    ap.add_argument("--ppc", type=int, default=64, help="particles per cell per species")
    ap.add_argument("--no-batch2d", action="store_true", help="skip the batched 2D runs")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint measurement")
    ap.add_argument("--no-poisson", action="store_true", help="skip the Poisson cleaning measurement")
    ap.add_argument("--no-thrust", action="store_true", help="skip the FP32-vs-FP64 thrust error leg")
    ap.add_argument("--configs2", action="store_true",
                    help="only the 256^3 x 32 ppc FP32-vs-FP64 comparison at three dipole moments (minutes)")
    ap.add_argument("--configs2-steps", type=int, default=100)
    ap.add_argument("--thrust-steps", type=int, default=200, help="steps of the thrust error leg")
    ap.add_argument("--runs2d", type=int, default=256, help="runs of the batched 2D workload")
    ap.add_argument("--adjoint-steps", type=int, default=200, help="steps of the adjoint measurement")
    ap.add_argument("--adjoint-every", type=int, default=20, help="its checkpoint interval")
    args = ap.parse_args()
    global NX, NY, NZ, PPC
    NX = NY = NZ = args.grid
    PPC = args.ppc

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        name = "cube128_t64"
        if (NX, NY, NZ, PPC) != (128, 128, 128, 64) or not ensure_reference_lib(name):
            print(json.dumps({"impl": "reference", "unavailable": "compiled reference library missing "
                                                                   "or not built for this grid"}))
            return
        threads = min(host_threads(), 64)
        r = reference_threaded(name, [(threads, args.steps)], min(args.warmup, 3))[0]
        value = r["psteps"] / r["secs"]
        cfg = {"workload": f"3D PIC solar wind + dipole (normalized units), {NX}x{NY}x{NZ} cells x "
                           f"{PPC} particles/cell/species, sort every 20, refill every 5",
               "grid": [NX, NY, NZ], "ppc_per_species": PPC, "particles": r["particles"],
               "sample": f"the full workload; {r['steps']} timed fdtd loop bodies after "
                         f"{min(args.warmup, 3)} untimed ones (init {r['init_s']:.0f} s, untimed)",
               "threads": threads, "particle_lists": r["lists"]}
        print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
                          "n_gpus": args.gpus, "steps": r["steps"], "warmup": min(args.warmup, 3),
                          "ms_per_step": r["secs"] / max(r["steps"], 1) * 1e3,
                          "higher_is_better": True, "scaling": "weak", "dtype": "f64",
                          "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                                           "kind": "reference", "sample": cfg["sample"]},
                          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    if args.configs2:
        import torch

        torch.cuda.set_device(0)
        print(json.dumps({"configs2": run_configs2(args.configs2_steps)}))
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    else:
        torch.cuda.set_device(0)
    from plasmasim_b200 import build as pbuild

    if not os.path.isfile(pbuild.LIB):
        pbuild.build()

    seed = 1000 * rank
    P, out = run_gpu(32, args.steps, args.warmup, seed, dist, clocks_index=local)
    ms = out["ms"]
    pushed = out["pushed"]
    ms_max, pushed_all = combine_over_ranks(ms, pushed, dist)
    value = pushed_all / (ms_max / 1e3)
    cells = (NX + 4) * (NY + 4) * (NZ + 4)
    nsp = pushed / max(args.steps, 1) / 2
    ach, bytes_launch, s_launch = roofline(out, nsp, cells, 4)
    peak, peak_kind = measured_peaks()
    step_bytes = pushed / max(args.steps, 1) * 56 + NX * NY * NZ * 200

    e2e = None
    if not args.no_e2e and world == 1:
        try:
            v, h2d, d2h = run_e2e(P, args.steps)
            e2e = {"value": v, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
        except Exception as exc:  # reported, not hidden
            log("e2e failed:", exc)
            e2e = {"value": None, "unit": UNIT, "error": str(exc)[:200]}
    P.close()
    del P

    fp64 = None
    if not args.no_fp64 and world == 1:
        P64, o64 = run_gpu(64, args.steps, args.warmup, seed, None, clocks_index=local)
        P64.close()
        v64 = o64["pushed"] / (o64["ms"] / 1e3)
        fp64 = {"value": v64, "ms_per_step": o64["ms"] / args.steps, "fp32_over_fp64": value / v64,
                "phase_ms": o64["phase_ms"]}

    batch2d = None
    if not args.no_batch2d and world == 1:
        try:
            batch2d = run_batch2d(args.runs2d, args.steps, args.warmup)
            if not args.no_cpu:
                batch2d["cpu_baseline"] = batch2d_cpu_sample()
        except Exception as exc:  # reported, not hidden
            log("batch2d failed:", exc)
            batch2d = {"error": str(exc)[:200]}

    adjoint = None
    if not args.no_adjoint and world == 1:
        try:
            adjoint = run_adjoint(args.adjoint_steps, args.adjoint_every)
        except Exception as exc:
            log("adjoint failed:", exc)
            adjoint = {"error": str(exc)[:200]}

    poisson = None
    if not args.no_poisson and world == 1:
        try:
            poisson = run_poisson()
            poisson["over_step"] = poisson["ms"] / (ms_max / args.steps)
        except Exception as exc:
            log("poisson failed:", exc)
            poisson = {"error": str(exc)[:200]}

    thrust = None
    if not args.no_thrust and world == 1:
        try:
            thrust = run_thrust_error(args.thrust_steps)
        except Exception as exc:
            log("thrust error leg failed:", exc)
            thrust = {"error": str(exc)[:200]}

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        if ensure_reference_lib("quarter128_t64"):
            threads = min(host_threads(), 64)
            r, r1 = reference_threaded("quarter128_t64", [(threads, 2), (1, 1)], 1, budget_s=30.0)
            cpu = {"value": r["psteps"] / r["secs"], "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"the reference with OpenMP on a quarter of the workload's volume, 64x64x128 cells x "
                             f"64 ppc/species ({r['particles']} particles), {r['steps']} fdtd loop bodies",
                   "one_core": {"value": r1["psteps"] / r1["secs"], "cores": 1,
                                "sample": f"the same, one thread (the reference as shipped, active_thread 1), "
                                          f"{r1['steps']} loop body"}}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "compiled reference library missing"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"3D PIC solar wind + dipole (normalized units), {NX}x{NY}x{NZ} cells x "
                                   f"{PPC} particles/cell/species, sort every 20, refill every 5",
                       "grid": [NX, NY, NZ], "ppc_per_species": PPC,
                       "particles": int(pushed / max(args.steps, 1)),
                       "l2": f"inputs larger than L2 ({28 * pushed / max(args.steps, 1) / 1e9:.2f} GB of "
                             "particle state per step)",
                       "parallelism": f"replicas{world}"},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak,
                         "traffic": PUSH_TRAFFIC_PER_PARTICLE * nsp if PPC == 64 else None,
                         "kernel": "push_tiled_kernel<float,1> (push phase, with its tail push_kernel)",
                         "peak_kind": peak_kind, "bytes_per_launch": bytes_launch,
                         "ms_per_launch": s_launch * 1e3},
            "step_roofline": {"bytes_per_step": step_bytes, "achieved": step_bytes / (ms_max / args.steps) / 1e6,
                              "frac": step_bytes / (ms_max / args.steps) / 1e6 / peak, "unit": "GB/s",
                              "bytes": "particles x 56 + cells x 200 (FP32)"},
            "phase_ms_per_step": {k: v / args.steps for k, v in out["phase_ms"].items()},
            "clocks": out["clocks"], "gpu_launches": out["launches"],
            "device_errors": out["errors"], "e2e": e2e, "fp64": fp64, "cpu_baseline": cpu,
            "batch2d": batch2d, "adjoint": adjoint, "poisson": poisson,
            "thrust_rel_err": thrust.get("thrust_rel_err") if thrust else None, "thrust": thrust,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
