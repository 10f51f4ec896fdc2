"""Benchmark of the per-timestep MHD hot path (one StepOnce = one step).

Workloads (--workload):

* c2: 6 blocks of 96 x 48 x 48 cells (1,327,104 cells), radial
  cells log-spaced over r in [1, 8], a Solid_Surface inner wall and a
  Farfield outer boundary, inflow rho = 1, v = (-8, 0, 0),
  B = (0, 0.5, 0.5)/sqrt(2), p = 0.05 with seeded 1e-3 noise, and the
  implicit resistive step (peak resistivity 1e-3, GMRES to rtol 1e-10)
  every step; the six blocks tile a curved slab (3 x 2 transverse tiles,
  periodic across the tiles) because the reference's halo exchange cannot
  run a cubed-sphere layout.  FP64.
* c1: the plain FP64 64^3 periodic curvilinear block (ideal MHD).
* c3 / c4: Hall MHD: 6 blocks of 128 x 64 x 64 cells (3,145,728 cells) on
  the C2 slab layout and inflow, ideal MHD plus the implicit Hall step
  (Newton rtol 1e-10, GMRES to 1e-5 per Newton step) after the explicit
  part of every step; FP64 (c3) or mixed precision (c4).
* c5: a parameter sweep of 48 independent runs in one batch context, each
  one slab block of Nr x Nt x Nt cells (Nr in 32..128, Nt in 24..96),
  inflow speed 4..12 and IMF clock angle 0..180 degrees drawn from
  MT19937_64(5) (beta1_b200.case.sweep_cases; 14.7 M cells in all), ideal
  MHD, each run with its own time step; mixed precision unless --precision
  fp64.  Host geometry is built by a spawned process pool.
* c5s (default): the same sweep (same draws) with every run a single-block
  spherical shell of Nr x Nt x Nph cells (Nph = Nt rounded up to even) with
  Pole patches at both ends of theta (case.sweep_cases(grid="shell")),
  15.3 M cells in all; geometry built on the device.  The line's value is
  the mixed-precision form; the FP64 form is timed on the same runs in the
  same job, and after the same steps every field of the mixed form is
  compared with the FP64 form's (relative L2 over all runs) together with
  max |div B| dx / |B|.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload c5s|c2|c1|c5|c3|c4]
                    [--precision fp64|mixed]

Multi-GPU (torchrun): the path does not shard, so N ranks run N independent
replicas; value = all cells updated by all ranks / max-over-ranks time.

Rank 0 prints one JSON line.  Inputs are seeded synthetic states in the
reference's restart format; the device working set (several GB) is larger
than the 126 MB L2, so no L2 flush is inserted between steps.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_lunar")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")

# Algorithmic bytes per cell of each kernel (FP64, every array the kernel
# must read or write counted once per cell, 8 bytes per element).
ALGO_BYTES_PER_CELL = {
    # fluid RHS: rho 1, PV 4, RhoE 1, Csound 1, JD 9, face area 3, Jac 1, B_cell 3, J_cell 3 read, RHS_H 5
    # written; with the contravariant velocities: U_plus 3 read, U_contra 3 written
    "k_fluid_ucontra": 37 * 8,
    "k_fluid_rhs": 31 * 8,
    # JD 9, Jac 1, U_plus 3 read; U_contra 3 written
    "k_ucontra": 16 * 8,
    # B 3, Badd 3, U_contra 3 read; Eface 9 written
    "k_eface": 18 * 8,
    # Eface 6, B 3, U_contra 3 read; E 3 written
    "k_eedge": 15 * 8,
    # E 3 read, RHS_B 3 written, B 3 read + written
    "k_curl_e2f": 12 * 8,
    # U 5 read + written, RHS_H 5 read
    "k_update_u": 15 * 8,
    # B_cell + J edges: B 3, Badd 3, W_B 18, beta 3, alpha 3 read; B_cell 3, Bind_cell 3, J 3 written
    "k_bcell_jedge": 39 * 8,
    # PV / U_plus / CFL with J_cell: U 5, Jac 1, B_cell 3, face area + normal 12, J 3, W_J 36 read;
    # PV 5, U_plus 3, Csound 1, RhoE 1, J_cell 3 written
    "k_pv_uplus_dt": 73 * 8,
    # Hall EMF: B_cell 3, J_cell 3, rho 1 read; E_hall_cell 3, beta 1 written (per cell) / E_hall_cell 3,
    # beta 1, B 3, face area 3, dl 3, dr 9 read; E_hall 3 written (per edge triple)
    "k_hall_cell": 11 * 8,
    "k_hall_edge": 25 * 8,
    # mixed form: FP32 face states rho, u, v, w, p, RhoE, c 7 and face area 3 read; FP64 JD 9, Jac 1,
    # U_plus 3, rho 1, u/v/w 3, B_cell 3, J_cell 3 read, RHS_H 5 and U_contra 3 written
    "k_fluid_mixed": 10 * 4 + 31 * 8,
}
ALGO_BYTES_PER_CELL.update({
    # B_cell alone (the Pole path's unfused derived pass): B 3, Badd 3, W_B 18 read; B_cell 3, Bind_cell 3 written
    "k_bcell": 30 * 8,
    # J edges: B 3, beta 3, alpha 3 read; J 3 written
    "k_jedge": 12 * 8,
})
# The flux + CT group (calc_PV, Scheme_U_ with its J x B source, the face and
# edge EMF, the curl and both Euler updates): reads U 5, B_face 3, Badd 3,
# JD 9, Jac 1, B_cell 3, J_cell 3; writes U 5, B_face 3.  FP64 35 x 8 =
# 280 B per cell; mixed (JD, Jac, B_cell, J_cell as FP32 copies) 16 x 4 +
# 19 x 8 = 216 B per cell.
FLUX_CT_GROUP = ("k_fluid_ucontra", "k_fluid_mixed", "k_eface", "k_eedge", "k_curl_e2f", "k_update_u")
FLUX_CT_BYTES = {False: 280, True: 216}
WHOLE_GRID_KERNELS = {"k_pv_uplus_dt", "k_fluid_ucontra", "k_fluid_mixed", "k_bcell_jedge", "k_eface", "k_eedge",
                      "k_update_u", "k_hall_cell", "k_hall_edge", "k_bcell", "k_jedge"}
# The mixed form's kernels where they differ: the PV pass reads the 36 J_cell
# weights and the face areas + normals (12) as FP32 copies and writes U_plus
# 3, J_cell 3 and the 7 FP32 face states (PV_H and the FP64 face states are
# left to read-out): U 5, Jac 1, B_cell 3, J 3 read as FP64 plus 48 FP32
# values; 6 FP64 and 7 FP32 written.  The B_cell passes read their 18 weights
# as FP32.
ALGO_BYTES_MIXED = {"k_pv_uplus_dt": 12 * 8 + 48 * 4 + 6 * 8 + 7 * 4,
                    "k_bcell": 12 * 8 + 18 * 4,
                    "k_bcell_jedge": 21 * 8 + 18 * 4}

# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per launch of
# the dominant kernel, from one ncu capture of a smaller case of the same
# workload, scaled by the cell count to a full launch (the kernels' traffic
# grows with the cells they cover):
# * C2 at half the cells per direction (165,888 cells: 114.26 MB read +
#   10.32 MB written) to the full C2 slab (1,327,104 cells);
# * the shell sweep's first 6 runs (2,269,318 cells; k_fluid_mixed at 3 CTAs
#   per SM 602.60 MB read + 145.68 MB written, k_pv_uplus_dt 763.50 + 185.09
#   MB) to all 48 runs (14,879,028 cells)
_SWEEP_SCALE = 14879028.0 / 2269318.0
NCU_TRAFFIC_BYTES = {
    ("k_pv_uplus_dt", "c2_slab6x96x48x48_implicit_resistive_fp64"): (114.25536e6 + 10.321408e6) * 8.0,
    ("k_fluid_mixed", "c5s_sweep48_shell_runs_mixed"): (602.596096e6 + 145.683968e6) * _SWEEP_SCALE,
    ("k_pv_uplus_dt", "c5s_sweep48_shell_runs_mixed"): (763.501568e6 + 185.093888e6) * _SWEEP_SCALE,
}


def sample_clocks(stop: threading.Event, out: list, gpu_id: str):
    """nvidia-smi clock / throttle samples of this rank's GPU every 100 ms."""
    cmd = ["nvidia-smi", "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
           "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
           "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-i", gpu_id]
    while not stop.is_set():
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=5)
            if r.returncode == 0 and r.stdout.strip():
                out.append(r.stdout.strip().splitlines()[0])
        except Exception:
            pass
        stop.wait(0.1)


def summarize_clocks(lines):
    if not lines:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    sm, smax, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        p = [x.strip() for x in ln.split(",")]
        try:
            sm.append(float(p[0]))
            smax.append(float(p[1]))
        except ValueError:
            continue
        for nm, v in zip(names, p[3:7]):
            if v.lower() == "active":
                reasons.add(nm)
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(PEAKS) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


WORKLOADS = {
    "c2": dict(name="c2_slab6x96x48x48_implicit_resistive_fp64", ref_steps=4, ref_rss_gb=12.0),
    "c1": dict(name="c1_periodic_64cubed_fp64", ref_steps=40, ref_rss_gb=1.0),
    "c5": dict(name="c5_sweep48_slab_runs_mixed", ref_steps=2, ref_rss_gb=4.0),
    "c5s": dict(name="c5s_sweep48_shell_runs_mixed", ref_steps=2, ref_rss_gb=4.0),
    "c3": dict(name="c3_slab6x128x64x64_hall_implicit_fp64", ref_steps=1, ref_rss_gb=28.0),
    "c4": dict(name="c4_slab6x128x64x64_hall_implicit_mixed", ref_steps=1, ref_rss_gb=28.0),
}
SWEEP_RUNS = 48
SWEEP_GRID = {"c5": ("slab", "tiled"), "c5s": ("shell", "shell")}  # sweep workload -> (grid, topology)
HALL_SAMPLE = ("the full workload (6 blocks of 128 x 64 x 64 cells), StepOnce as compiled with the implicit Hall "
               "solve (SolveOneStep at the step's dt, Newton rtol 1e-10, then calc_Bcell, before the closing syncs "
               "and derived fields)")



def max_over_ranks(ms: float, device) -> float:
    """The largest of every rank's time (the job's time), all-reduced over
    the process group when there is one (NCCL on the GPUs, gloo in tests)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, cells: int, steps: int, ms_max: float) -> float:
    """Whole-job cell-updates/s of `world` replicas that each advanced
    `cells` cells `steps` times, over the slowest rank's time."""
    return world * cells * steps / (ms_max / 1000.0)


def workload_name(name, mixed):
    base = name.rsplit("_", 1)[0]
    return base + ("_mixed" if mixed else "_fp64")


def build_case(workload, n=64, size=(96, 48), hall_size=(128, 64)):
    """(spec, restart state, topology, interior cells) of a workload; size:
    (radial, transverse) cells per block of the c2 slab, hall_size the same
    for c3 / c4."""
    from beta1_b200 import case
    if workload == "c1":
        spec = case.periodic_box_case((n, n, n))
        return spec, case.initial_state(spec), "periodic", n ** 3
    if workload in ("c3", "c4"):
        spec = case.slab_case(hall_size[0], (hall_size[1], hall_size[1]), (3, 2))
        cells = sum(b.ncell[0] * b.ncell[1] * b.ncell[2] for b in spec.blocks)
        return spec, case.inflow_state(spec), "tiled", cells
    sc = case.ref_scales()
    spec = case.slab_case(size[0], (size[1], size[1]), (3, 2), is_Lunar_resistance=1, use_implicit_lunar_resistance=1,
                          eta_max_lunar=1e-3 * case.MU0 * sc["U"] * sc["L_ref"], implicit_resistive_ksp_rtol=1e-10)
    cells = sum(b.ncell[0] * b.ncell[1] * b.ncell[2] for b in spec.blocks)
    return spec, case.inflow_state(spec), "tiled", cells


def mem_available_gb():
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable:"):
                return int(ln.split()[1]) / 1e6
    except OSError:
        pass
    return 16.0


def ref_warmup(workload, warmup):
    """untimed reference steps before the timed ones: the bench's warm-up,
    at most 3, none for the Hall workloads (one step of the reference takes
    minutes there)"""
    return 0 if workload in ("c3", "c4") else max(0, min(int(warmup), 3))


def cpu_reference(workload, n, steps, nproc, integrator="euler", warmup=0):
    """Times the reference's own StepOnce loop (oracle/_ref/ref_lunar, built
    from the reference sources) on `nproc` concurrent single-threaded
    processes (bounded by host memory), each on the same bounded sample,
    after `warmup` untimed steps; returns aggregate cell-updates/s, the
    per-process figures and the process count."""
    from beta1_b200 import case, rst
    if not os.path.exists(REF_BIN):
        return None
    nproc = max(1, min(nproc, int(0.6 * mem_available_gb() / WORKLOADS[workload]["ref_rss_gb"])))
    command = "timerk2" if integrator == "rk2" else "time"
    spec, st, _, _ = build_case(workload, n)
    if workload in ("c3", "c4"):
        # the step with the implicit Hall solve, at the workload's full size
        command = "timehall"
    d = tempfile.mkdtemp(prefix="b1ref_")
    try:
        case.write_case(d, spec)
        rst.write(os.path.join(d, "init.rst"), st)
        procs = []
        for p in range(nproc):
            wd = os.path.join(d, "r%d" % p)
            os.makedirs(wd)
            for entry in os.listdir(d):
                if entry not in ("init.rst",) and not entry.startswith("r"):
                    os.symlink(os.path.join(d, entry), os.path.join(wd, entry))
            procs.append(subprocess.Popen([REF_BIN, command, os.path.join(d, "init.rst"), str(steps), str(warmup)],
                                          cwd=wd,
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
        vals = []
        for pr in procs:
            out, _ = pr.communicate()
            lines = [ln for ln in out.strip().splitlines() if ln.startswith("{")]
            if pr.returncode != 0 or not lines:
                return None
            vals.append(json.loads(lines[-1]))
        agg = sum(v["cell_updates_per_s"] for v in vals)
        return agg, vals, nproc
    finally:
        shutil.rmtree(d, ignore_errors=True)


def cpu_reference_sweep(steps, nproc, nruns=SWEEP_RUNS, grid="slab", warmup=0):
    """The reference's StepOnce loop on a sample of the sweep's runs: the
    first `nproc` runs (bounded by host cores and memory), one
    single-threaded process per run, concurrently, each after `warmup`
    untimed steps; returns aggregate cell-updates/s, the per-process figures
    and the process count."""
    from beta1_b200 import case, rst
    if not os.path.exists(REF_BIN):
        return None
    runs = case.sweep_cases(nruns, grid=grid)
    nproc = max(1, min(nproc, len(runs), int(0.6 * mem_available_gb() / WORKLOADS["c5"]["ref_rss_gb"])))
    d = tempfile.mkdtemp(prefix="b1sweep_")
    try:
        procs = []
        for r in range(nproc):
            spec = runs[r][0]
            wd = os.path.join(d, "r%d" % r)
            os.makedirs(wd)
            case.write_case(wd, spec)
            rst.write(os.path.join(wd, "init.rst"), case.inflow_state(spec, seed=SWEEP_SEED0 + r))
            procs.append(subprocess.Popen([REF_BIN, "time", os.path.join(wd, "init.rst"), str(steps), str(warmup)],
                                          cwd=wd,
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
        vals = []
        for pr in procs:
            out, _ = pr.communicate()
            lines = [ln for ln in out.strip().splitlines() if ln.startswith("{")]
            if pr.returncode != 0 or not lines:
                return None
            vals.append(json.loads(lines[-1]))
        return sum(v["cell_updates_per_s"] for v in vals), vals, nproc
    finally:
        shutil.rmtree(d, ignore_errors=True)


SWEEP_SEED0 = 5000


def sweep_host_setup(workload="c5", nruns=SWEEP_RUNS, geometry_on="host", use_runs=None):
    """Host set-up of every run of the sweep (node mesh, sync tables and,
    unless the device builds it, the geometry) from a spawned process pool
    bounded by cores and memory; returns (runs, [host set-up per run])."""
    import multiprocessing as mp
    from beta1_b200 import case, solver
    grid, topo = SWEEP_GRID[workload]
    runs = case.sweep_cases(nruns, grid=grid)[:use_runs]
    nproc = max(1, min(len(runs), os.cpu_count() or 1, 16, int(mem_available_gb() / 8.0)))
    with mp.get_context("spawn").Pool(nproc) as pool:
        host = pool.map(solver.host_setup_run, [(spec, topo, geometry_on) for spec, _ in runs])
    return runs, host


def build_sweep(precision, runs, host, workload="c5"):
    """The sweep batch from its host set-up, every run's seeded inflow state
    loaded."""
    from beta1_b200 import case, solver
    topo = SWEEP_GRID[workload][1]
    bt = solver.Batch([(spec, topo) for spec, _ in runs], precision=precision, host=iter(host))
    bt.load_states([case.inflow_state(spec, seed=SWEEP_SEED0 + r) for r, (spec, _) in enumerate(runs)])
    return bt, sum(bt.cells)


ERROR_FIELDS = ["U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "B_cell", "J_cell"]


def _inner(ctx, name, b, a):
    """the inner points of a downloaded field (cells [0, n), faces [0, n])"""
    inf = ctx.field_info(name, b)
    blk = ctx.ncells[b]
    hi = [n + (1 if name == "B_" + ax else 0) for n, ax in zip(blk, ("xi", "eta", "zeta"))]
    return a[tuple(slice(-lo, -lo + h) for lo, h in zip(inf["lo"], hi))]


def error_report(test, ref, nblocks):
    """Relative L2 over every block's inner points of each field of `test`
    against `ref` (two contexts advanced the same steps from the same state),
    and max |div B| dx / |B| of `test` (dx the cube root of the cell
    volume)."""
    from beta1_b200 import mhd
    test.stage(mhd.STAGE_DIVB)
    num = {f: 0.0 for f in ERROR_FIELDS}
    den = {f: 0.0 for f in ERROR_FIELDS}
    divb = 0.0
    for b in range(nblocks):
        for f in ERROR_FIELDS:
            a = _inner(test, f, b, test.download(f, b))
            r = _inner(ref, f, b, ref.download(f, b))
            num[f] += float(np.sum((a - r) ** 2))
            den[f] += float(np.sum(r ** 2))
        dx = np.cbrt(np.abs(_inner(test, "Jac", b, test.download("Jac", b))[..., 0]))
        bmag = np.linalg.norm(_inner(test, "B_cell", b, test.download("B_cell", b)), axis=-1)
        dv = np.abs(_inner(test, "divB", b, test.download("divB", b))[..., 0])
        divb = max(divb, float(np.max(dv * dx / bmag)))
    rel = {f: (float(np.sqrt(num[f] / den[f])) if den[f] > 0 else float(np.sqrt(num[f]))) for f in ERROR_FIELDS}
    return rel, divb


def timed_steps(ctx, steps, warmup, world, local, stream):
    """W warm-up steps, then exactly `steps` steps between a barrier and a
    device synchronisation on both sides, timed with CUDA events on the
    context's stream while nvidia-smi samples the clocks.  Returns (ms,
    kernel launches, clock samples)."""
    import torch
    import torch.distributed as dist
    ctx.step(warmup)
    clocks, stop = [], threading.Event()
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        gpu_id = str(local)
    th = threading.Thread(target=sample_clocks, args=(stop, clocks, gpu_id), daemon=True)
    th.start()
    time.sleep(0.25)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = ctx.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    stop.set()
    th.join()
    return e0.elapsed_time(e1), ctx.launches() - l0, clocks


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]
    steps = min(args.steps, args.ref_steps or wl["ref_steps"])
    warm = ref_warmup(args.workload, args.warmup)
    if args.workload in SWEEP_GRID:
        res = cpu_reference_sweep(steps, os.cpu_count() or 1, grid=SWEEP_GRID[args.workload][0], warmup=warm)
    else:
        res = cpu_reference(args.workload, args.n, steps, os.cpu_count() or 1, args.integrator, warmup=warm)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_lunar not built or failed"}))
        return 0
    agg, vals, nproc = res
    cells = vals[0]["cells"] if args.workload not in SWEEP_GRID else sum(v["cells"] for v in vals)
    if args.workload in SWEEP_GRID:
        sample = "%s: the first %d runs of the sweep, one single-threaded process each, %d StepOnce per " \
                 "process after %d untimed, concurrently (bounded by host cores and memory)" \
                 % (wl["name"], nproc, steps, warm)
    elif args.workload in ("c3", "c4"):
        sample = "%s: %s; %d steps per process (no untimed step: one takes minutes), %d concurrent " \
                 "single-threaded processes (bounded by host cores and memory)" % (wl["name"], HALL_SAMPLE, steps,
                                                                                    nproc)
    else:
        sample = "%s: %d %s per process after %d untimed, %d concurrent single-threaded processes (bounded by " \
                 "host cores and memory)" % (wl["name"], steps,
                                             "SSP-RK2 steps" if args.integrator == "rk2" else "StepOnce", warm, nproc)
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": agg, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm,
        "ms_per_step": 1000.0 * max(v["seconds"] / v["steps"] for v in vals), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["name"], "cells": cells},
        "cpu_baseline": {"value": agg, "unit": "cell-updates/s", "cores": nproc, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": agg, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 200 for c2, 4000 for c1)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c5s", choices=list(WORKLOADS))
    ap.add_argument("--n", type=int, default=64, help="cells per direction of the c1 periodic block")
    ap.add_argument("--c2-size", default="96x48", help="radial x transverse cells per c2 block (profiling runs "
                                                         "use a smaller case; the bench line is quoted on 96x48)")
    ap.add_argument("--hall-size", default="128x64", help="radial x transverse cells per c3 / c4 block (profiling "
                                                            "runs use a smaller case; the bench line is quoted on "
                                                            "128x64)")
    ap.add_argument("--ref-steps", type=int, default=None, help="StepOnce per reference CPU sample")
    ap.add_argument("--e2e-iters", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep every kernel's default variant")
    ap.add_argument("--tune", default=None,
                    help="kernel=value,... variants applied with mhd_set_tune instead of autotuning (profiling)")
    ap.add_argument("--geometry", default=None, choices=["host", "device"],
                    help="geometry fields built on the host and uploaded, or built on the device from the node "
                         "meshes (mhd_build_geometry); same values (default: device for the sweeps, host otherwise)")
    ap.add_argument("--integrator", default=None, choices=["euler", "rk2"],
                    help="euler: the reference's StepOnce; rk2: SSP-RK2 of two of its Euler stages at one dt "
                         "(default: rk2 for c1, euler otherwise)")
    ap.add_argument("--sweep-runs", type=int, default=SWEEP_RUNS,
                    help="sweeps: the first N runs of the 48 (profiling captures use a few; the bench line is "
                         "quoted on all 48)")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="sweeps in mixed precision: skip timing the FP64 form on the same runs")
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="fp64, or FP32 face fluxes with FP64 CT / state / residuals (default: mixed for c5, c5s "
                         "and c4, fp64 otherwise)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.steps is None:
        args.steps = {"c2": 200, "c1": 4000, "c5": 100, "c5s": 100, "c3": 10, "c4": 10}[args.workload]
    if args.precision is None:
        args.precision = "mixed" if args.workload in ("c5", "c5s", "c4") else "fp64"
    if args.integrator is None:
        args.integrator = "rk2" if args.workload == "c1" else "euler"

    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from beta1_b200 import mhd, solver

    wl = WORKLOADS[args.workload]
    mixed = args.precision == "mixed"
    prec = mhd.PREC_MIXED if mixed else mhd.PREC_FP64
    sweep = args.workload in SWEEP_GRID
    geometry_on = args.geometry or ("device" if sweep else "host")
    t_setup = time.time()
    fp64_cmp = None
    if sweep:
        runs, host = sweep_host_setup(args.workload, geometry_on=geometry_on, use_runs=args.sweep_runs)
        s, cells = build_sweep(prec, runs, host, args.workload)
        spec = None
        nblocks = len(runs)
        if mixed and not args.no_fp64_compare:
            fp64_cmp, _ = build_sweep(mhd.PREC_FP64, runs, host, args.workload)
        del host
    else:
        c2size = tuple(int(v) for v in args.c2_size.split("x"))
        hallsize = tuple(int(v) for v in args.hall_size.split("x"))
        spec, st, topology, cells = build_case(args.workload, args.n, c2size, hallsize)
        s = solver.Solver(spec, topology=topology, precision=prec, geometry_on=geometry_on)
        if args.workload in ("c3", "c4"):
            # bounded: at most 10 Newton steps of at most 200 GMRES iterations per time step
            s.install_hall_implicit(topology, rtol=1e-10, atol=1e-50, maxit=10, ksp_rtol=1e-5, ksp_maxit=200)
        s.load_state(st)
        nblocks = len(spec.blocks)
    ctx = s.ctx
    if args.integrator == "rk2":
        for c in ([ctx] + ([fp64_cmp.ctx] if fp64_cmp is not None else [])):
            c.set_integrator(mhd.INTEGRATOR_SSPRK2)
    setup_s = time.time() - t_setup
    # register / occupancy variant of each hot kernel, timed on this state
    if args.tune:
        tuned = {kv.split("=")[0]: int(kv.split("=")[1]) for kv in args.tune.split(",")}
        ctx.set_tune(tuned)
    else:
        tuned = ctx.autotune(reps=10) if not args.no_autotune else None
    stream = torch.cuda.ExternalStream(ctx.stream())
    ctx_bytes = sum(ctx.field_info(f, b)["ncomp"] * int(np.prod([h - l for l, h in zip(
        ctx.field_info(f, b)["lo"], ctx.field_info(f, b)["hi"])])) * 8 for f in ("U_H", "PV_H", "JDxi", "JDet",
                                                                                 "JDze", "Jcell_from_Jedge_w",
                                                                                 "Bcell_from_Bface_w")
        for b in range(nblocks))
    res_stats = None

    # the FP64 form on the same runs, same steps, for the speed ratio and the
    # error report of the mixed form
    fp64_line = None
    if fp64_cmp is not None:
        ctx64 = fp64_cmp.ctx
        tuned64 = ctx64.autotune(reps=10) if not (args.no_autotune or args.tune) else None
        ms64, _, clocks64 = timed_steps(ctx64, args.steps, args.warmup, world, local,
                                        torch.cuda.ExternalStream(ctx64.stream()))
        ms64 = max_over_ranks(ms64, "cuda")
        fp64_line = {"value": replica_throughput(world, cells, args.steps, ms64), "ms_per_step": ms64 / args.steps,
                     "autotune_min_ctas_per_sm": tuned64, "clocks": summarize_clocks(clocks64)}

    ms, launches, clocks = timed_steps(ctx, args.steps, args.warmup, world, local, stream)
    if spec is not None and spec.params.get("is_Lunar_resistance", 0):
        rs = ctx.resistive_stats()
        res_stats = {"krylov_its_last_step": rs["its"], "rnorm": rs["rnorm"], "bnorm": rs["bnorm"],
                     "reason": rs["reason"], "unknowns": int(len(s.resistive_dofs[0])), "rtol": float(spec.params["implicit_resistive_ksp_rtol"])}
    hall_stats = None
    if args.workload in ("c3", "c4"):
        hs = ctx.hall_stats()
        hall_stats = {"newton_its_last_step": hs["its"], "gmres_its_last_step": hs["linear_its"],
                      "fnorm": hs["fnorm"], "fnorm0": hs["fnorm0"], "reason": hs["reason"],
                      "residual_evaluations_at_least": 1 + hs["its"] + hs["linear_its"]}
    ms_max = max_over_ranks(ms, "cuda")
    value = replica_throughput(world, cells, args.steps, ms_max)
    if fp64_cmp is not None:
        rel, divb = error_report(ctx, fp64_cmp.ctx, nblocks)
        t_m = [ctx.run_time(r)[1] for r in range(ctx.nruns)]
        t_d = [fp64_cmp.ctx.run_time(r)[1] for r in range(ctx.nruns)]
        fp64_line.update({
            "mixed_over_fp64": value / fp64_line["value"],
            "steps_compared": args.warmup + args.steps,
            "mixed_rel_l2_vs_fp64": {f: float("%.3e" % e) for f, e in rel.items()},
            "mixed_max_rel_l2": max(rel.values()),
            "mixed_max_divb_dx_over_b": divb,
            "time_rel_diff": max(abs(a - b) / b for a, b in zip(t_m, t_d)),
            "bounds": {"rel_l2": 1e-5, "divb_dx_over_b": 1e-12}})
        # the FP64 form's per-kernel durations (after the comparison: these steps advance it)
        prof64 = {}
        for _ in range(3):
            for name, t in fp64_cmp.ctx.profile_step():
                prof64[name] = prof64.get(name, 0.0) + t / 3.0
        fp64_line["kernels_ms_per_step"] = {k: round(v, 5) for k, v in sorted(prof64.items(), key=lambda kv: -kv[1])}
        fp64_cmp.ctx.close()

    # per-kernel durations: eager steps with an event pair around every launch
    prof = {}
    for _ in range(5):
        for name, t in ctx.profile_step():
            prof.setdefault(name, []).append(t)
    per_step = {k: sum(v) / 5.0 for k, v in prof.items()}
    total = sum(per_step.values())
    launches_of = {k: len(v) / 5.0 for k, v in prof.items()}
    # the dominant kernel by time over every kernel of the step
    dominant = max(per_step, key=lambda k: per_step[k])
    avg_launch_ms = per_step[dominant] / launches_of[dominant]
    if dominant == "k_gmres_resist" and res_stats is not None:
        # per solve: 18 doubles per unknown triple per matvec (its + one per
        # restart cycle) and (2k + 4) doubles per unknown in Arnoldi step k
        n, its = res_stats["unknowns"], max(1, res_stats["krylov_its_last_step"])
        bytes_per_launch = (its + 1) * 18 * 8 * (n / 3.0) + sum((2 * k + 4) * 8 * n for k in range(1, its + 1))
    elif dominant in ALGO_BYTES_PER_CELL:
        algo = ALGO_BYTES_MIXED.get(dominant, ALGO_BYTES_PER_CELL[dominant]) if mixed else ALGO_BYTES_PER_CELL[dominant]
        # kernels whose every launch covers the whole grid (the Hall EMF runs
        # once per Newton / Krylov evaluation); other kernels' per-step bytes
        # are shared by their launches (per-block or region launches)
        bytes_per_launch = algo * cells if dominant in WHOLE_GRID_KERNELS else algo * cells / launches_of[dominant]
    else:
        bytes_per_launch = None
    achieved = bytes_per_launch / (avg_launch_ms / 1000.0) / 1e9 if bytes_per_launch else None
    peak, peak_kind = measured_peak()
    group_ms = sum(per_step.get(k, 0.0) for k in FLUX_CT_GROUP)
    group_gbs = FLUX_CT_BYTES[mixed] * cells / (group_ms / 1000.0) / 1e9 if group_ms > 0 else None

    # end to end through host buffers (pinned), H2D + D2H inside the region:
    # the state's inner points (mhd_step_host_inner; the ghost points the
    # step reads are formed on the device by the Syncs)
    from beta1_b200.mhd import PinnedArray
    nstate = ctx.state_count_inner()
    hin, hout = PinnedArray(nstate), PinnedArray(nstate)
    # the state after the timed steps, as the caller would hold it
    off = 0
    for b in range(nblocks):
        for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
            inf = ctx.field_info(name, b)
            a = ctx.download(name, b)
            a = np.ascontiguousarray(a[tuple(slice(-l, h) for l, h in zip(inf["lo"], inf["hi"]))]).ravel()
            hin.a[off:off + a.size] = a
            off += a.size
    assert off == nstate
    ctx.step_host_inner(1, hin.a, hout.a)
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.e2e_iters):
        ctx.step_host_inner(1, hin.a, hout.a)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1) / args.e2e_iters
    e2e_value = replica_throughput(world, cells, 1, max_over_ranks(e2e_ms, "cuda"))
    hin.free()
    hout.free()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref_steps = args.ref_steps or wl["ref_steps"]
        warm = ref_warmup(args.workload, args.warmup)
        if args.workload in SWEEP_GRID:
            res = cpu_reference_sweep(ref_steps, 1, grid=SWEEP_GRID[args.workload][0], warmup=warm)
            if res is not None:
                cpu = {"value": res[0], "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                       "sample": "%s, run 0 of the sweep (%d cells), %d StepOnce of the reference solver built "
                                 "from its own sources after %d untimed, one single-threaded process"
                                 % (wl["name"], res[1][0]["cells"], ref_steps, warm)}
        else:
            res = cpu_reference(args.workload, args.n, ref_steps, 1, args.integrator, warmup=warm)
            if res is not None:
                agg, vals, _ = res
                what = HALL_SAMPLE if args.workload in ("c3", "c4") else (
                    "SSP-RK2 step" if args.integrator == "rk2" else "StepOnce")
                cpu = {"value": agg, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                       "sample": "%s, %d x %s of the reference solver built from its own sources after %d "
                                 "untimed, one single-threaded process" % (wl["name"], ref_steps, what, warm)}

    config_name = workload_name(wl["name"] if args.workload != "c2" or args.c2_size == "96x48" else
                                "c2_slab6x%sx%s_implicit_resistive_fp64" % (args.c2_size, args.c2_size.split("x")[1]), mixed)
    if args.workload in ("c3", "c4") and args.hall_size != "128x64":
        config_name = config_name.replace("128x64x64", "%sx%s" % (args.hall_size, args.hall_size.split("x")[1]))
    if sweep and len(runs) != SWEEP_RUNS:
        config_name = config_name.replace("sweep48", "sweep%d" % len(runs))
    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 fluxes + f64 CT/state" if mixed else "f64",
            "data": "synthetic (seeded 1e-3 noise on rho, v and div-free B; reference restart format)",
            "config": {"workload": config_name,
                       "cells_per_gpu": cells, "blocks": nblocks, "autotune_min_ctas_per_sm": tuned,
                       "integrator": ("SSP-RK2: two of StepOnce's forward-Euler stages at one dt and their "
                                      "convex average" if args.integrator == "rk2" else
                                      "forward Euler StepOnce (the reference's integrator)"),
                       "precision": args.precision,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "no flush: per-step working set %.2f GB > 126 MB L2" % (ctx_bytes / 1e9),
                       "geometry": geometry_on, "setup_s": round(setup_s, 2)},
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": nstate * 8,
                    "d2h_bytes_per_step": nstate * 8},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "peak_kind": peak_kind,
                         "traffic": NCU_TRAFFIC_BYTES.get((dominant, config_name)),
                         "algo_bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg_launch_ms,
                         "kernel_share": per_step[dominant] / total},
            "flux_ct_group": {"kernels": [k for k in FLUX_CT_GROUP if k in per_step], "ms_per_step": group_ms,
                              "algo_bytes_per_cell": FLUX_CT_BYTES[mixed], "achieved": group_gbs, "unit": "GB/s",
                              "frac": group_gbs / peak if group_gbs else None},
            "fp64_same_runs": fp64_line,
            "kernels_ms_per_step": {k: round(v, 5) for k, v in sorted(per_step.items(), key=lambda kv: -kv[1])},
            "resistive_solve": res_stats,
            "hall_solve": hall_stats,
            "cpu_baseline": cpu,
            "clocks": summarize_clocks(clocks),
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    s.ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
