#!/usr/bin/env python
"""Throughput of the B200 global ocean step on the 0.5-degree production
workload: 720x360x50 levels, float32 fields, dt = 1800 s, 24 barotropic
subcycles of 75 s, seeded synthetic bathymetry / thermocline / wind stress
(the reference's ETOPO/WOA/NCEP inputs are not available).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One "step" is one baroclinic time step of the resident state.  `value` is
simulated years per wall-clock day over all ranks (one independent replica
per GPU: the step does not shard), timed with CUDA events on the launching
stream; `e2e` is the same metric through the C ABI with host buffers (pinned
host -> device copy of the state and device -> host copy of the result every
step).  The per-step working set (~3 GB) is far larger than the 126 MB L2, so
no flush is needed between iterations.

`--impl reference` times the CPU restatement of the reference algorithm
(``oracle/``, float64 NumPy) on every host core, one spawned process per core,
each on a bounded sample: the same option set on a 180x90x50 grid (smaller
when many steps are asked for), scaled per grid point to 720x360x50; the
default line's `cpu_baseline` is the same on one core.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SECONDS_PER_YEAR = 365.0 * 86400.0
METRIC = "sim-years/day & ms/step at 720×360×50 on 1 B200: plain FP32 vs chosen form"
WORKLOAD = "plain"
SAMPLE_GRID = (180, 90, 50)

# Algorithmic bytes per launch of each kernel class, in units of one float32
# 3-D field (F = nx*ny*nz*4 bytes): distinct 3-D fields read + written by the
# stage the launch covers.  The nu_h class is counted per subcycle, as the
# stage structure has it (R+W of u and v, 4F, for each of the 2*n_nu
# subcycles of a step), however many subcycles one launch blocks together.
ALGO_FIELDS = {"nu_sub": None, "lin_finish": 10, "fz": 3, "madv": 5, "dealias": 4,
               "tracer_adv": 9, "tracer_rest": 10, "pgf": 10, "final": 12}
PROFILE_STEPS = 5
# DRAM bytes per launch measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum)
# for a kernel class on a grid, as summarised under profiles/; null for others.
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one full-size k_nu_tb launch (6 subcycles)
NCU_TRAFFIC_BYTES = {((720, 360, 50), "nu_sub"): 117752832 + 65883136}


def algo_fields_per_launch(cls, launches_per_step, n_nu):
    if cls == "nu_sub":
        return 4.0 * 2 * n_nu / launches_per_step
    return float(ALGO_FIELDS[cls])


def max_over_ranks(value, device="cuda"):
    """The largest of one float over all ranks of the process group (every
    rank's step time: the job is as fast as its slowest replica); the value
    itself without a group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sim_years_per_day(ms_per_step, dt):
    return (86400.0 / (ms_per_step * 1e-3)) * dt / SECONDS_PER_YEAR


def step_bytes(nx, ny, nz, n_nu, adv_nsub):
    """Stage-structure algorithmic bytes of one step (two L half steps with
    n_nu Laplacian sweeps, the N step, barotropic coupling and final pass)."""
    F = 4.0 * nx * ny * nz
    return (2 * (4 * n_nu + 10) + 46 + 12 * (adv_nsub - 1) + 8) * F


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


# Sample grids for the CPU timings (same option set), largest first; about
# 5.4 us per grid point per step for the float64 NumPy step on one core.
SAMPLE_GRIDS = ((180, 90, 50), (120, 60, 50), (90, 45, 50), (60, 30, 50), (48, 24, 50))
CPU_US_PER_POINT = 5.4


def sample_grid(total_steps, budget_s=150.0):
    for g in SAMPLE_GRIDS:
        if total_steps * g[0] * g[1] * g[2] * CPU_US_PER_POINT * 1e-6 <= budget_s:
            return g
    return SAMPLE_GRIDS[-1]


def cpu_baseline(steps=2, warmup=1, grid_shape=SAMPLE_GRID):
    """The float64 CPU restatement (oracle/) on a sample grid, scaled to the
    full grid per point; returns (ms_per_full_step, description)."""
    from oracle import params as oparams
    from oracle import step as ostep
    from zhenmode_b200 import workloads
    nx, ny, nz = grid_shape
    grid, physics, dt, kw, T, S = workloads.make_case(WORKLOAD, nx, ny, nz, dtype="float64")
    kw = {k: v for k, v in kw.items() if k in oparams.SUPPORTED}
    p = oparams.build_params(grid, physics, dt, **kw)
    st = oparams.init_state(p, T, S)
    for _ in range(warmup):
        st = ostep.step(st, p)
    t0 = time.perf_counter()
    for _ in range(steps):
        st = ostep.step(st, p)
    sample_ms = (time.perf_counter() - t0) * 1e3 / steps
    wl = workloads.WORKLOADS[WORKLOAD]
    scale = (wl.nx * wl.ny * wl.nz) / float(nx * ny * nz)
    desc = (f"float64 NumPy restatement of the reference step (oracle/), {steps} timed steps after {warmup} "
            f"warm-up at {nx}x{ny}x{nz} with the 0.5-degree option set ({sample_ms:.0f} ms/step), scaled "
            f"x{scale:.0f} per grid point to {wl.nx}x{wl.ny}x{wl.nz}")
    return sample_ms * scale, desc


def _cpu_worker(q, steps, warmup, shape):
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    q.put(cpu_baseline(steps=steps, warmup=warmup, grid_shape=shape))


def cpu_baseline_all_cores(steps, warmup, shape, procs):
    """cpu_baseline in `procs` concurrent processes (spawned; no GPU use), one
    sample grid each: the host's throughput with every core busy.  Returns
    (ms per full-grid step, description)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    workers = [ctx.Process(target=_cpu_worker, args=(q, steps, warmup, shape)) for _ in range(procs)]
    for w in workers:
        w.start()
    results = [q.get() for _ in workers]
    for w in workers:
        w.join()
    worst = max(r[0] for r in results)           # slowest worker, full-grid ms per step
    ms = worst / procs                            # procs samples advance concurrently
    desc = (f"{procs} concurrent processes (one per host core), each: " + results[0][1] +
            f"; slowest process {worst / 1e3:.1f} s per full-grid step, aggregate {ms / 1e3:.1f} s")
    return ms, desc


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from zhenmode_b200 import workloads
    wl = workloads.WORKLOADS[WORKLOAD]
    shape = sample_grid(args.steps + args.warmup)
    procs = max(1, len(os.sched_getaffinity(0)))
    ms, desc = cpu_baseline_all_cores(max(1, args.steps), max(0, args.warmup), shape, procs)
    value = sim_years_per_day(ms, wl.dt)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "sim-years/day",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded bathymetry, thermocline, wind stress)",
            "config": {"workload": f"{wl.nx}x{wl.ny}x{wl.nz} 0.5-degree plain FP32 option set, dt={wl.dt:.0f} s",
                       "sample": f"{shape[0]}x{shape[1]}x{shape[2]}"},
            "cpu_baseline": {"value": value, "unit": "sim-years/day", "cores": procs, "kind": "port",
                             "sample": desc, "cpu": platform.processor() or platform.machine(),
                             "host_cores": len(os.sched_getaffinity(0))},
            "e2e": {"value": value, "unit": "sim-years/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# the batched ensemble form: (members, nx, ny, nz) groups advanced together
ENSEMBLE_GROUPS = ((32, 360, 180, 30), (8, 720, 360, 50), (16, 180, 90, 20))


def run_ensemble(args):
    """All members of ENSEMBLE_GROUPS (each T perturbed by its own seed,
    sigma 0.05 K) advance one simulated day in one CUDA-graph launch per step;
    the same members advanced one after another (each its own graphs) give the
    sequential reference.  Value = aggregate simulated years per day."""
    import numpy as np
    import torch

    from zhenmode_b200 import make_solver_global, workloads
    from zhenmode_b200.ensemble import Ensemble

    wl = workloads.WORKLOADS[WORKLOAD]
    steps, states, sizes = [], [], []
    seed = 100
    for count, nx, ny, nz in ENSEMBLE_GROUPS:
        grid, physics, dt, kw, T, S = workloads.make_case(WORKLOAD, nx, ny, nz, dtype="float32")
        wet = np.asarray(grid.wet_mask_3d)
        for _ in range(count):
            step, init, _ = make_solver_global(grid, physics, dt, autotune=True, **kw)
            rng = np.random.default_rng(seed)
            seed += 1
            steps.append(step)
            states.append(init(T + 0.05 * rng.standard_normal(T.shape) * wet, S))
            sizes.append(nx * ny * nz)
    nday = int(round(86400.0 / wl.dt))
    ens = Ensemble(steps)
    ens.load(states)
    ens.advance(max(args.warmup, 3))
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.advance(nday)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_ens = e0.elapsed_time(e1)
    codes = ens.monitor_codes()
    # sequential: each member alone through its own graphs
    import ctypes
    sp = ctypes.c_void_p(stream.cuda_stream)
    for st in steps:
        st.solver.check(st.solver.lib.zm_advance(st.solver.handle, sp, 3), "zm_advance")
    torch.cuda.synchronize()
    e0.record(stream)
    for st in steps:
        st.solver.check(st.solver.lib.zm_advance(st.solver.handle, sp, nday), "zm_advance")
    e1.record(stream)
    torch.cuda.synchronize()
    ms_seq = e0.elapsed_time(e1)
    n = len(steps)
    years = n * nday * wl.dt / SECONDS_PER_YEAR
    value = years / (ms_ens * 1e-3) * 86400.0
    seq_value = years / (ms_seq * 1e-3) * 86400.0
    line = {"metric": METRIC, "value": value, "unit": "sim-years/day", "n_gpus": 1, "steps": nday,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_ens / nday, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded bathymetry, "
            "thermocline, wind stress; per-member seeded T perturbation sigma 0.05 K)",
            "config": {"workload": "batched ensemble: " + ", ".join(f"{c} x {x}x{y}x{z}" for c, x, y, z in
                                                                   ENSEMBLE_GROUPS) + ", 1 simulated day each",
                       "form": "ensemble", "members": n, "points": int(sum(sizes)),
                       "graph_kernels_per_step": ens.kernels_per_step, "monitor_codes_nonzero": sum(c != 0 for c in codes)},
            "sequential": {"value": seq_value, "ms_per_step": ms_seq / nday},
            "ensemble_speedup_vs_sequential": ms_seq / ms_ens,
            "roofline": None, "gpu_launches": nday * ens.kernels_per_step, "clocks": clk, "e2e": None,
            "cpu_baseline": None}
    print(json.dumps(line))
    return 0


def run_precision(args):
    """The precision form: 800x400x50, implicit vertical diffusion (FP32 Thomas
    plus one refinement step), float64 barotropic mode, a seasonal forcing
    (wind stress x (1 + 0.25 sin) and a +-100 W/m^2 heat flux over 12 monthly
    fields, blended on the device before every step) for 10 simulated days,
    with the compensated float64 heat / salt budgets taken every day."""
    import ctypes

    import numpy as np
    import torch

    from zhenmode_b200 import _native, make_solver_global, workloads

    # the 0.45-degree option set: nu_h, nu_bi, kappa_bi and dt_bt scaled from the
    # 0.5-degree values by the CFL powers of dx (runtime/cli.py:49-61)
    grid, physics, dt, kw, T, S = workloads.make_case("precision", dtype="float32")
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    kw = dict(kw)
    kw.update(vertical_diffusion="implicit")
    step, init_state, _ = make_solver_global(grid, physics, dt, autotune=not args.no_autotune, **kw)
    solver = step.solver
    st = init_state(T_init=T, S_init=S)
    lat = np.radians(np.asarray(grid.lat))
    tau0 = np.broadcast_to((0.1 * np.sin(2 * lat) * np.cos(lat))[None, :], (nx, ny))
    phase = np.sin(2 * np.pi * (np.arange(12) + 0.5) / 12.0)
    taux = torch.as_tensor(np.stack([tau0 * (1 + 0.25 * p) for p in phase]).astype(np.float32), device="cuda")
    qh = torch.as_tensor(np.stack([np.broadcast_to(100.0 * p * np.cos(lat)[None, :], (nx, ny)) for p in phase])
                         .astype(np.float32), device="cuda")
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    sin = _native.ZmState(*[t.data_ptr() for t in (st.u, st.v, st.T, st.S, st.eta)])
    solver.check(solver.lib.zm_load_state(solver.handle, sp, ctypes.byref(sin)), "zm_load_state")
    out = [torch.empty_like(t) for t in (st.u, st.v, st.T, st.S, st.eta)]
    sout = _native.ZmState(*[t.data_ptr() for t in out])

    def budgets():
        solver.check(solver.lib.zm_store_state(solver.handle, sp, ctypes.byref(sout)), "zm_store_state")
        b = (ctypes.c_double * 8)()
        solver.check(solver.lib.zm_budgets(solver.handle, sp, ctypes.c_void_p(out[2].data_ptr()),
                                           ctypes.c_void_p(out[3].data_ptr()), 1025.0, 3992.0, b), "zm_budgets")
        return list(b)

    per_day = int(round(86400.0 / dt))
    days = 10

    def one_step(n):
        step.set_forcing_seasonal(tau_x=taux, q_heat=qh, day=n * dt / 86400.0)
        solver.check(solver.lib.zm_advance(solver.handle, sp, 1), "zm_advance")

    for n in range(max(args.warmup, 3)):
        one_step(n)
    b0 = budgets()
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    total_ms = 0.0
    daily = [b0]
    for dday in range(days):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for n in range(per_day):
            one_step(dday * per_day + n)
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        daily.append(budgets())
    clk = clocks.stop()
    code = ctypes.c_int32()
    solver.check(solver.lib.zm_status(solver.handle, ctypes.byref(code)), "zm_status")
    nsteps = days * per_day
    ms = total_ms / nsteps
    audit = budget_audit_day(step, out, taux, qh, (days * per_day + max(args.warmup, 3)), per_day, dt)
    heat = [d[4] for d in daily]
    salt = [d[5] for d in daily]
    drift = lambda v: max(abs(v[i + 1] - v[i]) / abs(v[i]) for i in range(len(v) - 1))
    F = 4.0 * nx * ny * nz
    bstep = step_bytes(nx, ny, nz, solver.n_nu, solver.adv_nsub)
    peak, peak_kind = measured_peaks()
    line = {"metric": METRIC, "value": sim_years_per_day(ms, dt), "unit": "sim-years/day", "n_gpus": 1,
            "steps": nsteps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded bathymetry, thermocline; seasonal wind stress and +-100 W/m^2 heat flux)",
            "config": {"workload": f"{nx}x{ny}x{nz} precision form: implicit vertical diffusion with one refinement "
                                   f"step, float64 barotropic mode, {solver.n_subcyc} subcycles, seasonal forcing "
                                   f"blended on the device every step, {days} simulated days",
                       "form": "precision", "monitor_code": int(code.value)},
            "budgets": {"heat_content_J": heat, "salt_content_kg": salt,
                        "max_relative_change_per_day": {"heat": drift(heat), "salt": drift(salt)},
                        "total_volume_m3": daily[-1][6], "sums": "float64, compensated, fixed order",
                        "ledger_day_after": audit},
            "roofline": {"bound": "hbm", "step_stage_bytes": bstep, "step_frac": bstep / (ms * 1e-3) / 1e9 / peak,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s"},
            "gpu_launches": nsteps * (solver.kernels_per_step() + 3), "clocks": clk, "e2e": None,
            "cpu_baseline": None}
    print(json.dumps(line))
    return 0


def budget_audit_day(step, fields, taux, qh, n0, per_day, dt):
    """One more simulated day of the precision form through the stage/source
    ledger (the reference's budget audit step): per quantity (heat J, salt kg,
    volume m^3) the observed change of the day, the summed source inputs
    (surface heat and salt fluxes, restoring, sponge), and the budget residual
    observed - sources with its ratio to the change scale."""
    from zhenmode_b200 import JaxStateG, ledger

    advance = ledger.make_budget_step(step)
    st = JaxStateG(*fields, 0.0)
    total = ledger.empty_budget()
    for n in range(per_day):
        step.set_forcing_seasonal(tau_x=taux, q_heat=qh, day=(n0 + n) * dt / 86400.0)
        st, led = advance(st)
        total = ledger.accumulate_budget(total, led)
    names = ("heat_J", "salt_kg", "volume_m3")
    obs, src, res, scale = (total["observed_change"], total["source_inputs"].sum(axis=0),
                            total["budget_residual"], total["change_scale"])
    # what the fixed-node inventory leaves outside the sources (the reference
    # ledger reports these as diagnostics, not sources): the advective flux
    # through the rigid-lid surface, the eta x surface-tracer change, and the
    # closure of the stage decomposition (observed - sum of stage changes)
    advb, disp, dec = (total["advection_boundary_changes"], total["surface_displacement_tracer_change"],
                       total["decomposition_residual"])
    return {n: {"observed_change": float(obs[i]), "source_inputs": float(src[i]), "residual": float(res[i]),
                "residual_over_change_scale": float(abs(res[i]) / scale[i]) if scale[i] > 0 else None,
                "surface_advective_flux": float(advb[i]), "surface_displacement_tracer_change": float(disp[i]),
                "stage_decomposition_residual": float(dec[i])}
            for i, n in enumerate(names)}


def train_closure(step, st, dt, days):
    """The learned closure trained on the plain model's own columns: `days`
    simulated days of the plain step from `st`, 60 snapshots, at most 2M
    rows, 3000 Adam steps of 8192 rows.  Returns (network, record, the state
    at the end of the plain run)."""
    import torch

    from zhenmode_b200.closure import ClosureMLP, collect, fit
    steps_per_day = int(round(86400.0 / dt))
    nsteps = days * steps_per_day
    every = max(1, nsteps // 60)
    t0 = time.time()
    X, Tt, M, end = collect(step, st, nsteps, every=every, max_rows=2_000_000, seed=0)
    torch.cuda.synchronize()
    t1 = time.time()
    net = ClosureMLP(seed=0)
    loss = fit(net, X, Tt, M, steps=3000, batch=8192, lr=1e-3)
    torch.cuda.synchronize()
    info = {"rows": int(X.shape[0]), "collect_days": days, "snapshots": nsteps // every,
            "collect_s": round(t1 - t0, 1), "train_steps": 3000, "batch": 8192,
            "train_s": round(time.time() - t1, 1), "loss_log10_kappa_mse": loss}
    del X, Tt, M
    return net, info, end


def chosen_form(step, st, dt, grid, solver, args, plain_ms):
    """The learned-closure form beside the plain one: train the network on
    the plain model's columns, time the step with it (CUDA events around
    zm_advance on the resident state, as for the plain line), and compare
    10 simulated days of it with the plain run (daily-mean SST, SSS and
    mixed-layer depth)."""
    import ctypes

    import torch

    from zhenmode_b200 import _native
    from zhenmode_b200.closure import compare_with_plain
    net, info, end = train_closure(step, st, dt, args.closure_days)
    steps_per_day = int(round(86400.0 / dt))
    cmp = compare_with_plain(step, net, end, 10, steps_per_day, grid)
    step.set_closure(net)
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    sin = _native.ZmState(*[t.data_ptr() for t in (end.u, end.v, end.T, end.S, end.eta)])
    solver.check(solver.lib.zm_load_state(solver.handle, sptr, ctypes.byref(sin)), "zm_load_state")
    solver.check(solver.lib.zm_advance(solver.handle, sptr, args.warmup), "zm_advance")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.check(solver.lib.zm_advance(solver.handle, sptr, args.steps), "zm_advance")
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    prof = {}
    for _ in range(PROFILE_STEPS):
        for k, (pm, pc) in solver.profile(stream.cuda_stream).items():
            am, ac = prof.get(k, (0.0, 0))
            prof[k] = (am + pm / PROFILE_STEPS, pc)
    fallback = step.closure_stats()[0]
    step.set_closure(None)
    return {"form": "learned", "ms_per_step": ms, "value": sim_years_per_day(ms, dt), "unit": "sim-years/day",
            "speedup_vs_plain": plain_ms / ms, "target_speedup": 1.3,
            "kernel_ms_per_step": {k: round(v[0], 4) for k, v in prof.items() if v[1] > 0},
            "fallback_columns_last_step": int(fallback), "training": info,
            "vs_plain_10_days": {"days": 10, "start": f"day {args.closure_days} of the plain training run", **cmp,
                                 "sst_rmse_K_max": max(cmp["sst_rmse_K"]), "target_sst_rmse_K": 0.05}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default=None, help="NXxNYxNZ: same option set on another grid (profiling cases)")
    ap.add_argument("--form", default="plain", choices=["plain", "learned", "ensemble", "precision", "projected"],
                    help="learned: train the closure network on the plain model's own columns (30 days, "
                         "2M rows) first, then time the step with it; projected: the plain step with the "
                         "column-divergence projection of the stage-2 advective velocity on")
    ap.add_argument("--closure-days", type=int, default=30)
    ap.add_argument("--no-learned", action="store_true",
                    help="plain form only: skip training and timing the learned-closure form beside it")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shapes (profiling: no autotuner trial launches)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.form == "ensemble":
        return run_ensemble(args)
    if args.form == "precision":
        return run_precision(args)

    import ctypes

    import torch
    import torch.distributed as dist

    from zhenmode_b200 import _native, make_solver_global, workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    wl = workloads.WORKLOADS[WORKLOAD]
    if args.grid:
        import dataclasses
        gnx, gny, gnz = (int(x) for x in args.grid.lower().split("x"))
        wl = dataclasses.replace(wl, nx=gnx, ny=gny, nz=gnz)
    grid, physics, dt, kw, T, S = workloads.make_case(WORKLOAD, wl.nx, wl.ny, wl.nz, dtype="float32")
    if args.form == "projected":
        kw = dict(kw, project_adv_vel=True)
    step, init_state, _ = make_solver_global(grid, physics, dt, autotune=not args.no_autotune, **kw)
    solver = step.solver
    st = init_state(T_init=T, S_init=S)
    closure_info = None
    if args.form == "learned":
        net, closure_info, _ = train_closure(step, st, dt, args.closure_days)
        step.set_closure(net)
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    sin = _native.ZmState(*[t.data_ptr() for t in (st.u, st.v, st.T, st.S, st.eta)])
    solver.check(solver.lib.zm_load_state(solver.handle, sptr, ctypes.byref(sin)), "zm_load_state")
    solver.check(solver.lib.zm_advance(solver.handle, sptr, args.warmup), "zm_advance")
    torch.cuda.synchronize()

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.check(solver.lib.zm_advance(solver.handle, sptr, args.steps), "zm_advance")
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    code = ctypes.c_int32()
    solver.check(solver.lib.zm_status(solver.handle, ctypes.byref(code)), "zm_status")
    ms = max_over_ranks(ms)
    kernels_per_step = solver.kernels_per_step()

    # per-kernel-class breakdown of one step (CUDA events around every launch)
    # (average of PROFILE_STEPS un-graphed steps, events on the launching stream)
    prof = {}
    for _ in range(PROFILE_STEPS):
        for k, (pm, pc) in solver.profile(stream.cuda_stream).items():
            am, ac = prof.get(k, (0.0, 0))
            prof[k] = (am + pm / PROFILE_STEPS, pc)
    total_prof = sum(v[0] for v in prof.values())
    ranked = sorted(((v[0], k) for k, v in prof.items() if v[1] > 0), reverse=True)
    dominant = next(k for _, k in ranked if k in ALGO_FIELDS)
    dom_ms, dom_launches = prof[dominant]
    F = 4.0 * wl.nx * wl.ny * wl.nz
    algo = algo_fields_per_launch(dominant, dom_launches, solver.n_nu) * F
    achieved = algo / (dom_ms / dom_launches * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = NCU_TRAFFIC_BYTES.get(((wl.nx, wl.ny, wl.nz), dominant))
    bstep = step_bytes(wl.nx, wl.ny, wl.nz, solver.n_nu, solver.adv_nsub)

    # end to end through the C ABI with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        host = [t.cpu().pin_memory() for t in (st.u, st.v, st.T, st.S, st.eta)]
        hout = [torch.empty_like(h).pin_memory() for h in host]
        hin = _native.ZmState(*[h.data_ptr() for h in host])
        hres = _native.ZmState(*[h.data_ptr() for h in hout])
        solver.check(solver.lib.zm_step_host(solver.handle, sptr, ctypes.byref(hin), ctypes.byref(hres), 1),
                     "zm_step_host")
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(args.e2e_steps):
            solver.check(solver.lib.zm_step_host(solver.handle, sptr, ctypes.byref(hin), ctypes.byref(hres), 1),
                         "zm_step_host")
        e3.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(e2.elapsed_time(e3) / args.e2e_steps)
        nbytes = sum(h.numel() * h.element_size() for h in host)
        e2e = {"value": world * sim_years_per_day(ems, wl.dt), "unit": "sim-years/day", "ms_per_step": ems,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes}

    # the reference runtime's call (run_loop.py:56): step(JaxStateG) on device
    # tensors in the reference layout, each call loading the state through the
    # ABI, running the step graph and storing the result into new tensors
    dropin = None
    if args.e2e_steps > 0:
        cur = step(st)
        for _ in range(3):  # the caching allocator settles on the output tensors
            cur = step(cur)
        torch.cuda.synchronize()
        e4 = torch.cuda.Event(enable_timing=True)
        e5 = torch.cuda.Event(enable_timing=True)
        t_host = time.perf_counter()
        e4.record(stream)
        for _ in range(args.e2e_steps):
            cur = step(cur)
        e5.record(stream)
        torch.cuda.synchronize()
        t_host = (time.perf_counter() - t_host) * 1e3 / args.e2e_steps
        dms = max_over_ranks(e4.elapsed_time(e5) / args.e2e_steps)
        dropin = {"ms_per_call": dms, "host_ms_per_call": t_host, "over_resident_step_ms": dms - ms,
                  "call": "step(JaxStateG of CUDA tensors), reference layout in and out"}
        del cur

    chosen = None
    if args.form == "plain" and not args.no_learned and world == 1:
        chosen = chosen_form(step, st, wl.dt, grid, solver, args, ms)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cms, desc = cpu_baseline()
        cpu = {"value": sim_years_per_day(cms, wl.dt), "unit": "sim-years/day", "cores": 1, "kind": "port",
               "sample": desc, "ms_per_step": cms, "host_cores": len(os.sched_getaffinity(0))}

    if rank == 0:
        line = {"metric": METRIC, "value": world * sim_years_per_day(ms, wl.dt), "unit": "sim-years/day",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded bathymetry, thermocline, wind stress)",
                "config": {"workload": f"{wl.nx}x{wl.ny}x{wl.nz} 0.5-degree plain FP32 option set, dt={wl.dt:.0f} s, "
                                       f"{solver.n_subcyc} barotropic subcycles, {solver.n_nu} nu_h subcycles",
                           "parallelism": f"replicas x{world}", "l2": "per-step working set >> L2 (no flush)",
                           "monitor_code": int(code.value), "form": args.form,
                           "autotuned": solver.launch_shapes()},
                "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                             "traffic": traffic, "algorithmic_bytes_per_launch": algo,
                             "launch_ms": dom_ms / dom_launches,
                             "step_stage_bytes": bstep, "step_frac": bstep / (ms * 1e-3) / 1e9 / peak,
                             "step_floor_bytes": 8 * F, "floor_frac": 8 * F / (ms * 1e-3) / 1e9 / peak},
                "kernel_ms_per_step": {k: round(v[0], 4) for k, v in prof.items() if v[1] > 0},
                "kernel_ms_unrolled_total": total_prof,
                "gpu_launches": args.steps * kernels_per_step + 1,
                "clocks": clk, "e2e": e2e, "cpu_baseline": cpu}
        if closure_info is not None:
            closure_info["fallback_columns_last_step"] = step.closure_stats()[0]
            line["closure"] = closure_info
        if chosen is not None:
            line["chosen_form"] = chosen
        if dropin is not None:
            line["dropin_step_call"] = dropin
        if args.form == "projected":
            it = step.projection_stats()
            line["projection"] = {"cg_iterations": list(it[:3]), "refinement_solves": it[3],
                                  "ms_per_step": round(prof.get("projection", (0.0, 0))[0], 4)}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
