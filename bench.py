"""Benchmark of the B200 IFE-PIC step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config cfg4] [--impl ours|reference]

One step = one explicit IFE-PIC time step on one GPU (fused push + locate +
deposit of all particles, RHS + Poisson solve to the deck's tolerance, PPR
field recovery, MCC null collisions, counting sort every sort_interval
steps), data resident in HBM.  The metric is particle pushes/s with the
Poisson ms/step of the solvers side by side: the reference's Jacobi-PCG,
flexible CG with smoothing + a two-level coarse space or a multigrid V-cycle,
and the two-level one with the learned U-Net stage, all at the deck's
tolerance on the same systems.

The default workload is the 1024x1024-cell, 8-ellipse deck (about 101M
particles, Poisson tolerance 1e-8).  The run (1) trains the learned stage
online on --train-steps Jacobi-PCG steps, (2) solves the same systems with
every solver, (3) times --plain-steps steps of the plain FP64 Jacobi-PCG path,
(4) times --steps steps of the product path (the fastest FCG variant), then
the same through host buffers (e2e).  With N > 1 (launched by
torch.distributed.run) every rank runs an independent replica with its own
seed ("replicas only": the reference has no domain decomposition), the timed
region is bracketed by a barrier and the slowest rank's time is used.

--impl reference times the CPU restatement of the reference's step
(oracle/liboracle.so, the reference being Fortran with no compiler on the
host) on a bounded sample of the same workload and prints the same JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle pushes/s + Poisson ms/step: learned-precond FCG vs plain PCG at 1e-8"
# The roofline's per-particle unit is the scope table's algorithmic figure for
# push + gather + deposit: FP64 88 B (x, y, vx, vy, vz and the cell, read and
# written), mixed precision 48 B.  The kernels move less (vz stays untouched
# on steps without the energy diagnostic); their own bytes are reported
# beside it.
UNIT_PUSH_BYTES = {"fp64": 88, "mixed": 48}
FP64_PUSH_BYTES = 72   # read x,y,vx,vy,elem (36 B; vz only on diagnostic steps), write the same (36 B)
MIXED_PUSH_BYTES = 40  # read elem + 4 FP32 (20 B), write the same (20 B)
# + the particle id (4 B) when the push builds the step's MCC selection
SELECT_BYTES = 4
# r-z decks (delta 1): v_theta is read and written on every step
FP64_PUSH_BYTES_RZ = 88
MIXED_PUSH_BYTES_RZ = 48
# DRAM bytes per particle of one push launch measured by ncu (dram__bytes_read
# + dram__bytes_write; the traffic grows in proportion to the particle count):
# the 1024^2 eight-ellipse deck at 8 particles per cell (FP64 k_push_bulk,
# mixed k_push_mixed_bulk) and the 2048x1024 r-z deck at 8 (mixed r-z);
# "_sel": the push also builds the MCC selection (reads the ids)
NCU_PUSH_TRAFFIC = {"fp64": 68.0, "mixed": 38.0, "mixed_rz": 51.4,
                    "fp64_sel": 72.2, "mixed_sel": 42.4, "mixed_rz_sel": 55.5}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return dist, rank, ws


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def _max_over_ranks(dist, v: float) -> float:
    if dist is None:
        return v
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(dist, v: float) -> float:
    if dist is None:
        return v
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, every 50 ms, each sample
    stamped with the host time it arrived; summary() keeps the samples inside
    a marked window (the timed region).  Started before the warm-up so that
    nvidia-smi's own start-up does not eat the short timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.window = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append((time.perf_counter(), parts))

    def mark(self, t0: float, t1: float):
        """The host-time window [t0, t1] of the timed region."""
        self.window = (t0, t1)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows, where = [r for _, r in self.rows], "all"
        if self.window and self.rows:
            t0, t1 = self.window
            inside = [r for t, r in self.rows if t0 <= t <= t1]
            if inside:
                rows, where = inside, "timed region"
            else:  # the timed region fell between two samples: the nearest one
                tm = 0.5 * (t0 + t1)
                rows, where = [min(self.rows, key=lambda tr: abs(tr[0] - tm))[1]], "nearest to the timed region"
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows),
                "samples_from": where, "interval_ms": 50}


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return None


def cpu_baseline(cfg_name: str, sample_particles: int, steps: int, pcg_iters: int | None = None,
                 pcg_cap: int = 200):
    """Times the oracle (C restatement of the reference step, OpenMP on all
    the host's threads) on a bounded sample: push+deposit of `sample_particles` particles per
    species for `steps` steps, extrapolated to the full particle count, plus
    RHS + Jacobi-PCG + PPR on the full mesh.  The PCG runs at most `pcg_cap`
    iterations per step and its time is scaled to `pcg_iters` iterations (the
    count the reference's PCG needs for the step: the GPU Jacobi-PCG's, which
    runs the same algorithm, or one full oracle solve when None).  Returns
    (pushes/s, description, seconds per step, threads, particles loaded).
    Everything it runs is the oracle's: the mesh, interface geometry,
    operator, load matrices, volumes and patches come from or_mesh_build
    (with the quadrature constants as the reference compiles them), so this
    leg loads no library of the product."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob
    from pic_b200 import deck
    cfg = deck.config(cfg_name)
    mesh = ob.OracleMesh(deck.make_deck(cfg), ob.OR_QUAD_AS_COMPILED)
    sp, _ = deck.species_params(cfg)
    sc = cfg.scales
    nn = mesh.nn
    parts, full_n = [], 0
    for s in range(2):
        x, y, vx, vy, vz = deck.load_particles(cfg, mesh, s)
        full_n += x.size
        k = min(sample_particles, x.size)
        loc = np.array([ob.load().or_locate(mesh.ptr, a, b) for a, b in zip(x[:k], y[:k])], np.int32)
        parts.append({"x": x[:k].copy(), "y": y[:k].copy(), "vx": vx[:k].copy(), "vy": vy[:k].copy(),
                      "vz": vz[:k].copy(), "loc": loc})
        del x, y, vx, vy, vz
    sample_n = sum(p["x"].size for p in parts)
    phi = mesh.array("phi_dirichlet")
    efx = np.zeros(nn)
    efy = np.zeros(nn)
    coef = np.zeros(5 * nn)
    t_part = t_field = 0.0
    note = ""
    mover = ob.move_all_axi if cfg.delta == 1 else ob.move_all  # MoveOne's r-z or Cartesian branch
    for step in range(steps):
        t0 = time.perf_counter()
        qs, es, wq = [], [], []
        for s in range(2):
            qm = sp[s][0] / (sp[s][1] / deck.ME)
            mover(mesh.ptr, parts[s], efx, efy, coef, qm, cfg.dt)
            q, e, _ = ob.deposit(mesh.ptr, parts[s], sp[s][1], sc["v_ref"], nn)
            qs.append(q)
            es.append(e)
            wq.append(sp[s][2] * sp[s][0])
        t_part += time.perf_counter() - t0
        # full-size field phase on the sampled charge scaled to the full count
        t1 = time.perf_counter()
        rho, _, _ = ob.normalize(mesh.ptr, qs, es, wq, sc["L_ref"], cfg.n0, nn)
        rho *= full_n / max(sample_n, 1)
        b = ob.rhs(mesh.ptr, rho, nn)
        t_rhs = time.perf_counter() - t1
        if pcg_iters is None:  # one full solve gives the iteration count (not timed)
            tf = time.perf_counter()
            _, stf = ob.pcg(mesh.ptr, b, phi, cfg.pcg_tol, cfg.pcg_maxit)
            pcg_iters = max(1, stf["iterations"])
            note = f"; count from one full oracle solve ({time.perf_counter() - tf:.1f} s)"
        tp = time.perf_counter()
        phi, st = ob.pcg(mesh.ptr, b, phi, cfg.pcg_tol, min(pcg_cap, cfg.pcg_maxit))
        t_pcg = (time.perf_counter() - tp) / max(1, st["iterations"]) * pcg_iters
        t3 = time.perf_counter()
        c, efx, efy = ob.ppr(mesh.ptr, phi, nn)
        coef = np.ascontiguousarray(c.ravel())
        t_field += t_rhs + t_pcg + (time.perf_counter() - t3)
    per_step = t_part / steps * (full_n / sample_n) + t_field / steps
    mesh.close()
    threads = ob.load().or_threads()
    desc = (f"{cfg.name}: {threads} host threads; push+deposit of {sample_n} of {full_n} particles for {steps} "
            f"step(s), extrapolated "
            f"by particle count; RHS+Jacobi-PCG+PPR on the full {cfg.ncx}x{cfg.ncy} mesh, the PCG timed over "
            f"<= {pcg_cap} iterations and scaled to the step's {pcg_iters} iterations{note}; mesh and "
            f"operator built by the oracle")
    return full_n / per_step, desc, per_step, threads, full_n


def run_reference(args, dist, rank, ws):
    if rank != 0:
        return 0
    cpu_baseline(args.config, min(args.cpu_sample, 20000), 1, pcg_iters=1, pcg_cap=1)  # warm-up (caches)
    steps = max(1, args.steps)
    v, desc, per_step, threads, n_loaded = cpu_baseline(args.config, args.cpu_sample, min(steps, 2))
    from pic_b200 import deck
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "particle pushes/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded uniform Maxwellian plasma, seeded objects)",
        "config": _config(deck.config(args.config), "fp64", n_loaded, ws),
        "solver": "jacobi_pcg",
        "cpu_baseline": {"value": v, "unit": "particle pushes/s", "cores": threads, "kind": "port",
                         "sample": desc},
        "e2e": {"value": v, "unit": "particle pushes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _timed_steps(sim, lib, api, n):
    """n steps timed on the library stream; returns (ms, [StepStats])."""
    stats = []
    api.check(lib.pic_device_timer(0, None), "timer")
    for _ in range(n):
        stats.append(sim.step())
    ms = C.c_double()
    api.check(lib.pic_device_timer(1, C.byref(ms)), "timer")
    return ms.value, stats


def _poisson_compare(sim, lib, api, variants, repeats=3):
    """Each variant solves the same systems: the step's push + deposit, then
    the Poisson solve from the previous phi, `repeats` times (device timer).
    variants: name -> callable that selects the solver."""
    phi_prev = sim.field("phi")
    for s in range(2):
        sim.move_all(s)
    sim.get_par_chg()
    out = {}
    for name, select in variants.items():
        select()
        ms, its, fb = [], [], []
        for _ in range(repeats):
            sim.set_field("phi", phi_prev)
            st = api.SolveStats()
            api.check(lib.pic_device_timer(0, None), "timer")
            api.check(lib.pic_ife_solve(None, 0.0, C.byref(st)), "solve")
            t = C.c_double()
            api.check(lib.pic_device_timer(1, C.byref(t)), "timer")
            ms.append(t.value)
            its.append(st.iterations)
            fb.append(st.fallback)
        out[name] = {"ms": statistics.median(ms), "iterations": statistics.median(its),
                     "fallback": max(fb)}
    return out


def _config(cfg, precision: str, particles: int, ws: int) -> dict:
    """The workload as both arms print it (same keys, same values)."""
    soa = 48 if precision == "fp64" else 28  # bytes a particle holds in HBM (x, y, v, elem, id)
    return {"workload": cfg.name, "cells": [cfg.ncx, cfg.ncy], "particles": int(particles),
            "objects": len(cfg.objects), "geometry": "r-z" if cfg.delta == 1 else "x-y",
            "precision": precision, "pcg_tol": cfg.pcg_tol, "sort_interval": cfg.sort_interval,
            "mcc": bool(cfg.mcc), "parallelism": f"replicas x{ws}",
            "l2": ("inputs larger than L2" if particles * soa > 126e6 else "inputs fit in L2, not flushed")
                  + " (particle SoA %.2f GB)" % (particles * soa / 1e9)}


def _push_roofline(precision: str, rz: bool, stats, peak, peak_src, select: bool = False):
    """Algorithmic bytes of the fused push per launch / its CUDA-event time
    (select: the push also reads each particle's id for the MCC selection)."""
    push_ms = sum(s.ms_push_kernel for s in stats) / len(stats)
    push_n = sum(s.pushed for s in stats) / len(stats)
    if precision == "mixed":
        nbytes = MIXED_PUSH_BYTES_RZ if rz else MIXED_PUSH_BYTES
        kernel = "k_push_mixed_bulk"
    else:
        nbytes = FP64_PUSH_BYTES_RZ if rz else FP64_PUSH_BYTES
        kernel = "k_push_bulk"
    nbytes += SELECT_BYTES if select else 0
    unit = UNIT_PUSH_BYTES[precision]
    achieved = unit * push_n / (push_ms / 1e3) / 1e9
    own = nbytes * push_n / (push_ms / 1e3) / 1e9
    key = precision + ("_rz" if rz else "") + ("_sel" if select else "")
    tr = NCU_PUSH_TRAFFIC[key] * push_n if key in NCU_PUSH_TRAFFIC else None
    return {"kernel": kernel + (" r-z" if rz else "") + " (fused push+locate+deposit)", "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_src, "bytes_per_particle": unit,
            "kernel_bytes_per_particle": nbytes, "kernel_bytes_achieved": own, "kernel_bytes_frac": own / peak,
            "traffic": tr,
            "traffic_note": ("no ncu capture of this push" if tr is None else
                             "ncu DRAM bytes/particle of one launch at 8 particles per cell (6.4M particles; "
                             "r-z 16.7M) x particles per step")}, push_ms


def _push_select(cfg) -> bool:
    """Whether the push builds the step's MCC selection (decks with MCC,
    unless PIC_MCC_PUSH_SELECT=0)."""
    return bool(cfg.mcc) and os.environ.get("PIC_MCC_PUSH_SELECT", "1") != "0"


def _sel(sim, name, lp=None):
    """Select a Poisson solver variant by its bench name (set_solver switches
    the learned stage off; it is switched on after, for the learned variant)."""
    if name == "jacobi_pcg":
        sim.set_solver("jpcg")
    elif name == "fcg_smooth_coarse":
        sim.set_solver("fcg", coarse_cells=64, window=1)
    elif name == "fcg_smooth_coarse_learned":
        sim.set_solver("fcg", coarse_cells=64, window=4)
    elif name == "fcg_smooth_multigrid_learned":
        sim.set_solver("fcg", window=4, multigrid=True, omega=0.8)
    elif name == "fcg_smooth_coarse_fp32_iterations_in_fp64_refinement":
        sim.set_solver("fcg", coarse_cells=64, window=1, inner_fp32=True)
    elif name == "fcg_smooth_multigrid":
        # damped-Jacobi weight 0.8 with the V-cycle: 11 iterations at 1024^2 against 12 with 2/3
        sim.set_solver("fcg", window=1, multigrid=True, omega=0.8)
    elif name == "fcg_smooth_multigrid_fp32_iterations_in_fp64_refinement":
        sim.set_solver("fcg", window=1, multigrid=True, omega=0.8, inner_fp32=True)
    else:
        raise KeyError(name)
    if lp is not None and name.endswith("_learned"):
        lp.set_learned(True)


def _side_run(name, precision, solver, steps, warmup, peak, peak_src, dist):
    """A deck measured on its own simulation: setup, warm-up, timed steps."""
    from pic_b200 import api, deck
    from pic_b200.simulation import Simulation
    cfg = deck.config(name, precision=api.PIC_PREC_MIXED if precision == "mixed" else api.PIC_PREC_FP64)
    t0 = time.perf_counter()
    sim = Simulation(cfg)
    try:
        sim.initial_fields()
        n0 = sim.count(0) + sim.count(1)
        setup_s = time.perf_counter() - t0
        _sel(sim, solver)
        for _ in range(warmup):
            sim.step()
        _barrier(dist)
        ms, st = _timed_steps(sim, sim.lib, api, steps)
        roof, push_ms = _push_roofline(precision, cfg.delta == 1, st, peak, peak_src, _push_select(cfg))
        pushed = sum(s.pushed for s in st)
        return {"config": _config(cfg, precision, n0, 1), "solver": solver, "steps": steps,
                "ms_per_step": ms / steps, "value": pushed / (ms / 1e3), "unit": "particle pushes/s",
                "poisson_ms_per_step": sum(s.ms_solve for s in st) / steps,
                "poisson_iterations_per_step": sum(s.solve.iterations for s in st) / steps,
                "push_ms_per_step": push_ms, "mcc_ms_per_step": sum(s.ms_mcc for s in st) / steps,
                "setup_s": setup_s, "roofline": roof}
    finally:
        sim.close()


def run_ours(args, dist, rank, ws):
    import torch
    from pic_b200 import api, build, deck, unet
    from pic_b200.simulation import Simulation

    build.build()
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(dev)
    peaks = _peaks()
    if peaks and peaks.get("hbm_gbs"):
        peak, peak_src = peaks["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    cfg = deck.config(args.config)
    cfg.seed = cfg.seed + 1000 * rank
    prec = args.precision
    cfg.precision = api.PIC_PREC_MIXED if prec == "mixed" else api.PIC_PREC_FP64
    t_setup = time.perf_counter()
    sim = Simulation(cfg)
    lib = sim.lib
    st0 = sim.initial_fields()
    n_initial = sim.count(0) + sim.count(1)
    setup_s = time.perf_counter() - t_setup
    # ---- online training of the learned stage on Jacobi-PCG warm-up steps
    lp = None
    t_train = time.perf_counter()
    if args.train_steps > 0:
        # the network learns the error the multigrid V-cycle leaves (its
        # training pairs pass through the same classical stages)
        lp = unet.LearnedPreconditioner(sim, seed=rank, crop=128, batch=4, lr=2e-3, window=4,
                                        multigrid=True, omega=0.8)
        sim.set_solver("jpcg")
        for _ in range(args.train_steps):
            lp.before_step()
            sim.step()
            lp.after_step(train_iters=8)
    train_s = time.perf_counter() - t_train
    names = ["jacobi_pcg", "fcg_smooth_coarse", "fcg_smooth_multigrid"]
    if prec == "mixed":
        names += ["fcg_smooth_coarse_fp32_iterations_in_fp64_refinement",
                  "fcg_smooth_multigrid_fp32_iterations_in_fp64_refinement"]
    if lp is not None:
        names.append("fcg_smooth_multigrid_learned")
    variants = {k: (lambda k=k: _sel(sim, k, lp)) for k in names}
    poisson = _poisson_compare(sim, lib, api, variants)
    # product path: the fastest FCG variant that converged without falling back
    fcg_names = [k for k in variants if k != "jacobi_pcg" and poisson[k]["fallback"] == 0]
    best = min(fcg_names, key=lambda k: poisson[k]["ms"]) if fcg_names else "jacobi_pcg"
    # ---- the plain path: the same particles with the reference's Jacobi-PCG
    _sel(sim, "jacobi_pcg", lp)
    sim.step()
    _barrier(dist)
    ms_plain, st_plain = _timed_steps(sim, lib, api, max(1, args.plain_steps))
    ms_plain_max = _max_over_ranks(dist, ms_plain)
    # ---- product path, device-resident timed region
    _sel(sim, best, lp)
    with ClockSampler(dev) as clk:
        for _ in range(args.warmup):
            sim.step()
        _barrier(dist)
        if torch.cuda.is_available():
            torch.cuda.synchronize()
        launches0 = lib.pic_kernel_launches()
        t_clk0 = time.perf_counter()
        ms_total, stats = _timed_steps(sim, lib, api, args.steps)
        clk.mark(t_clk0, time.perf_counter())
        time.sleep(0.06)  # let the sample that covers the end arrive
    launches = lib.pic_kernel_launches() - launches0
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    _barrier(dist)
    ms_total = _max_over_ranks(dist, ms_total)
    pushed = _sum_over_ranks(dist, float(sum(s.pushed for s in stats)))
    value = pushed / (ms_total / 1e3)
    # ---- end to end through the C-ABI with host buffers (drop-in use)
    nn = sim.mesh.nn
    pinned = {}
    for k in ("phi", "rho", "efx", "efy"):
        pinned[k] = torch.empty(nn, dtype=torch.float64, pin_memory=torch.cuda.is_available()).numpy()
    pinned["phi"][:] = sim.field("phi")
    # whole sort periods (a sort every sort_interval steps), so both loops
    # below carry the same share of sorts as a long run
    e2e_steps = max(1, cfg.sort_interval) * max(1, min(2, -(-args.steps // max(1, cfg.sort_interval))))

    def e2e_run(overlap: bool) -> float:
        """Steps through the C-ABI with phi in from and rho, phi, efx, efy out
        to pinned host arrays every step; overlap: the upload of phi and the
        readback run on the library's copy stream alongside the step's push
        (pic_set_field_async, pic_get_fields_async; the last copies are
        waited for inside the timed region), else synchronous
        pic_set_field / pic_get_field calls."""
        _barrier(dist)
        pushed_e2e = 0
        api.check(lib.pic_device_timer(0, None), "timer")
        for _ in range(e2e_steps):
            if overlap:
                api.check(lib.pic_set_field_async(1, api.dptr(pinned["phi"])), "set phi")
            else:
                api.check(lib.pic_set_field(1, api.dptr(pinned["phi"])), "set phi")
            st = sim.step()
            pushed_e2e += st.pushed
            if overlap:
                api.check(lib.pic_get_fields_async(api.dptr(pinned["rho"]), api.dptr(pinned["phi"]),
                                                   api.dptr(pinned["efx"]), api.dptr(pinned["efy"])),
                          "get fields")
            else:
                for k, w in (("rho", 0), ("phi", 1), ("efx", 2), ("efy", 3)):
                    api.check(lib.pic_get_field(w, api.dptr(pinned[k])), "get field")
        if overlap:
            api.check(lib.pic_wait_fields(), "wait fields")
        ms = C.c_double()
        api.check(lib.pic_device_timer(1, C.byref(ms)), "timer")
        _barrier(dist)
        return _sum_over_ranks(dist, float(pushed_e2e)) / (_max_over_ranks(dist, ms.value) / 1e3)

    e2e_sync_value = e2e_run(False)
    e2e_value = e2e_run(True)
    roof, push_ms = _push_roofline(prec, cfg.delta == 1, stats, peak, peak_src, _push_select(cfg))
    solve_ms = [s.ms_solve for s in stats]
    its = [s.solve.iterations for s in stats]
    ms_step = ms_total / args.steps
    plain_step = ms_plain_max / len(st_plain)
    sim.close()
    line = {
        "metric": METRIC, "value": value, "unit": "particle pushes/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 particles/f64 fields" if prec == "mixed" else "f64",
        "data": "synthetic (seeded uniform Maxwellian plasma, seeded objects)",
        "config": _config(cfg, prec, n_initial, ws),
        "solver": best,
        "poisson_ms_per_step": sum(solve_ms) / len(solve_ms),
        "poisson_iterations_per_step": sum(its) / len(its),
        "poisson_solvers_same_systems": poisson,
        "plain_jacobi_pcg_path": {
            "precision": prec, "ms_per_step": plain_step, "steps": len(st_plain),
            "poisson_ms_per_step": sum(s.ms_solve for s in st_plain) / len(st_plain),
            "pcg_iterations_per_step": sum(s.solve.iterations for s in st_plain) / len(st_plain),
            "speedup_of_product_path": plain_step / ms_step},
        "push_ms_per_step": push_ms,
        "ppr_ms_per_step": sum(s.ms_ppr for s in stats) / len(stats),
        "mcc_ms_per_step": sum(s.ms_mcc for s in stats) / len(stats),
        "sort_ms_per_step": sum(s.ms_sort for s in stats) / len(stats),
        "initial_pcg_iterations": st0.iterations,
        "setup_s": setup_s,
        "learned_training": None if lp is None else {
            "warmup_steps": args.train_steps, "adam_steps": len(lp.losses), "seconds": train_s,
            "loss_first": lp.losses[0], "loss_last": lp.losses[-1]},
        # the metric names the learned-preconditioner FCG; the product path is
        # the fastest FCG variant on the same systems, and this says whether
        # the learned stage is it
        "learned_stage": None if "fcg_smooth_multigrid_learned" not in poisson else {
            "on_product_path": best.endswith("_learned"),
            "learned_ms": poisson["fcg_smooth_multigrid_learned"]["ms"],
            "learned_iterations": poisson["fcg_smooth_multigrid_learned"]["iterations"],
            "without_ms": poisson["fcg_smooth_multigrid"]["ms"],
            "without_iterations": poisson["fcg_smooth_multigrid"]["iterations"],
            "note": "the learned stage is on the product path" if best.endswith("_learned") else
                    ("the learned stage on top of the multigrid V-cycle needs more FCG iterations than the "
                     "V-cycle alone, so the product path runs without it")
                    if poisson["fcg_smooth_multigrid_learned"]["iterations"]
                    > poisson["fcg_smooth_multigrid"]["iterations"] else
                    ("the network's forward pass costs more than the iterations it saves, so the product "
                     "path runs without it")},
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": "particle pushes/s", "steps": e2e_steps,
                "transfers": "pic_set_field_async + pic_get_fields_async (copies alongside the push)",
                "value_with_synchronous_transfers": e2e_sync_value,
                "h2d_bytes_per_step": 8 * nn, "d2h_bytes_per_step": 4 * 8 * nn},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    # ---- the north star's chosen form (mixed precision) and the other decks,
    # each on its own simulation (one rank; untimed by the driver's ratio)
    if rank == 0 and ws == 1 and not args.no_side_runs:
        if prec == "fp64":
            mixed = _side_run(args.config, "mixed", best, args.steps, args.warmup, peak, peak_src, None)
            mixed["speedup_vs_plain_fp64_jacobi_pcg"] = plain_step / mixed["ms_per_step"]
            line["mixed_precision_path"] = mixed
        line["other_configs"] = {
            "cfg2": _side_run("cfg2", "fp64", "jacobi_pcg", 5, 2, peak, peak_src, None),
            "cfg5": _side_run("cfg5", "mixed", "fcg_smooth_multigrid", 5, 2, peak, peak_src, None)}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        jp = poisson["jacobi_pcg"]["iterations"]
        v, desc, _, threads, _ = cpu_baseline(args.config, args.cpu_sample, 1, pcg_iters=int(jp))
        line["cpu_baseline"] = {"value": v, "unit": "particle pushes/s", "cores": threads, "kind": "port",
                                "sample": desc}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_accuracy(args):
    """The mixed-precision error table on one deck: the plain FP64 path
    (FP64 particles, the reference's Jacobi-PCG; bit-exact with the oracle on
    the small decks), FP64 particles with the product's multigrid FCG, and
    the mixed-precision product path (element + FP32 offsets, multigrid FCG),
    all from the same seed for the same steps.  At each checkpoint step: the
    relative error (max |x - x_fp64| / max |x_fp64|) of phi, E and the
    Average_x profiles (Output_To_Tecplot_IJK_2D.f90:166-226) of the ion
    density and the electron mean energy (2/3 of it is the temperature).
    Prints one JSON line."""
    import torch
    from pic_b200 import api, build, deck
    from pic_b200.simulation import Simulation

    build.build()
    steps = args.acc_steps
    checks = sorted({c for c in (20, 100, 500, steps) if c <= steps})

    def run(precision, solver):
        cfg = deck.config(args.accuracy, precision=precision, diag_interval=1)
        sim = Simulation(cfg)
        try:
            sim.initial_fields()
            if solver == "mg":
                try:
                    sim.set_solver("fcg", window=1, multigrid=True, omega=0.8)
                except api.PicError:  # a grid too small to coarsen: the two-level space
                    sim.set_solver("fcg", window=1)
            else:
                sim.set_solver("jpcg")
            out, ms, its, done = {}, 0.0, 0, 0
            for c in checks:
                m, st = _timed_steps(sim, sim.lib, api, c - done)
                ms += m
                its += sum(s.solve.iterations for s in st)
                done = c
                avg = sim.average_x()
                out[c] = {"phi": sim.field("phi"), "efx": sim.field("efx"), "efy": sim.field("efy"),
                          "ion_density_profile": avg["Rho_" + sim.SPECIES_TAGS[1]].copy(),
                          "electron_energy_profile": avg["Ek_" + sim.SPECIES_TAGS[0]].copy(),
                          "counts": [sim.count(q) for q in range(2)]}
            particles = sum(out[checks[0]]["counts"])
            return out, {"ms_per_step": ms / steps, "poisson_iterations_per_step": its / steps,
                         "particles_at_start": particles}
        finally:
            sim.close()

    ref, t_ref = run(api.PIC_PREC_FP64, "jpcg")
    f64mg, t_f64mg = run(api.PIC_PREC_FP64, "mg")
    mix, t_mix = run(api.PIC_PREC_MIXED, "mg")
    mixj, t_mixj = run(api.PIC_PREC_MIXED, "jpcg")
    fields = ("phi", "efx", "efy", "ion_density_profile", "electron_energy_profile")

    def table(other, base=None):
        base = ref if base is None else base
        t = {}
        for c in checks:
            a, b = base[c], other[c]
            row = {f: float(np.abs(b[f] - a[f]).max() / np.abs(a[f]).max()) for f in fields}
            row["counts_fp64"], row["counts"] = a["counts"], b["counts"]
            t[str(c)] = row
        return t

    bars = {"phi": 1e-5, "ion_density_profile": 1e-2}
    mixed = table(mix)
    last = mixed[str(steps)]
    line = {"accuracy": deck.config(args.accuracy).name, "steps": steps, "seed": deck.config(args.accuracy).seed,
            "reference_path": "fp64 particles, Jacobi-PCG (MY_PCG), pcg_tol of the deck",
            "errors_mixed_multigrid_vs_fp64_jpcg": mixed,
            "errors_fp64_multigrid_vs_fp64_jpcg": table(f64mg),
            "errors_mixed_multigrid_vs_fp64_multigrid": table(mix, f64mg),
            "errors_mixed_jpcg_vs_fp64_jpcg": table(mixj),
            "bars_at_last_step": bars,
            "pass": {f: last[f] <= b for f, b in bars.items()},
            "timing": {"fp64_jacobi_pcg": t_ref, "fp64_multigrid_fcg": t_f64mg, "mixed_multigrid_fcg": t_mix,
                       "mixed_jacobi_pcg": t_mixj,
                       "speedup_mixed_vs_plain_fp64": t_ref["ms_per_step"] / t_mix["ms_per_step"]},
            "device": torch.cuda.get_device_name(0) if torch.cuda.is_available() else None}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="cfg4")
    ap.add_argument("--train-steps", type=int, default=30,
                    help="Jacobi-PCG warm-up steps that train the learned stage (0: no learned stage)")
    ap.add_argument("--plain-steps", type=int, default=5,
                    help="steps of the plain FP64 Jacobi-PCG path timed for comparison")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="particles in FP64 (the headline, like the reference), or element + FP32 "
                         "offsets and velocities (then measured beside it)")
    ap.add_argument("--no-side-runs", action="store_true",
                    help="skip the mixed-precision path and the other decks")
    ap.add_argument("--cpu-sample", type=int, default=400000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--accuracy", default=None,
                    help="print the mixed-precision error table of this deck (e.g. cfg3) instead of a bench line")
    ap.add_argument("--acc-steps", type=int, default=1000)
    args = ap.parse_args()
    if args.accuracy:
        return run_accuracy(args)
    dist, rank, ws = _dist()
    try:
        if args.impl == "reference":
            rc = run_reference(args, dist, rank, ws)
        else:
            rc = run_ours(args, dist, rank, ws)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
