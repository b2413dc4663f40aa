"""Benchmark of the B200 IFE-PIC step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config cfg2] [--impl ours|reference]

One step = one explicit IFE-PIC time step on one GPU (fused push + locate +
deposit of all particles, RHS + Jacobi-PCG Poisson solve to the deck's
tolerance, PPR field recovery, MCC null collisions, counting sort every
sort_interval steps), data resident in HBM.  The metric is particle
pushes/s; Poisson ms/step, PCG iterations/step and full-step ms ride along.

The default workload is the 512x512-cell, 4-disk deck (about 52M
particles).  With N > 1 (launched by torch.distributed.run) every rank runs
an independent replica with its own seed ("replicas only": the reference has
no domain decomposition), the timed region is bracketed by a barrier and the
slowest rank's time is used.

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
FP64_PUSH_BYTES = 80  # read x,y,vx,vy,vz,elem (44 B) + write x,y,vx,vy,elem (36 B)


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
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
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
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[3 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows)}


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return None


def cpu_baseline(cfg_name: str, sample_particles: int, steps: int, seed_offset: int = 0):
    """Times the oracle (C restatement of the reference step, one host thread)
    on a bounded sample: push+deposit of `sample_particles` particles per
    species for `steps` steps, extrapolated to the full particle count, plus
    RHS + Jacobi-PCG + PPR on the full mesh (warm started).  Returns
    (pushes/s, description)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob
    from pic_b200 import deck
    cfg = deck.config(cfg_name, seed=deck.config(cfg_name).seed + seed_offset)
    mesh = deck.Mesh(cfg)
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
    sample_n = sum(p["x"].size for p in parts)
    phi = mesh.array("phi_dirichlet")
    efx = np.zeros(nn)
    efy = np.zeros(nn)
    coef = np.zeros(5 * nn)
    t_part = 0.0
    t_field = 0.0
    for step in range(steps):
        t0 = time.perf_counter()
        qs, es, wq = [], [], []
        for s in range(2):
            qm = sp[s][0] / (sp[s][1] / deck.ME)
            ob.move_all(mesh.ptr, parts[s], efx, efy, coef, qm, cfg.dt)
            q, e, _ = ob.deposit(mesh.ptr, parts[s], sp[s][1], sc["v_ref"], nn)
            qs.append(q)
            es.append(e)
            wq.append(sp[s][2] * sp[s][0])
        t1 = time.perf_counter()
        # full-size field phase on the sampled charge scaled to the full count
        rho, _, _ = ob.normalize(mesh.ptr, qs, es, wq, sc["L_ref"], cfg.n0, nn)
        rho *= full_n / max(sample_n, 1)
        b = ob.rhs(mesh.ptr, rho, nn)
        phi, st = ob.pcg(mesh.ptr, b, phi, cfg.pcg_tol, cfg.pcg_maxit)
        c, efx, efy = ob.ppr(mesh.ptr, phi, nn)
        coef = np.ascontiguousarray(c.ravel())
        t2 = time.perf_counter()
        t_part += t1 - t0
        t_field += t2 - t1
    per_step = t_part / steps * (full_n / sample_n) + t_field / steps
    mesh.close()
    desc = (f"{cfg.name}: push+deposit of {sample_n} of {full_n} particles for {steps} steps, "
            f"extrapolated by particle count; RHS+Jacobi-PCG+PPR on the full {cfg.ncx}x{cfg.ncy} mesh")
    return full_n / per_step, desc, per_step


def run_reference(args, dist, rank, ws):
    if rank != 0:
        return 0
    value, desc, per_step = None, None, None
    vals = []
    # warm-up + timed steps of the CPU restatement, each step a bounded sample
    v, desc, per_step = cpu_baseline(args.config, args.cpu_sample, max(1, args.warmup))
    t0 = time.perf_counter()
    tot_steps = max(1, args.steps)
    v, desc, per_step = cpu_baseline(args.config, args.cpu_sample, tot_steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "particle pushes/s",
        "n_gpus": args.gpus, "steps": tot_steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.config},
        "cpu_baseline": {"value": v, "unit": "particle pushes/s", "cores": 1, "kind": "port",
                         "sample": desc},
        "e2e": {"value": v, "unit": "particle pushes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, dist, rank, ws):
    import torch
    from pic_b200 import api, build, deck
    from pic_b200.simulation import Simulation

    build.build()
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(dev)
    cfg = deck.config(args.config)
    cfg.seed = cfg.seed + 1000 * rank
    t_setup = time.perf_counter()
    sim = Simulation(cfg)
    lib = sim.lib
    st0 = sim.initial_fields()
    setup_s = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        sim.step()
    # ---- device-resident timed region
    _barrier(dist)
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    launches0 = lib.pic_kernel_launches()
    stats = []
    with ClockSampler(dev) as clk:
        api.check(lib.pic_device_timer(0, None), "timer")
        for _ in range(args.steps):
            stats.append(sim.step())
        ms = C.c_double()
        api.check(lib.pic_device_timer(1, C.byref(ms)), "timer")
    launches = lib.pic_kernel_launches() - launches0
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    _barrier(dist)
    ms_total = _max_over_ranks(dist, ms.value)
    pushed = _sum_over_ranks(dist, float(sum(s.pushed for s in stats)))
    value = pushed / (ms_total / 1e3)
    # ---- end to end through the C-ABI with host buffers (drop-in use)
    nn = sim.mesh.nn
    pinned = {}
    for k in ("phi", "rho", "efx", "efy"):
        pinned[k] = torch.empty(nn, dtype=torch.float64, pin_memory=torch.cuda.is_available()).numpy()
    pinned["phi"][:] = sim.field("phi")
    e2e_steps = max(1, min(args.steps, 10))
    _barrier(dist)
    e2e_pushed = 0
    api.check(lib.pic_device_timer(0, None), "timer")
    for _ in range(e2e_steps):
        api.check(lib.pic_set_field(1, api.dptr(pinned["phi"])), "set phi")
        st = sim.step()
        e2e_pushed += st.pushed
        for k, w in (("rho", 0), ("phi", 1), ("efx", 2), ("efy", 3)):
            api.check(lib.pic_get_field(w, api.dptr(pinned[k])), "get field")
    ms_e2e = C.c_double()
    api.check(lib.pic_device_timer(1, C.byref(ms_e2e)), "timer")
    _barrier(dist)
    ms_e2e_max = _max_over_ranks(dist, ms_e2e.value)
    e2e_value = _sum_over_ranks(dist, float(e2e_pushed)) / (ms_e2e_max / 1e3)
    # ---- roofline of the fused push kernel
    push_ms = sum(s.ms_push_kernel for s in stats) / len(stats)
    push_n = sum(s.pushed for s in stats) / len(stats)
    achieved = FP64_PUSH_BYTES * push_n / (push_ms / 1e3) / 1e9
    peaks = _peaks()
    if peaks and peaks.get("hbm_gbs"):
        peak, peak_src = peaks["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    solve_ms = [s.ms_solve for s in stats]
    its = [s.solve.iterations for s in stats]
    line = {
        "metric": METRIC, "value": value, "unit": "particle pushes/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded uniform Maxwellian plasma, seeded objects)",
        "config": {"workload": cfg.name, "cells": [cfg.ncx, cfg.ncy],
                   "particles": int(stats[0].pushed), "objects": len(cfg.objects),
                   "precision": "fp64", "solver": "jacobi-pcg", "pcg_tol": cfg.pcg_tol,
                   "sort_interval": cfg.sort_interval, "mcc": bool(cfg.mcc),
                   "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (particle SoA %.1f GB)" % (push_n * 48 / 1e9)},
        "poisson_ms_per_step": sum(solve_ms) / len(solve_ms),
        "pcg_iterations_per_step": sum(its) / len(its),
        "push_ms_per_step": push_ms,
        "ppr_ms_per_step": sum(s.ms_ppr for s in stats) / len(stats),
        "mcc_ms_per_step": sum(s.ms_mcc for s in stats) / len(stats),
        "sort_ms_per_step": sum(s.ms_sort for s in stats) / len(stats),
        "initial_pcg_iterations": st0.iterations,
        "setup_s": setup_s,
        "roofline": {"kernel": "k_push (fused push+locate+deposit)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "bytes_per_particle": FP64_PUSH_BYTES,
                     "traffic": None},
        "e2e": {"value": e2e_value, "unit": "particle pushes/s", "steps": e2e_steps,
                "h2d_bytes_per_step": 8 * nn, "d2h_bytes_per_step": 4 * 8 * nn},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, desc, _ = cpu_baseline(args.config, args.cpu_sample, 2)
        line["cpu_baseline"] = {"value": v, "unit": "particle pushes/s", "cores": 1, "kind": "port",
                                "sample": desc}
    sim.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=400000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
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
