"""Small, self-contained workloads for profiling one part of the step under
ncu (each runs a few launches of its kernels and exits):

    python profile_cases.py step  <deck> <ppc> <steps> [jpcg|fcg|mg] [fp64|mixed]
    python profile_cases.py solve <cells> [jpcg|fcg|mg] [repeats] [coarse_cells] [fp64|mixed] [omega] [max_coarse_nodes]
    python profile_cases.py unet  <nodes> [repeats]
    python profile_cases.py diag  <deck> <ppc> [fp64|mixed] [repeats]
    python profile_cases.py sort  <deck> <ppc> <drift_steps> [fp64|mixed] [repeats]

step:  the deck at <ppc> particles per cell and species, <steps> steps.
solve: the 8-ellipse deck at <cells>^2 without particles, a seeded random
       charge density, Poisson solves from phi = 0 (mg: the multigrid
       V-cycle in place of the two-level coarse space).
unet:  forward passes of the learned stage's network on a <nodes>^2 grid.
diag:  the deck after one step, then the device diagnostics (Average_x
       profiles, energy spectra, velocity moments) of every species.
sort:  the deck after <drift_steps> steps from the initial sort, then the
       counting sort of every species, <repeats> times with <drift_steps>
       steps between (the sort alone is timed).
Each prints one line with its own CUDA-event time.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np


def _step(deck_name, ppc, steps, solver="fcg", precision="fp64"):
    import torch
    from pic_b200 import api, deck
    from pic_b200.simulation import Simulation
    prec = api.PIC_PREC_MIXED if precision == "mixed" else api.PIC_PREC_FP64
    cfg = deck.config(deck_name, ppc=int(ppc), precision=prec)
    sim = Simulation(cfg)
    sim.initial_fields()
    if solver == "mg":
        sim.set_solver("fcg", multigrid=True, omega=0.8)
    elif solver != "jpcg":
        sim.set_solver("fcg")
    sim.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(int(steps)):
        sim.step()
    e1.record()
    torch.cuda.synchronize()
    print(f"step {cfg.name} ppc={ppc} solver={solver} {precision}: {e0.elapsed_time(e1) / int(steps):.3f} ms/step")
    sim.close()


def _solve(cells, solver="fcg", repeats=3, coarse_cells=64, precision="fp64", omega=2.0 / 3.0,
           max_coarse_nodes=4500):
    import torch
    from pic_b200 import api, deck
    from pic_b200.simulation import Simulation
    n = int(cells)
    prec = api.PIC_PREC_MIXED if precision == "mixed" else api.PIC_PREC_FP64
    cfg = deck.config("cfg4", ncx=n, ncy=n, ppc=1, precision=prec)
    sim = Simulation(cfg, load=False)
    sim.set_field("rho", np.random.default_rng(0).standard_normal(sim.mesh.nn))
    import time
    t0 = time.perf_counter()
    if solver == "mg":
        sim.set_solver("fcg", multigrid=True, omega=float(omega), max_coarse_nodes=int(max_coarse_nodes))
    else:
        sim.set_solver(solver, coarse_cells=int(coarse_cells), omega=float(omega))
    setup = time.perf_counter() - t0
    out = []
    for _ in range(int(repeats)):
        sim.set_field("phi", np.zeros(sim.mesh.nn))
        st = api.SolveStats()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        api.check(sim.lib.pic_ife_solve(None, 0.0, C.byref(st)), "pic_ife_solve")
        e1.record()
        torch.cuda.synchronize()
        out.append((st.iterations, st.outer, round(e0.elapsed_time(e1), 3)))
    print(f"solve {n}^2 {solver} {precision} coarse_cells={coarse_cells} max_coarse_nodes={max_coarse_nodes} "
          f"omega={float(omega):.3f} (setup {setup:.2f} s): "
          f"(iterations, outer, ms) {out}")
    sim.close()


def _unet(nodes, repeats=10):
    import torch
    from pic_b200 import unet
    n = int(nodes)
    net = unet.UNet(seed=0)
    net._ensure(1, n, n)
    torch.cuda.synchronize()
    for _ in range(2):
        net.forward()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(int(repeats)):
        net.forward()
    e1.record()
    torch.cuda.synchronize()
    print(f"unet forward {n}x{n}: {e0.elapsed_time(e1) / int(repeats):.3f} ms")


def _diag(deck_name, ppc, precision="mixed", repeats=5):
    import time
    from pic_b200 import api, deck
    from pic_b200.simulation import Simulation
    prec = api.PIC_PREC_MIXED if precision == "mixed" else api.PIC_PREC_FP64
    sim = Simulation(deck.config(deck_name, ppc=int(ppc), precision=prec, diag_interval=1))
    sim.initial_fields()
    sim.set_solver("fcg")
    sim.step()
    ns = len(sim.species)
    n = [sim.count(s) for s in range(ns)]
    calls = {"average_x": lambda: sim.average_x(),
             "energy_spectrum": lambda: [sim.energy_spectrum(s) for s in range(ns)],
             "velocity_moments": lambda: [sim.velocity_moments(s) for s in range(ns)]}
    res = {}
    for name, fn in calls.items():
        fn()
        t0 = time.perf_counter()
        for _ in range(int(repeats)):
            fn()
        res[name] = round((time.perf_counter() - t0) / int(repeats) * 1e3, 3)
    print(f"diag {sim.cfg.name} {precision} particles {n}: host ms per call (all species) {res}")
    sim.close()


def _sort(deck_name, ppc, drift_steps, precision="fp64", repeats=2):
    import torch
    from pic_b200 import api, deck
    from pic_b200.simulation import Simulation
    prec = api.PIC_PREC_MIXED if precision == "mixed" else api.PIC_PREC_FP64
    # sort_interval beyond the run: only the sorts called here reorder
    sim = Simulation(deck.config(deck_name, ppc=int(ppc), precision=prec, sort_interval=1 << 30))
    sim.initial_fields()
    sim.set_solver("fcg", multigrid=True, omega=0.8)
    ms = 0.0
    for _ in range(int(repeats)):
        for _ in range(int(drift_steps)):
            sim.step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s in range(len(sim.species)):
            sim.sort(s)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    n = [sim.count(s) for s in range(len(sim.species))]
    print(f"sort {sim.cfg.name} {precision} particles {n} after {drift_steps} steps: "
          f"{ms / int(repeats):.3f} ms (all species)")
    sim.close()


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(__doc__)
    case, rest = sys.argv[1], sys.argv[2:]
    {"step": _step, "solve": _solve, "unet": _unet, "diag": _diag, "sort": _sort}[case](*rest)
