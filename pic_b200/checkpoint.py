"""Checkpoint and restart of a running simulation: the role of the
reference's restart dumps (code/PIC/Dump_2D.f90: control variables, phi and
the particle array; MCC_jw/code/base/ParticleBundle.f90:286-375
DumpParticleBundle / LoadParticleBundle), in this package's own format.

A checkpoint is one .npz file holding what the next step depends on: the
step index, phi (the solver's warm start; E and the PPR coefficients are
recomputed from it, as the step itself computes them), and per species the
live particles (absolute FP64 position, velocity, element, id) and the id
the next created particle receives.  Random numbers are counter-based
(Philox, and the selection hash, keyed by seed, step and particle id), so
nothing else carries state: a restored run continues bit for bit like the
uninterrupted one.
The deck itself is not stored.  restore() checks that the deck it is given
matches the checkpoint's: mesh size, seed, precision, and the physics the
state depends on (Cartesian or r-z, extent, dt, n0, Te, gas, per-species
charge, mass and macro-weight, the RF wall drive).  A mismatch raises
ValueError before anything touches the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api
from .deck import Config, species_params
from .simulation import Simulation

_VERSION = 2


def _physics(cfg: Config) -> np.ndarray:
    """The deck's physics parameters the saved state depends on, as one
    FP64 vector: geometry kind and extent, time step, reference density and
    temperature, gas, per-species (charge, mass, weight), RF drive (wall,
    volts, frequency, phase; NaN when static)."""
    rf = list(cfg.rf) if cfg.rf is not None else [np.nan] * 4
    rf = (rf + [0.0])[:4] if cfg.rf is not None and len(rf) == 3 else rf
    sp, _ = species_params(cfg)
    v = [cfg.delta, cfg.Lx, cfg.Ly, cfg.dt, cfg.n0, cfg.Te_eV, cfg.gas_p_Pa, cfg.gas_T_K]
    for q, m, w, _ in sp:
        v += [q, m, w]
    return np.array(v + [float(x) for x in rf], dtype=np.float64)


_PHYSICS_NAMES = ["delta", "Lx", "Ly", "dt", "n0", "Te_eV", "gas_p_Pa", "gas_T_K"]


def save(sim: Simulation, path: str) -> None:
    out = {"version": np.int64(_VERSION), "step": np.int64(sim.step_index),
           "nnx": np.int64(sim.mesh.nnx), "nny": np.int64(sim.mesh.nny),
           "seed": np.uint64(sim.cfg.seed), "precision": np.int64(sim.cfg.precision),
           "n_species": np.int64(len(sim.species)), "phi": sim.field("phi"),
           "physics": _physics(sim.cfg)}
    for s in range(len(sim.species)):
        p = sim.download(s)
        for k, v in p.items():
            out[f"s{s}_{k}"] = v
        nid = C.c_uint32()
        api.check(sim.lib.pic_get_next_id(s, C.byref(nid)), "pic_get_next_id")
        out[f"s{s}_next_id"] = np.uint64(nid.value)
    np.savez(path, **out)


def restore(cfg: Config, path: str, capacity_factor: float = 1.5, **sim_kw) -> Simulation:
    """A Simulation of `cfg` in the state saved at `path`; set the solver as
    before (it is a choice of the run, not state)."""
    z = np.load(path)
    if int(z["version"]) != _VERSION:
        raise ValueError(f"checkpoint version {int(z['version'])}, expected {_VERSION}")
    want = {"nnx": cfg.ncx + 1, "nny": cfg.ncy + 1, "seed": cfg.seed, "precision": cfg.precision}
    for k, v in want.items():
        if int(z[k]) != int(v):
            raise ValueError(f"checkpoint {k} = {int(z[k])} does not match the deck's {v}")
    got, want_p = np.asarray(z["physics"]), _physics(cfg)
    if got.shape != want_p.shape:
        raise ValueError("checkpoint physics: another number of species or parameters than the deck's")
    same = (got == want_p) | (np.isnan(got) & np.isnan(want_p))
    if not same.all():
        k = int(np.flatnonzero(~same)[0])
        nsp = (got.size - len(_PHYSICS_NAMES) - 4) // 3
        names = _PHYSICS_NAMES + [f"species{s}_{f}" for s in range(nsp) for f in ("charge", "mass", "weight")]
        names += ["rf_wall", "rf_volts", "rf_frequency", "rf_phase"]
        raise ValueError(f"checkpoint {names[k]} = {got[k]!r} does not match the deck's {want_p[k]!r}")
    ns = int(z["n_species"])
    counts = [z[f"s{s}_x"].size for s in range(ns)]
    sim = Simulation(cfg, load=False, capacity=[max(int(n * capacity_factor) + 1024, 1024) for n in counts],
                     **sim_kw)
    try:
        for s in range(ns):
            f = {k: np.ascontiguousarray(z[f"s{s}_{k}"]) for k in ("x", "y", "vx", "vy", "vz", "loc", "id")}
            sim.upload(s, f["x"], f["y"], f["vx"], f["vy"], f["vz"], f["loc"].astype(np.int32),
                       f["id"].astype(np.uint32))
            api.check(sim.lib.pic_set_next_id(s, int(z[f"s{s}_next_id"])), "pic_set_next_id")
        sim.set_field("phi", np.ascontiguousarray(z["phi"]))
        api.check(sim.lib.pic_get_efield_ppr(None, None), "pic_get_efield_ppr")
        sim.step_index = int(z["step"])
    except Exception:
        sim.close()
        raise
    return sim
