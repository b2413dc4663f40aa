"""MCC_jw collision tables for e-Ar and Ar+-Ar.

Restates the table set-up of the reference:
  grid ................ mc/MCCSigma.f90:9-11, SigmaNormalizedInit (log10 E grid,
                        electrons: 10001 points over [-3, 3]; non-reactive ions
                        (model 2): 10001 points over [-1, 3])
  sigma(E) ............ SigmaNormalizedUpdate (mc/MCCSigma.f90:123-172): linear
                        interpolation in grid-index space between the raw
                        points, 0 at or below threshold, Alfa/E above the last
                        raw energy, raw sigma converted cm^2 -> m^2
                        (ReactionOnePegasus.f90:448)
  probability ......... ProbilityNonReactive (mc/MCCInit.F90:107-152):
                        nu = sigma*v*n_gas cumulated over reactions and
                        normalised by its maximum nu_max
  P_null .............. CollisionRatio = 1 - exp(-nu_max*dt) (MCCInit.F90:54)
  reaction types ...... ConvertReactionOneBase2ReactionOne
                        (ReactionOnePegasus.f90:151-300): e- elastic 1 -> 11,
                        excitation 100 -> 12, ionisation 2 -> 13; ion elastic
                        1 -> 101, charge exchange 6 -> 103.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import api
from .deck import AR_MASS, KB, ME, QE

JTOEV = 1.6022e-19
DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "ar_pegasus.json")

ELECTRON_TYPES = {1: 11, 100: 12, 2: 13}
ION_TYPES = {1: 101, 6: 103}


def _locate(xx: np.ndarray, x: float) -> int:
    """Numerical Recipes bisection `locate` (MCC_jw/code/base/Numrical.F90:157-184),
    1-based result."""
    n = xx.size
    jl, ju = 0, n + 1
    asc = xx[n - 1] >= xx[0]
    while ju - jl > 1:
        jm = (ju + jl) // 2
        if asc == (x >= xx[jm - 1]):
            jl = jm
        else:
            ju = jm
    if x == xx[0]:
        return 1
    if x == xx[n - 1]:
        return n - 1
    return jl


def sigma_table(reaction: dict, emin: float, eint: float, nsigma: int) -> np.ndarray:
    raw = np.array(reaction["table"], dtype=np.float64)
    e_raw = raw[:, 0].copy()
    s_raw = raw[:, 1] / 1.0e4
    thr = reaction["threshold"]
    nraw = int(np.argmax(e_raw)) + 1      # Maxloc of the raw energies
    max_energy = e_raw[nraw - 1]
    alfa = s_raw[nraw - 1] * max_energy
    idx = np.empty(nraw)
    for i in range(nraw):
        if e_raw[i] < 10.0 ** emin:
            idx[i] = emin                  # as written in SigmaNormalizedUpdate
        else:
            idx[i] = (math.log10(e_raw[i]) - emin) / eint
    out = np.zeros(nsigma)
    for i in range(1, nsigma + 1):
        energy = 10.0 ** (emin + (i - 1) * eint)
        if energy <= thr:
            out[i - 1] = 0.0
        elif energy >= max_energy:
            out[i - 1] = alfa / energy
        else:
            k = _locate(idx, float(i - 1))
            if k < 1:
                k = 1
            le, ue = idx[k - 1], idx[k]
            s1 = (float(i) - le) / (ue - le)
            s2 = 1.0 - s1
            out[i - 1] = s2 * s_raw[k - 1] + s1 * s_raw[k]
    return out


def build_table(bundle: dict, species: int, mass: float, gas_mass: float, n_gas: float,
                dt_s: float, resultant: int, ion: bool):
    model = bundle["model"]
    nsigma = 10001
    if model == 1:
        emin, emax = -3.0, 3.0
    else:
        emin, emax = -1.0, 3.0
    eint = (emax - emin) / (nsigma - 1)
    reactions = bundle["reactions"]
    nr = len(reactions)
    sig = np.stack([sigma_table(r, emin, eint, nsigma) for r in reactions])  # [nr, ns]
    miu = mass * gas_mass / (mass + gas_mass)
    # 10^x per point through libm's pow, as the reference's 10.d0**x: numpy's
    # vectorised power differs from it by an ulp at some grid energies
    energy = np.array([math.pow(10.0, emin + i * eint) for i in range(nsigma)])
    v = np.sqrt(2.0 * energy * JTOEV / miu)
    prob = sig * v[None, :] * n_gas
    prob = np.cumsum(prob, axis=0)
    pmax = float(prob.max())
    prob = prob / pmax
    t = api.MccTable()
    t.species = species
    t.n_reaction = nr
    t.n_sigma = nsigma
    t.energy_min = emin
    t.energy_interval = eint
    t.energy_max = 10.0 ** emax
    t.collision_ratio = 1.0 - math.exp(-pmax * dt_s)
    types = ION_TYPES if ion else ELECTRON_TYPES
    for k, r in enumerate(reactions):
        t.reaction_type[k] = types[r["pegasus_type"]]
        t.threshold[k] = r["threshold"]
        t.resultant[k] = resultant if t.reaction_type[k] == 13 else -1
    arr = np.ascontiguousarray(prob.T)  # [ns][nr]
    t.probability = api.dptr(arr)
    return t, arr, pmax


def ar_tables(cfg, dt_s: float):
    """(gas, [tables], keepalive) for e- (species 0) and Ar+ (species 1)."""
    with open(DATA) as f:
        data = json.load(f)
    n_gas = cfg.gas_p_Pa / (KB * cfg.gas_T_K)
    gas = api.Gas(AR_MASS, cfg.gas_T_K, n_gas)
    te, ae, _ = build_table(data["electron"], 0, ME, AR_MASS, n_gas, dt_s, 1, False)
    ti, ai, _ = build_table(data["ion"], 1, AR_MASS, AR_MASS, n_gas, dt_s, -1, True)
    return gas, [te, ti], [ae, ai]
