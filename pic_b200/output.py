"""ASCII writers for the reference's diagnostic files, fed by the device-side
diagnostics of Simulation (only the small results cross to the host):

    write_average_x   OUTPUT/Field/Average_x_<it>.dat      Output_To_Tecplot_IJK_2D.f90:217-226
    write_energy      OUTPUT/Energy/energy_IJ2_<it>.dat    Output_Energy.f90:74-108
    write_velocity    OUTPUT/Velocity/velocity_IJ_3<it>.dat OUTPUT_velocity.f90:131-139
    append_partcount  OUTPUT/PartcountReal.dat              Main_IFE_Test_2.f90:473-499

Same header lines and columns as the reference; numbers are written with
%.16e (17 significant digits: they read back exactly) rather
than the Fortran edit descriptors.
"""
from __future__ import annotations

import os

import numpy as np

# Output_Energy.f90:20-35
ENERGY_BINS = 100
EK_MAX = 5.0
VK_MAX = (10.0, 0.1, 0.01)
K_ENERGY = 10.0
K_V = (20.0, 1000.0, 10000.0)
N_INI = 4000 * 4 * 128
# OUTPUT_velocity.f90:47
VELOCITY_BINS = 1024


def _open(path):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    return open(path, "w")


def write_average_x(sim, path: str) -> dict:
    prof = sim.average_x()
    names = list(prof)
    with _open(path) as f:
        f.write(' TITLE = "Field Plot"\n')
        f.write(" VARIABLES = " + " ".join('"%s"' % n for n in names) + "\n")
        f.write(" ZONE I = %6d\n" % sim.mesh.nnx)
        for row in np.stack([prof[n] for n in names], axis=1):
            f.write(" ".join("%.16e" % v for v in row) + "\n")
    return prof


def energy_tables(sim):
    """dN/dE and dN/dV per species with the reference's constants, and the
    bin edges it writes beside them."""
    ns = len(sim.species)
    n = ENERGY_BINS
    de, dv = [], []
    for s in range(ns):
        ce, cv = sim.energy_spectrum(s, n, EK_MAX, VK_MAX[min(s, 2)])
        de.append(K_ENERGY * ce / N_INI)
        dv.append(K_V[min(s, 2)] * cv / N_INI)
    i = np.arange(n)
    e_edge = EK_MAX * i.astype(np.float32).astype(np.float64) / n
    v_edge = [vm * (i.astype(np.float32) - np.float32(0.5 * n)).astype(np.float64) / n for vm in VK_MAX]
    return de, dv, e_edge, v_edge


def write_energy(sim, path: str):
    de, dv, e_edge, v_edge = energy_tables(sim)
    ns = len(de)
    with _open(path) as f:
        f.write(' TITLE = "EnergySpectrum Plot"\n')
        f.write(' VARIABLES = "dN/dE_ele" "dN/dE_ion" "E" "V1" "V2" "dN/dV_ele" "dN/dV_ion" \n')
        for b in range(ENERGY_BINS):
            cols = [de[s][b] for s in range(ns)] + [e_edge[b]] + [v[b] for v in v_edge] + \
                   [dv[s][b] for s in range(ns)]
            f.write("     ".join("%.16e" % v for v in cols) + "\n\n")
    return de, dv


def write_velocity(sim, path: str):
    ns = len(sim.species)
    mom = [sim.velocity_moments(s, VELOCITY_BINS) for s in range(ns)]
    with _open(path) as f:
        for b in range(VELOCITY_BINS):
            cols = [m[1][0, b] for m in mom] + [m[2][0, b] for m in mom] + [float(m[0][b]) for m in mom]
            f.write("     ".join("%.16e" % v for v in cols) + "     %5d\n" % (b + 1))
    return mom


def append_partcount(sim, it: int, path: str):
    ntot, per = sim.particle_totals()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "a") as f:
        f.write(" %d %.16e " % (it, ntot) + " ".join("%.16e" % v for v in per) + "\n")
    return ntot, per
