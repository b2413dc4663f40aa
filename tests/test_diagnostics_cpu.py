"""The oracle's diagnostics (or_energy_spectrum, or_velocity_moments,
or_average_x) against a line-by-line Python transcription of the reference
loops, and the file writers against a stand-in simulation.  CPU only.

Reference loops: Output_Energy.f90:41-71 (bin edges with REAL(i), i.e. single
precision integers, each particle tested against every bin), OUTPUT_velocity.f90
:48-103, Output_To_Tecplot_IJK_2D.f90:184-215.
"""
import math

import numpy as np

import oracle_bind as ob
from pic_b200 import output

JTOEV = 1.6022e-19


def _f32(v):
    return float(np.float32(v))


def _ref_energy(parts, mass, vref, n, ek_max, vk_max):
    """Output_Energy.f90:41-71, transcribed."""
    ek_per = [ek_max * _f32(i) / n for i in range(n + 1)]
    vk_per = [vk_max * _f32(np.float32(i) - np.float32(0.5) * np.float32(n)) / n for i in range(n + 1)]
    n_per, nv_per = [0] * n, [0] * n
    for vx, vy, vz, loc in zip(parts["vx"], parts["vy"], parts["vz"], parts["loc"]):
        if loc < 0:
            continue
        ek = 0.5 * mass * (vx * vx + vy * vy + vz * vz)
        ek = ek * vref * vref / JTOEV
        for i in range(1, n + 1):
            if ek_per[i - 1] < ek <= ek_per[i]:
                n_per[i - 1] += 1
            if vk_per[i - 1] < vx <= vk_per[i]:
                nv_per[i - 1] += 1
    return np.array(n_per), np.array(nv_per)


def _ref_velocity(parts, n):
    """OUTPUT_velocity.f90:48-103, transcribed (in double precision)."""
    tot = np.zeros((3, n))
    num = np.zeros(n, np.int64)
    live = [k for k in range(parts["x"].size) if parts["loc"][k] >= 0]
    bins = {k: min(max(1, math.floor(parts["x"][k]) + 1), n) - 1 for k in live}
    comps = (parts["vx"], parts["vy"], parts["vz"])
    for k in live:
        for c in range(3):
            tot[c, bins[k]] += comps[c][k]
        num[bins[k]] += 1
    drift = np.zeros((3, n))
    for b in range(n):
        if num[b]:
            drift[:, b] = tot[:, b] / num[b]
    var = np.zeros((3, n))
    for k in live:
        for c in range(3):
            var[c, bins[k]] += (comps[c][k] - drift[c, bins[k]]) ** 2
    thermal = np.zeros((3, n))
    for b in range(n):
        if num[b]:
            thermal[:, b] = np.sqrt(var[:, b] / num[b])
    return num, drift, thermal


def _parts(n=3000, seed=5, vmax=2.0, nbins=100):
    rng = np.random.default_rng(seed)
    vx = rng.normal(0.0, vmax / 3, n)
    # particles exactly on vx bin edges, at zero velocity (energy 0: no
    # energy bin) and one dead slot
    edges = np.array([vmax * _f32(np.float32(i) - np.float32(0.5) * np.float32(nbins)) / nbins
                      for i in (0, 1, 37, 50, 99, 100)])
    vx[:edges.size] = edges
    vy = rng.normal(0.0, vmax / 3, n)
    vz = rng.normal(0.0, vmax / 3, n)
    vx[10] = vy[10] = vz[10] = 0.0
    loc = np.zeros(n, np.int32)
    loc[11] = -1
    x = rng.uniform(-0.5, 40.5, n)
    x[:4] = [0.0, 1.0, 39.0, 39.999999]
    return {"x": x, "vx": vx, "vy": vy, "vz": vz, "loc": loc}


def test_oracle_energy_spectrum_is_the_reference_loop():
    mass, vref = 9.1095e-31, 5.9e5
    p = _parts()
    e = 0.5 * mass * (p["vx"] ** 2 + p["vy"] ** 2 + p["vz"] ** 2) * vref * vref / JTOEV
    for nbins, e_max, v_max in ((100, 5.0, 2.0), (7, float(np.median(e)), 1.3), (100, float(e.max()), 2.0)):
        oe, ov = ob.energy_spectrum(p, mass, vref, nbins, e_max, v_max)
        re, rv = _ref_energy(p, mass, vref, nbins, e_max, v_max)
        assert np.array_equal(oe, re) and np.array_equal(ov, rv), nbins
        assert oe.sum() > 0 and ov.sum() > 0
    # the edge particles land in the bin whose upper edge they are
    _, ov = ob.energy_spectrum(p, mass, vref, 100, 5.0, 2.0)
    _, rv = _ref_energy({k: v[:6] for k, v in p.items()}, mass, vref, 100, 5.0, 2.0)
    assert rv.sum() == 5 and rv[0] == 1 and rv[36] == 1 and rv[49] == 1 and rv[98] == 1 and rv[99] == 1


def test_oracle_velocity_moments_are_the_reference_loop():
    p = _parts()
    for nbins in (40, 1024, 3):
        oc, od, ot = ob.velocity_moments(p, nbins)
        rc, rd, rt = _ref_velocity(p, nbins)
        assert np.array_equal(oc, rc)
        assert oc.sum() == p["x"].size - 1
        assert np.allclose(od, rd, rtol=1e-13, atol=1e-15)
        assert np.allclose(ot, rt, rtol=1e-13, atol=1e-15)


def test_oracle_average_x_is_the_reference_loop():
    rng = np.random.default_rng(2)
    nnx, nny = 9, 13
    f = rng.standard_normal(nnx * nny)
    got = ob.average_x(f, nnx, nny, 3.5)
    want = []
    for i in range(nnx):
        s, cnt = 0.0, 0
        for j in range(nny):
            s += f[i * nny + j]
            cnt += 1
        want.append(s / cnt * 3.5)
    assert np.array_equal(got, np.array(want))


class _FakeMesh:
    nnx = 5


class _FakeSim:
    """Duck-typed Simulation: what the writers read."""
    species = [(-1.0, 1.0, 2.0), (1.0, 1836.0, 2.0)]
    mesh = _FakeMesh()

    def average_x(self):
        names = ["x", "Phi", "Rho", "Rho_ele", "Rho_ion", "Ek_ele", "Ek_ion", "Ek_tot_ele", "Ek_tot_ion"]
        return {n: np.arange(5) * (k + 1) / 3.0 for k, n in enumerate(names)}

    def energy_spectrum(self, s, nbins, e_max, v_max):
        return np.arange(nbins, dtype=np.int64) + s, np.full(nbins, 2 + s, np.int64)

    def velocity_moments(self, s, nbins):
        return (np.full(nbins, 3 + s, np.int64), np.full((3, nbins), 0.5 + s), np.full((3, nbins), 0.25 + s))

    def particle_totals(self):
        return 7.0 + 9.0, [7.0, 9.0]


def test_writers_layout(tmp_path):
    sim = _FakeSim()
    output.write_average_x(sim, str(tmp_path / "a.dat"))
    lines = open(tmp_path / "a.dat").read().splitlines()
    assert lines[0].strip() == 'TITLE = "Field Plot"'
    assert '"Ek_tot_ion"' in lines[1] and lines[2].split() == ["ZONE", "I", "=", "5"]
    tab = np.loadtxt(tmp_path / "a.dat", skiprows=3)
    assert tab.shape == (5, 9) and np.array_equal(tab[:, 4], np.arange(5) * 5 / 3.0)

    de, dv = output.write_energy(sim, str(tmp_path / "e.dat"))
    tab = np.loadtxt(tmp_path / "e.dat", skiprows=2)
    assert tab.shape == (100, 8)
    assert np.array_equal(tab[:, 0], output.K_ENERGY * np.arange(100) / output.N_INI)
    assert np.array_equal(tab[:, 2], output.EK_MAX * np.arange(100) / 100)
    assert tab[0, 3] == -output.VK_MAX[0] / 2 and tab[50, 4] == 0.0
    assert np.array_equal(tab[:, 7], np.full(100, output.K_V[1] * 3 / output.N_INI))

    output.write_velocity(sim, str(tmp_path / "v.dat"))
    tab = np.loadtxt(tmp_path / "v.dat")
    assert tab.shape == (output.VELOCITY_BINS, 7)
    assert np.all(tab[:, 0] == 0.5) and np.all(tab[:, 3] == 1.25) and np.all(tab[:, 5] == 4)
    assert np.array_equal(tab[:, 6], np.arange(1, output.VELOCITY_BINS + 1))

    for it in (1, 2000):
        output.append_partcount(sim, it, str(tmp_path / "p.dat"))
    tab = np.loadtxt(tmp_path / "p.dat")
    assert tab.tolist() == [[1, 16, 7, 9], [2000, 16, 7, 9]]
