"""Device diagnostics (pic_average_x, pic_energy_spectrum,
pic_velocity_moments, the Ek_tot node field) against the oracle, through the
C-ABI, on the FP64 and the mixed-precision particle layouts.

Bars: bit-exact for Ek_tot, the Average_x column means (each column summed in
node order on both sides), and every histogram count; the velocity moments
within 1e-12 relative (FP64 atomic sums on the device, in an order that
varies; sequential on the CPU).  The x column of Average_x within 1e-15
relative.  The reference has no stored outputs of these routines, so the
oracle is checked against a direct transcription of the reference loops in
test_diagnostics_cpu.py.
"""
import numpy as np
import pytest

import oracle_bind as ob
from pic_b200 import api, deck, output
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

PRECISIONS = [api.PIC_PREC_FP64, api.PIC_PREC_MIXED]


def _evolved(name="tiny", prec=api.PIC_PREC_FP64, steps=4, **over):
    """A simulation a few steps in, with energy deposited on the last step."""
    sim = Simulation(deck.config(name, precision=prec, diag_interval=1, **over))
    sim.initial_fields()
    for _ in range(steps):
        sim.step()
    return sim


def test_ek_tot_bit_exact():
    sim = Simulation(deck.config("tiny"))
    try:
        sim.get_par_chg()
        for s, tag in enumerate(("e", "i")):
            parts = _oracle_parts(sim, s)
            _, e, bad = ob.deposit(sim.mesh.ptr, parts, sim.species[s][1], sim.scales["v_ref"], sim.mesh.nn)
            assert bad == 0
            want = ob.ek_tot(sim.mesh.ptr, e, sim.species[s][2], sim.scales["L_ref"], sim.cfg.n0, sim.mesh.nn)
            got = sim.field("ektot_" + tag)
            assert np.array_equal(got, want)
            assert np.count_nonzero(got) > 0
    finally:
        sim.close()


def _oracle_parts(sim, s):
    x, y, vx, vy, vz = [a.copy() for a in sim.particles0[s]]
    loc = np.array([ob.load().or_locate(sim.mesh.ptr, a, b) for a, b in zip(x, y)], np.int32)
    return {"x": x, "y": y, "vx": vx, "vy": vy, "vz": vz, "loc": loc}


@pytest.mark.parametrize("prec", PRECISIONS)
def test_average_x_bit_exact(prec):
    sim = _evolved(prec=prec)
    try:
        got = sim.average_x()
        nnx, nny = sim.mesh.nnx, sim.mesh.nny
        sc = sim.scales
        src = {"Phi": ("phi", sc["Phi_ref"]), "Rho": ("rho", sim.cfg.n0),
               "Rho_ele": ("rho_e", sim.cfg.n0), "Rho_ion": ("rho_i", sim.cfg.n0),
               "Ek_ele": ("ek_e", 1.0), "Ek_ion": ("ek_i", 1.0),
               "Ek_tot_ele": ("ektot_e", 1.0), "Ek_tot_ion": ("ektot_i", 1.0)}
        assert list(got) == ["x"] + list(src)
        for col, (field, scale) in src.items():
            want = ob.average_x(sim.field(field), nnx, nny, scale)
            assert np.array_equal(got[col], want), col
            assert np.any(got[col] != 0.0), col
        d = sim.mesh.desc
        xs = d.xmin + sim.mesh.hx * np.arange(nnx)
        assert np.allclose(got["x"], xs * sc["L_ref"], rtol=1e-15, atol=0.0)
    finally:
        sim.close()


def _live(sim, s):
    p = sim.download(s)
    return {k: np.ascontiguousarray(v) for k, v in p.items()}


@pytest.mark.parametrize("prec", PRECISIONS)
def test_energy_spectrum_bit_exact(prec):
    sim = _evolved(prec=prec)
    try:
        for s in range(2):
            parts = _live(sim, s)
            mass = sim.species[s][1]
            vref = sim.scales["v_ref"]
            e = 0.5 * mass * (parts["vx"] ** 2 + parts["vy"] ** 2 + parts["vz"] ** 2) * vref * vref / 1.6022e-19
            cases = [(100, 5.0, (10.0, 0.1)[s]),                       # the reference's settings
                     (7, float(np.quantile(e, 0.9)), float(np.abs(parts["vx"]).max()) * 1.5),
                     (256, float(e.max()), float(np.abs(parts["vx"]).max()) * 0.5)]
            for nbins, e_max, v_max in cases:
                ce, cv = sim.energy_spectrum(s, nbins, e_max, v_max)
                oe, ov = ob.energy_spectrum(parts, mass, vref, nbins, e_max, v_max)
                assert np.array_equal(ce, oe), (s, nbins)
                assert np.array_equal(cv, ov), (s, nbins)
                assert ce.sum() <= parts["vx"].size and cv.sum() <= parts["vx"].size
            assert ce.sum() == np.count_nonzero(e > 0.0)  # e_max = the largest energy
    finally:
        sim.close()


@pytest.mark.parametrize("prec", PRECISIONS)
def test_velocity_moments_match_oracle(prec):
    sim = _evolved(prec=prec)
    try:
        for s in range(2):
            parts = _live(sim, s)
            for nbins in (1024, 9):
                cnt, drift, thermal = sim.velocity_moments(s, nbins)
                oc, od, ot = ob.velocity_moments(parts, nbins)
                assert np.array_equal(cnt, oc), (s, nbins)
                assert cnt.sum() == parts["x"].size
                for g, o in ((drift, od), (thermal, ot)):
                    tol = 1e-12 * np.abs(o).max(axis=1, keepdims=True)
                    assert np.all(np.abs(g - o) <= tol), (s, nbins)
                assert np.all(drift[:, cnt == 0] == 0.0) and np.all(thermal[:, cnt == 0] == 0.0)
    finally:
        sim.close()


def test_diagnostics_reject_bad_arguments():
    sim = Simulation(deck.config("tiny"))
    try:
        c = np.zeros(8, np.int64)
        v = np.zeros(24)
        lib = sim.lib
        assert lib.pic_energy_spectrum(2, 8, 5.0, 1.0, api.lptr(c), api.lptr(c)) == api.PIC_ERR_ARG
        assert lib.pic_energy_spectrum(0, 0, 5.0, 1.0, api.lptr(c), api.lptr(c)) == api.PIC_ERR_ARG
        assert lib.pic_energy_spectrum(0, 8, -1.0, 1.0, api.lptr(c), api.lptr(c)) == api.PIC_ERR_ARG
        assert lib.pic_velocity_moments(0, 4096, api.lptr(c), api.dptr(v), api.dptr(v)) == api.PIC_ERR_ARG
        assert lib.pic_average_x(None) == api.PIC_ERR_ARG
        # the library still works after the rejected calls
        ce, _ = sim.energy_spectrum(0, 8, 5.0, 10.0)
        assert ce.sum() > 0
    finally:
        sim.close()


def test_output_files(tmp_path):
    sim = _evolved(steps=2)
    try:
        prof = output.write_average_x(sim, str(tmp_path / "Field" / "Average_x_000002.dat"))
        tab = np.loadtxt(tmp_path / "Field" / "Average_x_000002.dat", skiprows=3)
        assert tab.shape == (sim.mesh.nnx, 9)
        assert np.array_equal(tab[:, 1], prof["Phi"])
        de, dv = output.write_energy(sim, str(tmp_path / "Energy" / "energy_IJ2_000002.dat"))
        tab = np.loadtxt(tmp_path / "Energy" / "energy_IJ2_000002.dat", skiprows=2)
        assert tab.shape == (100, 2 + 1 + 3 + 2)
        assert np.array_equal(tab[:, 0], de[0]) and np.array_equal(tab[:, -1], dv[1])
        mom = output.write_velocity(sim, str(tmp_path / "Velocity" / "velocity_IJ_3000002.dat"))
        tab = np.loadtxt(tmp_path / "Velocity" / "velocity_IJ_3000002.dat")
        assert tab.shape == (1024, 7)
        assert np.array_equal(tab[:, 4], mom[0][0].astype(float))
        for it in (1, 2):
            output.append_partcount(sim, it, str(tmp_path / "PartcountReal.dat"))
        tab = np.loadtxt(tmp_path / "PartcountReal.dat")
        assert tab.shape == (2, 4) and tab[1, 1] == tab[1, 2] + tab[1, 3]
    finally:
        sim.close()
