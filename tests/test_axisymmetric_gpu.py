"""GPU parity of the axisymmetric (r-z, delta = 1) path against the CPU
oracle, through the C-ABI, on the tiny r-z deck (a dielectric torus in a
cylinder): the push in the particle's own frame (MoveOne.f90:213-263), the
r-weighted deposit with the axis-row factor (GetParChg_2D.f90:803-821), the
RHS from the per-row load matrices and the Jacobi-PCG solve, all bit-exact
on the FP64 path.  The full step (with MCC and the sort) is covered by the
multi-step oracle comparison in test_gpu_parity.py."""
import numpy as np
import pytest

import oracle_bind as ob
from pic_b200 import deck
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def _sim(**over):
    return Simulation(deck.config("tiny_axi", **over))


def _by_id(p):
    o = np.argsort(p["id"])
    return {k: v[o] for k, v in p.items()}


def _oracle_parts(sim, s):
    x, y, vx, vy, vz = [a.copy() for a in sim.particles0[s]]
    loc = np.array([ob.load().or_locate(sim.mesh.ptr, a, b) for a, b in zip(x, y)], np.int32)
    return {"x": x, "y": y, "vx": vx, "vy": vy, "vz": vz, "loc": loc, "id": np.arange(x.size, dtype=np.uint32)}


@pytest.mark.parametrize("species", [0, 1])
def test_axi_move_all_bit_exact(species):
    sim = _sim()
    try:
        rng = np.random.default_rng(21)
        nn = sim.mesh.nn
        efx, efy = rng.standard_normal(nn) * 5.0, rng.standard_normal(nn) * 5.0
        coef = rng.standard_normal((5, nn)) * 5.0
        sim.set_field("efx", efx)
        sim.set_field("efy", efy)
        for k in range(5):
            sim.set_field("c%d" % (k + 2), coef[k])
        sim.move_all(species)
        g = _by_id(sim.download(species))
        o = _oracle_parts(sim, species)
        qm = sim.species[species][0] / (sim.species[species][1] / deck.ME)
        lost = ob.move_all_axi(sim.mesh.ptr, o, efx, efy, np.ascontiguousarray(coef.ravel()), qm, sim.cfg.dt)
        live = o["loc"] >= 0
        assert sim.count(species) == int(live.sum()) == o["x"].size - lost
        for k in ("x", "y", "vx", "vy", "vz", "loc"):
            assert np.array_equal(g[k], o[k][live]), k
        assert np.all(g["y"] >= 0.0)
    finally:
        sim.close()


def test_axi_get_par_chg_bit_exact():
    sim = _sim()
    try:
        rho = np.zeros(sim.mesh.nn)
        sim.get_par_chg(rho)
        qs, es, wq = [], [], []
        for s in range(2):
            o = _oracle_parts(sim, s)
            q, e, bad = ob.deposit(sim.mesh.ptr, o, sim.species[s][1], sim.scales["v_ref"], sim.mesh.nn)
            assert bad == 0
            qs.append(q)
            es.append(e)
            wq.append(sim.species[s][2] * sim.species[s][0])
        r, rs, ek = ob.normalize(sim.mesh.ptr, qs, es, wq, sim.scales["L_ref"], sim.cfg.n0, sim.mesh.nn)
        assert np.array_equal(rho, r)
        assert np.array_equal(sim.field("rho_e"), rs[0]) and np.array_equal(sim.field("rho_i"), rs[1])
        assert np.array_equal(sim.field("ek_e"), ek[0]) and np.array_equal(sim.field("ek_i"), ek[1])
    finally:
        sim.close()


def test_axi_ife_solve_bit_exact():
    sim = _sim()
    try:
        rng = np.random.default_rng(6)
        nn = sim.mesh.nn
        rho = rng.standard_normal(nn) * 0.05
        sim.set_field("rho", rho)
        phi0 = sim.mesh.array("phi_dirichlet").copy()
        phi = phi0.copy()
        st = sim.ife_solve(phi)
        b = ob.rhs(sim.mesh.ptr, rho, nn)
        assert np.array_equal(sim.field("b"), b)
        po, so = ob.pcg(sim.mesh.ptr, b, phi0, sim.cfg.pcg_tol, sim.cfg.pcg_maxit)
        assert st.ierr == 0 and so["ierr"] == 0
        assert st.iterations == so["iterations"]
        assert np.array_equal(phi, po)
    finally:
        sim.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cfg5_geometry_steps_with_the_rf_electrode(precision):
    """The config-5 cell (r-z, RF electrode at z = 0, dielectric wafer) at a
    reduced mesh and particle count: steps solve, keep every particle off
    the axis' far side (r >= 0) and drive the electrode at 200 V sin(2 pi f t)."""
    import math
    prec = deck.api.PIC_PREC_MIXED if precision == "mixed" else deck.api.PIC_PREC_FP64
    cfg = deck.config("cfg5", ncx=512, ncy=100, ppc=4, nt=5, precision=prec)
    cfg.objects = [deck.ObjectSpec(deck.api.PIC_SHAPE_BOX, 0.010, -0.001, 0.011, 0.0755, eps=3.9)]
    sim = Simulation(cfg)
    try:
        assert sim.initial_fields().ierr == 0
        static = sim.mesh.array("phi_dirichlet").copy()
        amp = 200.0 / sim.scales["Phi_ref"]
        w = 2.0 * math.pi * 13.56e6 * sim.scales["time_ref"]
        for k in range(1, 6):
            st = sim.step()
            assert st.solve.ierr == 0, k
            phi = sim.field("phi")
            left = np.arange(sim.mesh.nny)
            assert np.allclose(phi[left] - static[left], amp * math.sin(w * k * cfg.dt), rtol=0, atol=1e-9)
        for s in range(2):
            p = sim.download(s)
            assert p["y"].size > 0 and np.all(p["y"] >= 0.0) and np.all(np.isfinite(p["vz"]))
    finally:
        sim.close()


def _both_prec(fn, **over):
    out = []
    for prec in (deck.api.PIC_PREC_FP64, deck.api.PIC_PREC_MIXED):
        sim = Simulation(deck.config("tiny_axi", precision=prec, **over))
        try:
            out.append(fn(sim))
        finally:
            sim.close()
    return out


def test_axi_mixed_push_and_deposit_match_fp64():
    """The mixed-precision r-z push (element + FP32 offsets, FP64 radial
    move) against the FP64 one after one push: positions within 1e-5 of a
    cell, velocities (v_theta included) within 1e-5 relative; node charge
    within 1e-4 of the largest, before and after."""
    def fn(sim):
        sim.initial_fields()
        rho0 = sim.field("rho")
        for s in range(2):
            sim.move_all(s)
        sim.get_par_chg()
        return rho0, sim.field("rho"), [_by_id(sim.download(s)) for s in range(2)], sim.mesh.hy

    (r0d, r1d, pd, hy), (r0m, r1m, pm, _) = _both_prec(fn)
    assert np.abs(r0d - r0m).max() <= 1e-6 * np.abs(r0d).max()
    assert np.abs(r1d - r1m).max() <= 1e-4 * np.abs(r1d).max()
    for a, b in zip(pd, pm):
        common, ia, ib = np.intersect1d(a["id"], b["id"], return_indices=True)
        assert common.size >= 0.999 * max(a["id"].size, b["id"].size)
        assert np.abs(a["x"][ia] - b["x"][ib]).max() <= 1e-5 * hy
        assert np.abs(a["y"][ia] - b["y"][ib]).max() <= 1e-5 * hy
        for v in ("vx", "vy", "vz"):
            assert np.allclose(a[v][ia], b[v][ib], rtol=1e-5, atol=1e-5 * np.abs(a[v]).max()), v


def test_axi_mixed_steps_track_fp64():
    def fn(sim):
        sim.initial_fields()
        for _ in range(10):
            sim.step()
        return {f: sim.field(f) for f in ("phi", "efx", "efy")}, [sim.count(s) for s in range(2)]

    (fd, nd), (fm, nm) = _both_prec(fn, ppc=40)
    for f in ("phi", "efx", "efy"):
        err = np.abs(fd[f] - fm[f]).max() / np.abs(fd[f]).max()
        assert err <= 1e-2, f
    for a, b in zip(nd, nm):
        assert abs(a - b) <= 0.01 * a


@pytest.mark.parametrize("bulk", ["0", "1"])
def test_axi_tiled_push_matches_direct(bulk, monkeypatch):
    """The r-z push with tiles (cp.async, or bulk copies on mbarriers) is
    bit-identical to the one-particle-per-thread kernel over 5 steps."""
    monkeypatch.setenv("PIC_PUSH_BULK", bulk)

    def fn(sim):
        sim.initial_fields()
        for _ in range(5):
            sim.step()
        return [_by_id(sim.download(s)) for s in range(2)], sim.field("rho"), sim.field("phi")

    out = []
    for st in ("0", "4"):
        monkeypatch.setenv("PIC_PUSH_STAGES", st)
        sim = Simulation(deck.config("tiny_axi", precision=deck.api.PIC_PREC_MIXED))
        try:
            out.append(fn(sim))
        finally:
            sim.close()
    (pa, ra, fa), (pb, rb, fb) = out
    for a, b in zip(pa, pb):
        for k in ("id", "loc", "x", "y", "vx", "vy", "vz"):
            assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(ra, rb) and np.array_equal(fa, fb)
