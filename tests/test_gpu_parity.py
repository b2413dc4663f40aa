"""GPU parity of every kernel of the step against the CPU oracle, through the
C-ABI (libpicgpu.so), on seeded inputs at sizes the oracle finishes quickly.

Bars: bit-exact for cell ids, sort order, deposits (int64 fixed point),
collision selection and particle counts; phase space, rho, phi, E within
1e-10 relative on the FP64 path (most comparisons below are bit-exact).
"""
import ctypes as C

import numpy as np
import pytest

import oracle_bind as ob
from pic_b200 import api, deck
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def _sim(name="tiny", **over):
    cfg = deck.config(name, **over)
    return Simulation(cfg)


def _by_id(p):
    o = np.argsort(p["id"])
    return {k: v[o] for k, v in p.items()}


def _oracle_parts(sim, s):
    x, y, vx, vy, vz = [a.copy() for a in sim.particles0[s]]
    n = x.size
    loc = np.zeros(n, np.int32)
    for k in range(n):
        loc[k] = ob.load().or_locate(sim.mesh.ptr, x[k], y[k])
    return {"x": x, "y": y, "vx": vx, "vy": vy, "vz": vz, "loc": loc,
            "id": np.arange(n, dtype=np.uint32)}


def test_upload_locate_matches_oracle():
    sim = _sim()
    try:
        for s in range(2):
            g = _by_id(sim.download(s))
            o = _oracle_parts(sim, s)
            assert np.array_equal(g["loc"], o["loc"])
            assert np.array_equal(g["x"], o["x"]) and np.array_equal(g["vz"], o["vz"])
    finally:
        sim.close()


def _random_fields(sim, seed=1, scale=0.2):
    rng = np.random.default_rng(seed)
    nn = sim.mesh.nn
    efx = rng.standard_normal(nn) * scale
    efy = rng.standard_normal(nn) * scale
    coef = rng.standard_normal((5, nn)) * scale
    sim.set_field("efx", efx)
    sim.set_field("efy", efy)
    for k in range(5):
        sim.set_field("c%d" % (k + 2), coef[k])
    return efx, efy, np.ascontiguousarray(coef.ravel())


@pytest.fixture
def push64(request, monkeypatch):
    """FP64 push form: one particle per thread loaded directly, particle
    tiles staged through shared memory by per-thread cp.async copies, or by
    one thread's bulk copies completing on mbarriers (PIC_PUSH64_TILED
    0 / 1 / 2); all run the same per-particle code."""
    monkeypatch.setenv("PIC_PUSH64_TILED", {"direct": "0", "tiled": "1", "bulk": "2"}[request.param])
    return request.param


@pytest.mark.parametrize("push64", ["direct", "tiled", "bulk"], indirect=True)
@pytest.mark.parametrize("species", [0, 1])
def test_move_all_bit_exact(species, push64):
    sim = _sim()
    try:
        efx, efy, coef = _random_fields(sim, scale=5.0)
        sim.move_all(species)
        g = _by_id(sim.download(species))
        o = _oracle_parts(sim, species)
        qm = sim.species[species][0] / (sim.species[species][1] / deck.ME)
        lost = ob.move_all(sim.mesh.ptr, o, efx, efy, coef, qm, sim.cfg.dt)
        live = o["loc"] >= 0
        assert sim.count(species) == int(live.sum()) == o["x"].size - lost
        for k in ("x", "y", "vx", "vy", "loc"):
            assert np.array_equal(g[k], o[k][live]), k
    finally:
        sim.close()


def test_get_par_chg_bit_exact():
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
        # charge conservation of the fixed-point deposit on a Cartesian mesh:
        # each particle adds exactly 2^40 (corner 2 takes the rest)
        for s in range(2):
            n = sim.count(s)
            assert int(qs[s].sum()) == n * (1 << 40)
    finally:
        sim.close()


@pytest.fixture
def pcg_mode(request, monkeypatch):
    monkeypatch.setenv("PIC_PCG_PERSISTENT", "0" if request.param == "two-kernel" else "1")
    monkeypatch.setenv("PIC_PCG_SMEM", "1" if request.param == "smem-resident" else "0")
    return request.param


@pytest.mark.parametrize("pcg_mode", ["smem-resident", "persistent", "two-kernel"], indirect=True)
@pytest.mark.parametrize("name", ["tiny", "cfg1"])
def test_ife_solve_bit_exact(name, pcg_mode):
    sim = _sim(name)
    try:
        rng = np.random.default_rng(5)
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
        assert st.rel_residual <= sim.cfg.pcg_tol
        # warm start from the solution converges at once
        st2 = sim.ife_solve(phi)
        assert st2.iterations <= 2
    finally:
        sim.close()


def test_pcg_barrier_wait_times_out_cleanly(monkeypatch):
    """The persistent PCG's grid barrier waits at most PIC_PCG_SPIN_LIMIT
    polls.  Expecting one arrival that never comes makes every CTA give up:
    the solve returns an error status and the context stays usable."""
    monkeypatch.setenv("PIC_PCG_PERSISTENT", "1")
    monkeypatch.setenv("PIC_PCG_BARRIER_EXTRA", "1")
    monkeypatch.setenv("PIC_PCG_SPIN_LIMIT", "20000")
    sim = _sim("tiny")
    try:
        sim.set_field("rho", np.full(sim.mesh.nn, 0.01))
        with pytest.raises(api.PicError) as ei:
            sim.ife_solve()
        assert ei.value.code == -2 and "timed out" in str(ei.value)
    finally:
        sim.close()
    monkeypatch.delenv("PIC_PCG_BARRIER_EXTRA")
    monkeypatch.delenv("PIC_PCG_SPIN_LIMIT")
    sim = _sim("tiny")
    try:
        sim.set_field("rho", np.full(sim.mesh.nn, 0.01))
        assert sim.ife_solve().ierr == 0
    finally:
        sim.close()


@pytest.mark.parametrize("name", ["tiny", "cfg1"])
def test_ppr_parity(name):
    sim = _sim(name)
    try:
        nn = sim.mesh.nn
        rng = np.random.default_rng(9)
        xs = np.repeat(np.arange(sim.mesh.nnx), sim.mesh.nny) * sim.mesh.hx
        ys = np.tile(np.arange(sim.mesh.nny), sim.mesh.nnx) * sim.mesh.hy
        phi = np.sin(0.1 * xs) * np.cos(0.07 * ys) + 0.01 * rng.standard_normal(nn)
        sim.set_field("phi", phi)
        efx = np.zeros(nn)
        efy = np.zeros(nn)
        sim.get_efield_ppr(efx, efy)
        coef, ox, oy = ob.ppr(sim.mesh.ptr, phi, nn)
        scale = max(np.abs(ox).max(), np.abs(oy).max())
        assert np.abs(efx - ox).max() <= 1e-10 * scale
        assert np.abs(efy - oy).max() <= 1e-10 * scale
        for k in range(5):
            gk = sim.field("c%d" % (k + 2))
            assert np.abs(gk - coef[k]).max() <= 1e-10 * max(1.0, np.abs(coef[k]).max())
    finally:
        sim.close()


def test_ppr_exact_for_quadratic():
    """PPR reproduces the gradient of a quadratic potential exactly
    (least-squares fit of a quadratic on every patch)."""
    sim = _sim("cfg1")
    try:
        nn = sim.mesh.nn
        xs = np.repeat(np.arange(sim.mesh.nnx), sim.mesh.nny) * sim.mesh.hx
        ys = np.tile(np.arange(sim.mesh.nny), sim.mesh.nnx) * sim.mesh.hy
        phi = 0.3 + 0.2 * xs - 0.1 * ys + 0.01 * xs * xs + 0.02 * xs * ys - 0.005 * ys * ys
        sim.set_field("phi", phi)
        efx = np.zeros(nn)
        efy = np.zeros(nn)
        sim.get_efield_ppr(efx, efy)
        pp = sim.mesh.array("patch_ptr")
        has = (pp[1:] - pp[:-1]) >= 6
        ex = -(0.2 + 0.02 * xs + 0.02 * ys)
        ey = -(-0.1 + 0.02 * xs - 0.01 * ys)
        assert np.abs(efx - ex)[has].max() < 1e-9
        assert np.abs(efy - ey)[has].max() < 1e-9
    finally:
        sim.close()


def test_sort_matches_oracle_order():
    sim = _sim()
    try:
        _random_fields(sim, scale=20.0)
        for s in range(2):
            sim.move_all(s)
        sim.get_par_chg()
        for s in range(2):
            before = sim.download(s)
            sim.sort(s)
            after = sim.download(s)
            perm = ob.sort_perm(before["loc"], before["id"])
            assert np.array_equal(after["id"], before["id"][perm])
            assert np.array_equal(after["loc"], before["loc"][perm])
            assert np.all(np.diff(after["loc"]) >= 0)
    finally:
        sim.close()


def test_mcc_parity():
    # high pressure so that a tiny deck sees every reaction type in one step
    sim = _sim("tiny", gas_p_Pa=2000.0, ppc=64, Te_eV=30.0)
    try:
        before = [sim.download(s) for s in range(2)]
        st = sim.mcc(7)
        after = [_by_id(sim.download(s)) for s in range(2)]
        vref = sim.scales["v_ref"]
        total_new = 0
        for s in range(2):
            o = {k: v.copy() for k, v in before[s].items()}
            ncoll, counts, par, ne, ni = ob.mcc(sim.mcc_tables[s], sim.gas, sim.species[s][1], vref,
                                               sim.cfg.seed, 7, s, o)
            assert st.n_selected[s] == ncoll
            assert list(st.n_by_reaction[s])[:sim.mcc_tables[s].n_reaction] == \
                list(counts[:sim.mcc_tables[s].n_reaction])
            n0 = before[s]["x"].size
            oo = _by_id(o)
            a = {k: v[:n0] if k != "id" else v[:n0] for k, v in after[s].items()}
            assert np.array_equal(a["id"], oo["id"])
            for k in ("vx", "vy", "vz"):
                sc = np.abs(oo[k]).max()
                assert np.abs(a[k] - oo[k]).max() <= 1e-12 * sc, k
            total_new += par.size
            if s == 0 and par.size:
                # created electrons follow the existing ones, ids in parent order
                ne_g = after[0]
                k0 = n0
                new_ids = ne_g["id"][k0:k0 + par.size]
                assert np.array_equal(new_ids, np.arange(n0, n0 + par.size, dtype=np.uint32))
                assert np.abs(ne_g["vx"][k0:k0 + par.size] - ne[:, 0]).max() <= 1e-12 * np.abs(ne).max()
                ion = after[1]
                n1 = before[1]["x"].size
                assert np.abs(ion["vx"][n1:n1 + par.size] - ni[:, 0] / vref).max() <= \
                    1e-12 * np.abs(ni[:, 0] / vref).max()
        assert sum(st.n_created) == 2 * total_new
        assert sum(st.n_by_reaction[0]) > 0 and sum(st.n_by_reaction[1]) > 0
    finally:
        sim.close()


def _oracle_step(sim, parts, phi, step):
    """One step of the oracle in the order of pic_step (push, deposit, RHS,
    PCG, PPR, MCC, sort)."""
    m = sim.mesh
    nn = m.nn
    efx, efy, coef = parts["_efx"], parts["_efy"], parts["_coef"]
    qs, es, wq = [], [], []
    for s in range(2):
        p = parts[s]
        qm = sim.species[s][0] / (sim.species[s][1] / deck.ME)
        mover = ob.move_all_axi if sim.cfg.delta == 1 else ob.move_all
        mover(m.ptr, p, efx, efy, coef, qm, sim.cfg.dt)
        q, e, bad = ob.deposit(m.ptr, p, sim.species[s][1], sim.scales["v_ref"], nn)
        qs.append(q)
        es.append(e)
        wq.append(sim.species[s][2] * sim.species[s][0])
    rho, _, ek = ob.normalize(m.ptr, qs, es, wq, sim.scales["L_ref"], sim.cfg.n0, nn)
    parts["_ek"] = ek
    b = ob.rhs(m.ptr, rho, nn)
    phi, st = ob.pcg(m.ptr, b, phi, sim.cfg.pcg_tol, sim.cfg.pcg_maxit)
    c, efx, efy = ob.ppr(m.ptr, phi, nn)
    parts["_efx"], parts["_efy"], parts["_coef"] = efx, efy, np.ascontiguousarray(c.ravel())
    new = {0: [], 1: []}
    for s in range(2):
        p = parts[s]
        ncoll, counts, par, ne, ni = ob.mcc(sim.mcc_tables[s], sim.gas, sim.species[s][1],
                                           sim.scales["v_ref"], sim.cfg.seed, step, s, p)
        if par.size:
            new[0].append((p["x"][par], p["y"][par], ne, p["loc"][par]))
            new[1].append((p["x"][par], p["y"][par], ni / sim.scales["v_ref"], p["loc"][par]))
    for s in range(2):
        p = parts[s]
        for (x, y, v, loc) in new[s]:
            k = x.size
            nid = np.arange(p["_next"], p["_next"] + k, dtype=np.uint32)
            p["_next"] += k
            for key, val in (("x", x), ("y", y), ("vx", v[:, 0]), ("vy", v[:, 1]), ("vz", v[:, 2]),
                             ("loc", loc), ("id", nid)):
                p[key] = np.ascontiguousarray(np.concatenate([p[key], val]))
    for s in range(2):
        p = parts[s]
        if step % sim.cfg.sort_interval == 0:
            perm = ob.sort_perm(p["loc"], p["id"])
            for key in ("x", "y", "vx", "vy", "vz", "loc", "id"):
                p[key] = np.ascontiguousarray(p[key][perm])
    return phi, st, rho


@pytest.mark.parametrize("push64", ["direct", "tiled", "bulk"], indirect=True)
@pytest.mark.parametrize("name", ["tiny", "tiny_axi"])
def test_full_steps_match_oracle(name, push64):
    sim = _sim(name, gas_p_Pa=300.0, Te_eV=20.0, sort_interval=3, diag_interval=4)
    try:
        st0 = sim.initial_fields()
        parts = {}
        for s in range(2):
            parts[s] = _oracle_parts(sim, s)
            parts[s]["_next"] = parts[s]["x"].size
        nn = sim.mesh.nn
        qs, es, wq = [], [], []
        for s in range(2):
            q, e, _ = ob.deposit(sim.mesh.ptr, parts[s], sim.species[s][1], sim.scales["v_ref"], nn)
            qs.append(q)
            es.append(e)
            wq.append(sim.species[s][2] * sim.species[s][0])
        rho, _, _ = ob.normalize(sim.mesh.ptr, qs, es, wq, sim.scales["L_ref"], sim.cfg.n0, nn)
        phi, _ = ob.pcg(sim.mesh.ptr, ob.rhs(sim.mesh.ptr, rho, nn), sim.mesh.array("phi_dirichlet"),
                        sim.cfg.pcg_tol, sim.cfg.pcg_maxit)
        assert np.array_equal(phi, sim.field("phi"))
        c, efx, efy = ob.ppr(sim.mesh.ptr, phi, nn)
        parts["_efx"], parts["_efy"], parts["_coef"] = efx, efy, np.ascontiguousarray(c.ravel())
        created = 0
        for step in range(1, 13):
            gst = sim.step()
            phi, ost, rho = _oracle_step(sim, parts, phi, step)
            created += sum(gst.mcc.n_created)
            gphi = sim.field("phi")
            assert np.abs(gphi - phi).max() <= 1e-10 * max(1.0, np.abs(phi).max()), step
            if step % 4 == 0:  # diagnostic step: per-node mean energies deposited
                for s, nm in ((0, "ek_e"), (1, "ek_i")):
                    ref = parts["_ek"][s]
                    assert np.abs(sim.field(nm) - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())
            for s in range(2):
                g = _by_id(sim.download(s))
                o = parts[s]
                live = o["loc"] >= 0
                assert gst.n_particles[s] == int(live.sum()), (step, s)
                oo = _by_id({k: o[k][live] for k in ("x", "y", "vx", "vy", "vz", "loc", "id")})
                assert np.array_equal(g["id"], oo["id"])
                assert np.array_equal(g["loc"], oo["loc"])
                for k in ("x", "y", "vx", "vy", "vz"):
                    sc = max(1.0, np.abs(oo[k]).max())
                    assert np.abs(g[k] - oo[k]).max() <= 1e-10 * sc, (step, s, k)
        assert created > 0
    finally:
        sim.close()


def test_edge_cases():
    sim = _sim()
    lib = api.load()
    try:
        # empty species
        z = np.zeros(0)
        sim.upload(1, z, z, z, z, z)
        assert sim.count(1) == 0
        sim.get_par_chg()
        st = sim.ife_solve()
        assert st.ierr == 0
        sim.step()
        # particle outside the mesh is rejected at upload
        bad = np.array([-1.0])
        one = np.zeros(1)
        rc = lib.pic_upload_particles(1, 1, api.dptr(bad), api.dptr(one), api.dptr(one),
                                      api.dptr(one), api.dptr(one), None, None)
        assert rc == -5
        # particles on the upper walls are located in the last element
        xm = np.array([sim.mesh.desc.xmax - 1e-12, 0.5 * sim.mesh.hx])
        ym = np.array([0.5 * sim.mesh.hy, sim.mesh.desc.ymax])
        sim.upload(1, xm, ym, np.zeros(2), np.zeros(2), np.zeros(2))
        g = _by_id(sim.download(1))
        assert g["loc"][0] == ob.load().or_locate(sim.mesh.ptr, xm[0], ym[0])
        assert g["loc"][1] == ob.load().or_locate(sim.mesh.ptr, xm[1], ym[1])
        # capacity overflow is an error, not a crash
        cap = sim.params.species[1].capacity
        big = np.full(cap + 1, 0.5 * sim.mesh.hx)
        rc = lib.pic_upload_particles(1, cap + 1, api.dptr(big), api.dptr(big), api.dptr(big),
                                      api.dptr(big), api.dptr(big), None, None)
        assert rc == -7
        # every particle absorbed by the walls
        n = sim.count(0)
        sim.set_field("efx", np.full(sim.mesh.nn, -1e6))
        sim.set_field("efy", np.zeros(sim.mesh.nn))
        sim.move_all(0)
        assert sim.count(0) == 0 or sim.count(0) < n
    finally:
        sim.close()


@pytest.mark.parametrize("precision,mode", [(api.PIC_PREC_FP64, "bounded"), (api.PIC_PREC_MIXED, "bounded"),
                                            (api.PIC_PREC_MIXED, "fallback")])
def test_mcc_bounded_selection_matches_full(precision, mode, monkeypatch):
    """The selection under a key bound (histogram and compact list of the
    keys below it, built by the step's push from the particles it leaves
    live; threshold and ties found on the device) picks the same ncoll
    smallest (key, id) as the full key histogram (PIC_MCC_FULL=1):
    after 6 steps with MCC the particles, fields and reaction counts are
    bit-identical.  "fallback": the bound made too small (a test hook), so
    every bounded selection finds too few keys and redoes the selection with
    the full histogram."""
    out = []
    for full in ("1", "0"):
        monkeypatch.setenv("PIC_MCC_FULL", full)
        if mode == "fallback":
            monkeypatch.setenv("PIC_MCC_BOUND_SCALE", "0.01")
        sim = Simulation(deck.config("cfg1", precision=precision))
        try:
            sim.initial_fields()
            counts = []
            for _ in range(6):
                st = sim.step()
                counts.append([list(st.mcc.n_by_reaction[s]) for s in range(2)] +
                              [list(st.mcc.n_selected)[:2], list(st.mcc.n_created)[:2]])
            parts = [_by_id(sim.download(s)) for s in range(2)]
            out.append((counts, parts, sim.field("rho"), sim.field("phi")))
        finally:
            sim.close()
    (ca, pa, ra, fa), (cb, pb, rb, fb) = out
    assert ca == cb
    assert sum(ca[-1][2]) > 0  # collisions were selected
    for a, b in zip(pa, pb):
        for k in ("id", "loc", "x", "y", "vx", "vy", "vz"):
            assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(ra, rb) and np.array_equal(fa, fb)
