"""Analytic known answers for the parts of the oracle that the reference
holds no outputs for (push, stiffness, Jacobi-PCG, MCC): free streaming, a
uniform field through both gathers (bilinear nodal E and the interface
elements' PPR gradients), the Q1 stiffness stencil, the PCG solution
against a direct sparse solve, and the energy bookkeeping of elastic,
excitation and ionisation collisions.  CPU only."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import oracle_bind as ob
from pic_b200 import deck


def _parts(cfg, mesh, s=0):
    x, y, vx, vy, vz = [a.copy() for a in deck.load_particles(cfg, mesh, s)]
    loc = np.array([ob.load().or_locate(mesh.ptr, a, b) for a, b in zip(x, y)], np.int32)
    return {"x": x, "y": y, "vx": vx, "vy": vy, "vz": vz, "loc": loc}


def _fields(mesh, e0, e1):
    nn = mesh.nn
    efx, efy = np.full(nn, e0), np.full(nn, e1)
    coef = np.zeros((5, nn))  # c2..c6: the PPR gradient is (-c2, -c3) plus the linear terms
    coef[0], coef[1] = -e0, -e1
    return efx, efy, np.ascontiguousarray(coef.ravel())


def test_free_streaming_push():
    cfg = deck.config("tiny")
    mesh = deck.Mesh(cfg)
    try:
        p = _parts(cfg, mesh)
        before = {k: v.copy() for k, v in p.items()}
        efx, efy, coef = _fields(mesh, 0.0, 0.0)
        ob.move_all(mesh.ptr, p, efx, efy, coef, -1.0, cfg.dt)
        live = p["loc"] >= 0
        assert live.sum() > 0.9 * live.size
        assert np.array_equal(p["vx"], before["vx"]) and np.array_equal(p["vy"], before["vy"])
        assert np.array_equal(p["x"][live], before["x"][live] + cfg.dt * before["vx"][live])
        assert np.array_equal(p["y"][live], before["y"][live] + cfg.dt * before["vy"][live])
    finally:
        mesh.close()


def test_uniform_field_push():
    cfg = deck.config("tiny")
    mesh = deck.Mesh(cfg)
    try:
        p = _parts(cfg, mesh)
        before = {k: v.copy() for k, v in p.items()}
        e0, e1, qm = 0.37, -0.21, -1.0
        efx, efy, coef = _fields(mesh, e0, e1)
        interface = np.array([mesh.array("element_index")[e] > 0 if e >= 0 else False for e in before["loc"]])
        assert interface.any() and (~interface).any()  # both gathers are exercised
        ob.move_all(mesh.ptr, p, efx, efy, coef, qm, cfg.dt)
        live = p["loc"] >= 0
        for v, e in (("vx", e0), ("vy", e1)):
            want = before[v] + qm * e * cfg.dt
            assert np.allclose(p[v][live], want[live], rtol=0, atol=1e-14 * np.abs(want).max())
        assert np.allclose(p["x"][live], before["x"][live] + cfg.dt * p["vx"][live], rtol=0, atol=1e-14)
    finally:
        mesh.close()


def test_q1_stiffness_stencil_is_the_analytic_element_matrix():
    """Square cells, vacuum, away from objects and walls: the assembled row is
    the Q1 Laplacian stencil 8/3 at the centre and -1/3 at the 8 neighbours."""
    cfg = deck.config("cfg1")
    mesh = deck.Mesh(cfg)
    try:
        nt = mesh.array("node_type")
        srow, jcol, ak = mesh.array("a_srow"), mesh.array("a_jcol"), mesh.array("a_k")
        node_of = np.zeros(mesh.desc.n_unknowns, np.int64)
        node_of[nt[nt > 0] - 1] = np.nonzero(nt > 0)[0]
        for i, j in ((5, 5), (5, 40), (58, 12)):
            n = i * mesh.nny + j
            u = nt[n] - 1
            cols = node_of[jcol[srow[u] - 1:srow[u + 1] - 1] - 1]
            vals = ak[srow[u] - 1:srow[u + 1] - 1]
            row = dict(zip(cols.tolist(), vals.tolist()))
            assert len(row) == 9
            assert abs(row[n] - 8.0 / 3.0) <= 1e-12
            for di in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    if di or dj:
                        assert abs(row[n + di * mesh.nny + dj] + 1.0 / 3.0) <= 1e-12
    finally:
        mesh.close()


def test_pcg_matches_direct_solve():
    cfg = deck.config("tiny")
    mesh = deck.Mesh(cfg)
    try:
        nn = mesh.nn
        rho = np.random.default_rng(11).standard_normal(nn) * 0.05
        b = ob.rhs(mesh.ptr, rho, nn)
        phi0 = mesh.array("phi_dirichlet").copy()
        phi, st = ob.pcg(mesh.ptr, b, phi0, 1e-13, 20000)
        assert st["ierr"] == 0
        nt = mesh.array("node_type")
        nu = mesh.desc.n_unknowns
        node_of = np.zeros(nu, np.int64)
        node_of[nt[nt > 0] - 1] = np.nonzero(nt > 0)[0]
        A = sp.csr_matrix((mesh.array("a_k"), mesh.array("a_jcol") - 1, mesh.array("a_srow") - 1), shape=(nu, nu))
        x = spl.spsolve(A.tocsc(), b[node_of])
        assert np.abs(phi[node_of] - x).max() <= 1e-9 * np.abs(x).max()
        # Dirichlet nodes keep their values
        assert np.array_equal(phi[nt <= 0], phi0[nt <= 0])
    finally:
        mesh.close()


# ---- MCC collision laws in the limit of an infinitely heavy, cold gas: the
# target is at rest and the mass ratio M/(m+M) rounds to 1, so an elastic
# scattering keeps the speed, an excitation leaves E - E_thr, and an
# ionisation splits E - E_thr between the scattered and the created electron
# (the ion is created at rest).

import ctypes as C  # noqa: E402

from pic_b200 import api  # noqa: E402

_JTOEV = 1.6022e-19


def _table(rtype, thr):
    """Every particle collides (ratio 1) and takes reaction `rtype`
    (cumulative probability 1 from its column on, at every energy)."""
    t = api.MccTable()
    t.species, t.n_reaction, t.n_sigma = 0, 3, 12
    t.energy_min, t.energy_interval, t.energy_max = -3.0, 0.5, 1e6
    t.collision_ratio = 1.0
    types = (11, 12, 13)
    col = types.index(rtype)
    for j in range(3):
        t.reaction_type[j] = types[j]
        t.threshold[j] = 0.0 if types[j] == 11 else thr
        t.resultant[j] = 1 if types[j] == 13 else -1
    prob = np.zeros((12, 3))
    prob[:, col:] = 1.0
    keep = np.ascontiguousarray(prob.ravel())
    t.probability = keep.ctypes.data_as(C.POINTER(C.c_double))
    return t, keep


def _electrons(n, vref, seed=3):
    rng = np.random.default_rng(seed)
    # speeds for 5..60 eV electrons, random directions (normalised by vref)
    e = rng.uniform(5.0, 60.0, n)
    v = np.sqrt(2.0 * e * _JTOEV / deck.ME) / vref
    d = rng.standard_normal((3, n))
    d /= np.linalg.norm(d, axis=0)
    return {"x": np.zeros(n), "loc": np.zeros(n, np.int32), "id": np.arange(n, dtype=np.uint32),
            "vx": v * d[0], "vy": v * d[1], "vz": v * d[2]}


def _energy(p, vref):
    v2 = p["vx"] ** 2 + p["vy"] ** 2 + p["vz"] ** 2
    return 0.5 * deck.ME * v2 * vref * vref / _JTOEV


def _run(rtype, thr=11.5):
    vref = 5.93e5
    gas = api.Gas()
    gas.mass, gas.temperature, gas.density = 1e30, 0.0, 1e21
    t, keep = _table(rtype, thr)
    p = _electrons(3000, vref)
    e0 = _energy(p, vref)
    ncoll, counts, par, ne, ni = ob.mcc(t, gas, deck.ME, vref, 17, 5, 0, p)
    return p, e0, ncoll, counts, par, ne, ni, vref, keep


def test_mcc_elastic_keeps_the_speed():
    p, e0, ncoll, counts, _, _, _, vref, _ = _run(11)
    assert ncoll == p["vx"].size and counts[0] == ncoll
    assert np.allclose(_energy(p, vref), e0, rtol=1e-12, atol=0)


def test_mcc_excitation_loses_the_threshold():
    thr = 11.5
    p, e0, ncoll, counts, _, _, _, vref, _ = _run(12, thr)
    hit = e0 > thr
    assert counts[1] == hit.sum() and counts[0] == 0
    e1 = _energy(p, vref)
    assert np.allclose(e1[hit], e0[hit] - thr, rtol=1e-12, atol=1e-12 * e0.max())
    # below threshold no reaction: the speed only passes through SI units and back
    assert np.allclose(e1[~hit], e0[~hit], rtol=1e-14, atol=0)


def test_mcc_ionisation_balances_energy():
    thr = 11.5
    p, e0, ncoll, counts, par, ne, ni, vref, _ = _run(13, thr)
    hit = e0 > thr
    assert counts[2] == hit.sum() == par.size
    assert np.all(np.diff(p["id"][par].astype(np.int64)) > 0)  # created in parent-id order
    e1 = _energy(p, vref)
    e_new = 0.5 * deck.ME * (ne ** 2).sum(axis=1) * vref * vref / _JTOEV
    assert np.allclose(e1[par] + e_new, e0[par] - thr, rtol=1e-12, atol=1e-12 * e0.max())
    assert np.all(ni == 0.0)  # the ion takes the (resting) target's velocity


def test_mcc_selection_keys_pick_uniform_subsets():
    """The null-collision selection (the ncoll smallest keys of the live
    ids) behaves as the reference's uniform random N-subset
    (MCCPublic.F90:148-171): every id is picked at the rate ncoll/n, ids next
    to each other and the same id on consecutive steps are picked together
    at the product rate, keys of one step are distinct, and species and
    seeds draw different keys.  Bounds are 5 standard deviations."""
    n, ncoll, steps, seed = 4096, 64, 2000, 12345
    ids = np.arange(n, dtype=np.uint32) * np.uint32(7) + np.uint32(1000)  # ids need not be contiguous
    picked = np.zeros((steps, n), bool)
    for t in range(steps):
        k = ob.mcc_select_keys(seed, t, 0, ids)
        if t == 0:
            assert np.unique(k).size == n
        picked[t, np.argpartition(k, ncoll)[:ncoll]] = True
    p = ncoll / n
    counts = picked.sum(0)
    chi2 = ((counts - steps * p) ** 2 / (steps * p * (1 - p))).sum()
    assert abs(chi2 - n) < 5 * np.sqrt(2 * n)
    for a, b in ((picked[:, :-1], picked[:, 1:]), (picked[:-1], picked[1:])):
        both = int((a & b).sum())
        q = p * (ncoll - 1) / (n - 1) if a.shape[1] == n - 1 else p * p
        mean = a.size * q
        assert abs(both - mean) < 5 * np.sqrt(mean), (both, mean)
    k0 = ob.mcc_select_keys(seed, 5, 0, ids)
    assert (k0 != ob.mcc_select_keys(seed, 5, 1, ids)).mean() > 0.99
    assert (k0 != ob.mcc_select_keys(seed + 1, 5, 0, ids)).mean() > 0.99
