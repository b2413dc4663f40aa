"""Analytic known answers for the parts of the oracle that the reference
holds no outputs for (push, stiffness, Jacobi-PCG): free streaming, a
uniform field through both gathers (bilinear nodal E and the interface
elements' PPR gradients), the Q1 stiffness stencil, and the PCG solution
against a direct sparse solve.  CPU only."""
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
