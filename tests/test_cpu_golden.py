"""CPU checks of the oracle and the mesh builder against the reference's own
known answers (no GPU needed).

Goldens used:
  - OUTPUT/physics_parameter.inp:42-47 (normalisation at n_ref=1e21 m^-3, 1 eV)
  - Philox4x32-10 known-answer vectors of the Random123 distribution
  - closed-form Q1 IFE basis of Retangular_reference_basis_IFE.f90 (oracle)
  - IFE convergence, Norm_Error_{0064,0128,0256}.txt (manufactured circle of
    code/IFE-error/Function_True.f90)
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

import oracle_bind as ob
from pic_b200 import api, deck

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_reference_scales_known_answer():
    g = json.load(open(os.path.join(GOLDEN, "physics_parameter.json")))
    out = ob.scales(g["n_ref"], g["T_ref_eV"])
    for k, v in zip(("L_ref", "time_ref", "v_ref", "Phi_ref"), out):
        assert abs(v - g[k]) <= 1e-14 * abs(g[k]), (k, v, g[k])
    # the package's host copy agrees with the oracle
    sc = deck.reference_scales(g["n_ref"], g["T_ref_eV"])
    for k in ("L_ref", "time_ref", "v_ref", "Phi_ref"):
        assert abs(sc[k] - g[k]) <= 1e-14 * abs(g[k])
    # dimensionless ion mass of the same file: m_ion / ElectronMass (Constants.f90)
    assert abs(g["ion_mass_kg"] / 9.1095e-31 - g["ion_mass_over_me"]) < 1e-9


def test_philox_known_answers():
    kat = json.load(open(os.path.join(GOLDEN, "philox4x32_10_kat.json")))
    for case in kat:
        assert ob.philox(case["ctr"], case["key"]) == case["out"]


def _corner_xy(mesh, e):
    i, j = divmod(e, mesh.nny - 1)
    xs = mesh.desc.xmin + mesh.hx * np.arange(mesh.nnx)
    ys = mesh.desc.ymin + mesh.hy * np.arange(mesh.nny)
    return np.array([[xs[i], ys[j]], [xs[i + 1], ys[j]], [xs[i + 1], ys[j + 1]], [xs[i], ys[j + 1]]])


def test_ife_basis_matches_reference_closed_form():
    """The mesh builder derives the Q1 IFE basis from its defining conditions;
    the oracle restates the reference's closed form.  Both must agree."""
    lib = api.load()
    cfg = deck.config("cfg1")
    mesh = deck.Mesh(cfg)
    checked = {1: 0, 2: 0}
    for k in range(1, mesh.desc.n_interface + 1):
        el = C.c_int32()
        typ = C.c_int32()
        r2l = (C.c_int32 * 4)()
        beta = (C.c_double * 2)()
        D = (C.c_double * 2)()
        E = (C.c_double * 2)()
        api.check(lib.pic_mesh_interface_info(mesh.ptr, k, C.byref(el), C.byref(typ), r2l, beta, D, E),
                  "info")
        V = _corner_xy(mesh, el.value - 1)
        X = np.array([V[r2l[r] - 1] for r in range(4)])
        x1, y1 = X[0]
        x2, y2 = X[1]
        x4, y4 = X[3]
        bottom = (x2 - x1) * (y4 - y1) - (x4 - x1) * (y2 - y1)
        xi = lambda x, y: ((y4 - y1) * (x - x1) - (x4 - x1) * (y - y1)) / bottom
        et = lambda x, y: ((x2 - x1) * (y - y1) - (y2 - y1) * (x - x1)) / bottom
        a = xi(E[0], E[1])
        b = et(D[0], D[1]) if typ.value == 1 else xi(D[0], D[1])
        R = beta[0] / beta[1]
        Dp, Ep = np.array(D[:]), np.array(E[:])
        if typ.value == 1:
            pieces = {1: [X[0], Dp, Ep], 2: [X[2], Dp, Ep]}
            cases = [(1, 1), (1, 2), (3, 2)]
        else:
            pieces = {2: [X[1], X[2], Dp, Ep]}
            cases = [(2, 2)]
        for bi, pf in cases:
            Cc = ob.closed_form(typ.value, bi, pf, a, b, R)
            assert Cc is not None
            poly = np.array(pieces[pf])
            for w in ([1, 1, 1, 1], [2, 1, 1, 1], [1, 2, 1, 1], [1, 1, 2, 1]):
                w = np.array(w[:len(poly)], float)
                px, py = (poly * w[:, None]).sum(0) / w.sum()
                val, gx, gy = C.c_double(), C.c_double(), C.c_double()
                api.check(lib.pic_mesh_ife_basis(mesh.ptr, k, r2l[bi - 1] - 1, px, py, C.byref(val),
                                                 C.byref(gx), C.byref(gy)), "basis")
                s, t = xi(px, py), et(px, py)
                ref = Cc[0] + Cc[1] * s + Cc[2] * t + Cc[3] * s * t
                assert abs(val.value - ref) < 1e-11, (k, typ.value, bi, pf, val.value, ref)
        checked[typ.value] += 1
    assert checked[1] > 0 and checked[2] > 0
    mesh.close()


def _manufactured(N):
    """u = r^4/10 outside, r^4 - 0.9 r0^4 inside the circle r0 on [-1,1]^2,
    beta_out/beta_in = 10 (Function_True.f90, delta = 0)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    r0 = 0.500253607
    dk = api.Deck()
    dk.nnx = dk.nny = N + 1
    dk.xmin, dk.xmax, dk.ymin, dk.ymax = -1.0, 1.0, -1.0, 1.0
    dk.delta = 0
    for w in range(4):
        dk.wall_dirichlet[w] = 1
    dk.n_objects = 1
    o = dk.objects[0]
    o.shape, o.conductor, o.cx, o.cy, o.a, o.b, o.eps = api.PIC_SHAPE_CIRCLE, 0, 0.0, 0.0, r0, r0, 0.1
    lib = api.load()
    ptr = C.POINTER(api.MeshDesc)()
    api.check(lib.pic_mesh_build(C.byref(dk), C.byref(ptr)), "mesh")
    m = ptr.contents
    nn = (N + 1) ** 2
    xs = np.linspace(-1, 1, N + 1)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    r2 = (X * X + Y * Y).ravel()
    exact = np.where(r2 - r0 * r0 > 0, r2 * r2 / 10.0, r2 * r2 - 0.9 * r0 ** 4)
    phid = np.ctypeslib.as_array(m.phi_dirichlet, shape=(nn,))
    nt = np.ctypeslib.as_array(m.node_type, shape=(nn,))
    phid[nt < 0] = exact[nt < 0]
    rho = -1.6 * r2
    b = ob.rhs(ptr, rho, nn)
    nu = m.n_unknowns
    srow = np.ctypeslib.as_array(m.a_srow, shape=(nu + 1,)) - 1
    jcol = np.ctypeslib.as_array(m.a_jcol, shape=(m.nnz,)) - 1
    kk = np.ctypeslib.as_array(m.a_k, shape=(m.nnz,))
    A = sp.csr_matrix((kk, jcol, srow), shape=(nu, nu))
    u = spl.spsolve(A.tocsc(), b[nt > 0])
    err = u - exact[nt > 0]
    vol = np.ctypeslib.as_array(m.cell_volume, shape=(nn,))[nt > 0]
    l2 = math.sqrt(float((err * err * vol).sum()))
    # oracle PCG reproduces the direct solution
    phi0 = np.where(nt > 0, 0.0, phid)
    phi, st = ob.pcg(ptr, b, phi0, 1e-12, 20000)
    pcg_err = np.abs(phi[nt > 0] - u).max()
    lib.pic_mesh_free(ptr)
    return l2, pcg_err, st


def test_ife_convergence_matches_norm_error_files():
    ref = json.load(open(os.path.join(GOLDEN, "norm_error.json")))
    l2 = {}
    for N in (64, 128, 256):
        e, pcg_err, st = _manufactured(N)
        l2[N] = e
        assert st["ierr"] == 0 and pcg_err < 1e-9
        # same order of magnitude as the reference's IFE L2 error
        assert 0.2 * ref[str(N)]["L2"] < e < 5.0 * ref[str(N)]["L2"], (N, e, ref[str(N)]["L2"])
    rate1 = math.log2(l2[64] / l2[128])
    rate2 = math.log2(l2[128] / l2[256])
    assert rate1 > 1.6 and rate2 > 1.6, (rate1, rate2)


def test_canonical_dot_is_a_sum():
    rng = np.random.default_rng(0)
    for n in (1, 255, 1024, 5000, 100003):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        s = ob.canon_dot(a, b)
        assert abs(s - float(np.dot(a, b))) < 1e-12 * (1 + np.abs(a * b).sum())
