"""The product's mesh builder (pic_mesh_build) against the oracle's own
restatement of the reference's setup phase (oracle/oracle_mesh.c), entry by
entry, on the benchmark decks' geometries.  The two share no code: the
oracle derives node labels, unknown numbering, interface geometry (the
reference's case table and line-object intersections), the closed-form IFE
basis, stiffness by the reference's Gauss rules, load matrices, dual volumes
and PPR patches itself.

Bars:
* integer arrays (node_type, node_index, element_index, patch structure)
  and the interface elements' type and vertex order: identical;
* dual volumes and Dirichlet values: identical bits;
* with FP64 quadrature constants (OR_QUAD_EXACT): stiffness, Dirichlet
  block and Jacobi diagonal within 1e-12 of the largest entry; regular load
  matrices within 1e-13 (r-weighted rows 1e-12: the reference forms them
  from bilinear coefficients in absolute coordinates); interface load
  matrices within 1e-8 (the reference
  solves their 8x8 basis systems in absolute coordinates, up to ~900 Debye
  lengths here, which costs digits the product's vertex-relative systems
  keep: 4.3e-9 measured on the 8-ellipse deck);
* with the constants as the reference compiles them (default-kind REAL(4)
  literals, OR_QUAD_AS_COMPILED): within 6e-8, the size of that rounding.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import oracle_bind as ob
from pic_b200 import api, deck

DECKS = [("tiny", {}), ("tiny_axi", {}), ("cfg1", {}), ("cfg2", dict(ncx=128, ncy=128)),
         ("cfg4", dict(ncx=128, ncy=128)), ("cfg5", dict(ncx=256, ncy=128))]


def _csr(m, pre):
    srow = m.array(pre + "_srow").astype(np.int64) - 1
    jcol = m.array(pre + "_jcol").astype(np.int64) - 1
    n = len(srow) - 1
    return sp.csr_matrix((m.array(pre + "_k"), jcol, srow), shape=(n, m.nn if pre == "xt" else n))


def _rel_sparse(a, b):
    return abs(a - b).max() / abs(a).max()


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(a).max()


@pytest.fixture(scope="module", params=DECKS, ids=[d[0] for d in DECKS])
def meshes(request):
    name, over = request.param
    pm = deck.Mesh(deck.config(name, **over))
    om = {q: ob.OracleMesh(pm.deck, q) for q in (ob.OR_QUAD_EXACT, ob.OR_QUAD_AS_COMPILED)}
    yield pm, om
    for m in om.values():
        m.close()
    pm.close()


def test_integer_arrays_identical(meshes):
    pm, om = meshes
    o = om[ob.OR_QUAD_AS_COMPILED]
    for a in ("node_type", "node_index", "element_index", "patch_ptr", "patch_nodes"):
        assert np.array_equal(pm.array(a), o.array(a)), a
    assert pm.desc.n_unknowns == o.desc.n_unknowns and pm.desc.n_interface == o.desc.n_interface
    for a in ("cell_volume", "phi_dirichlet"):
        assert np.array_equal(pm.array(a), o.array(a)), a


def test_interface_elements_identical(meshes):
    pm, om = meshes
    o = om[ob.OR_QUAD_EXACT]
    lib = api.load()
    for k in range(1, pm.desc.n_interface + 1):
        el, ty = C.c_int32(), C.c_int32()
        r2l, beta, D, E = np.zeros(4, np.int32), np.zeros(2), np.zeros(2), np.zeros(2)
        api.check(lib.pic_mesh_interface_info(pm.ptr, k, C.byref(el), C.byref(ty), ob.i32(r2l), ob.d(beta),
                                              ob.d(D), ob.d(E)), "interface info")
        f = o.interface(k)
        assert (el.value, ty.value) == (f["element"], f["type"]), k
        assert np.array_equal(r2l, f["r2l"]) and np.array_equal(beta, f["beta"]), k
        scale = max(abs(pm.desc.xmax), abs(pm.desc.ymax))
        assert np.abs(D - f["D"]).max() <= 1e-13 * scale and np.abs(E - f["E"]).max() <= 1e-13 * scale, k


def test_operator_with_fp64_constants(meshes):
    pm, om = meshes
    o = om[ob.OR_QUAD_EXACT]
    assert _rel_sparse(_csr(pm, "a"), _csr(o, "a")) <= 1e-12
    assert _rel_sparse(_csr(pm, "xt"), _csr(o, "xt")) <= 1e-12
    assert _rel(pm.array("a_diag"), o.array("a_diag")) <= 1e-12
    assert _rel(pm.array("mass_q1"), o.array("mass_q1")) <= 1e-13
    if pm.desc.delta == 1:
        assert _rel(pm.array("mass_rows"), o.array("mass_rows")) <= 1e-12
    if pm.desc.n_interface:
        assert _rel(pm.array("ife_mass"), o.array("ife_mass")) <= 1e-8


def test_operator_with_the_references_constants(meshes):
    pm, om = meshes
    o, x = om[ob.OR_QUAD_AS_COMPILED], om[ob.OR_QUAD_EXACT]
    for pre in ("a", "xt"):
        r = _rel_sparse(_csr(pm, pre), _csr(o, pre))
        # the single-precision constants are what separates the two
        assert 1e-10 < r <= 6e-8, (pre, r)
        assert _rel_sparse(_csr(x, pre), _csr(o, pre)) > 1e-10
    for a in ("mass_q1", "ife_mass") + (("mass_rows",) if pm.desc.delta == 1 else ()):
        if a == "ife_mass" and not pm.desc.n_interface:
            continue
        assert _rel(pm.array(a), o.array(a)) <= 6e-8, a


def test_quadrature_constants_are_the_compiled_literals():
    """Generate_Gauss_reference(_triangle).f90 write their weights and points
    as default-kind literals: each value is the single-precision evaluation
    of its expression, widened to FP64."""
    f = np.float32
    c = ob.quad_constants(ob.OR_QUAD_AS_COMPILED)
    x = ob.quad_constants(ob.OR_QUAD_EXACT)
    s6 = np.sqrt(f(0.6))
    assert c[0] == float(f(64.0) / f(81.0)) and x[0] == 64.0 / 81.0
    assert c[9 + 2] == float(s6) and x[9 + 2] == np.sqrt(0.6)          # p9[1] = (s6, s6)
    assert c[27 + 1] == float(f(100.0) / f(324.0) * (f(1) - s6) / f(8.0))  # wt9[1]
    assert c[-1] == float(f(1.0) / f(3.0)) and x[-1] == 1.0 / 3.0        # IFE_RHS_2D gwght
    assert np.abs(c - x).max() > 1e-9 and np.abs(c - x).max() < 1e-7


def test_potential_from_either_operator():
    """The oracle's Jacobi-PCG on the oracle's operator and on the product's
    reach the same potential: 1e-10 with FP64 constants; the reference's
    REAL(4) constants move it by less than 1e-6."""
    cfg = deck.config("cfg1")
    pm = deck.Mesh(cfg)
    try:
        rho = np.random.default_rng(5).standard_normal(pm.nn) * 0.05
        phis = []
        for m in (pm, ob.OracleMesh(pm.deck, ob.OR_QUAD_EXACT), ob.OracleMesh(pm.deck, ob.OR_QUAD_AS_COMPILED)):
            b = ob.rhs(m.ptr, rho, m.nn)
            phi, st = ob.pcg(m.ptr, b, m.array("phi_dirichlet"), 1e-12, 20000)
            assert st["ierr"] == 0
            phis.append(phi)
        scale = np.abs(phis[0]).max()
        assert np.abs(phis[1] - phis[0]).max() <= 1e-10 * scale
        d = np.abs(phis[2] - phis[0]).max()
        assert 1e-12 * scale < d <= 1e-6 * scale
    finally:
        pm.close()


def test_reference_case_table_orientation():
    """Opposite-edge interface elements cut on edges 2-3 and 4-1 take local
    corner 4 as reference vertex 1 (El_Object_Intersection_info_2D_BL.f90);
    on an r-z mesh the load matrix depends on that choice (its sub-triangle
    rule is not exact for r-weighted integrands), and both builders agree."""
    pm = deck.Mesh(deck.config("tiny_axi"))
    o = ob.OracleMesh(pm.deck, ob.OR_QUAD_EXACT)
    try:
        seen = 0
        for k in range(1, pm.desc.n_interface + 1):
            f = o.interface(k)
            if f["type"] == 2 and f["r2l"][0] == 4:
                seen += 1
                a = pm.array("ife_mass")[16 * (k - 1):16 * k]
                b = o.array("ife_mass")[16 * (k - 1):16 * k]
                assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
        assert seen > 0
    finally:
        o.close()
        pm.close()
