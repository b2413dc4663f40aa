"""The multigrid V-cycle of the flexible-CG preconditioner
(pic_multigrid_setup): one application against an independent scipy
V-cycle built from the mesh's CSR matrix, the iteration counts it buys, the
persistent solver against the one-launch-per-operation path, and the grids
it refuses.

Bars: the V-cycle within 1e-5 of max|z| (the device holds the coarse
stencils and 1/diag in FP32; the scipy reference is FP64 except for the
coarsest inverse, which both round to the same scaled FP16); solves to the
requested tolerance on the FP64 true residual; persistent and launch-per-operation iterations within 2 of each
other and their potentials within 1e-7 relative.
"""
import ctypes as C
import os

import numpy as np
import pytest
import scipy.sparse as sp

from pic_b200 import api, deck

pytestmark = pytest.mark.gpu


def _interp1(nf):
    nc = (nf - 1) // 2 + 1
    rows, cols, vals = [], [], []
    for i in range(nf):
        if i % 2 == 0:
            rows.append(i)
            cols.append(i // 2)
            vals.append(1.0)
        else:
            rows += [i, i]
            cols += [i // 2, i // 2 + 1]
            vals += [0.5, 0.5]
    return sp.csr_matrix((vals, (rows, cols)), shape=(nf, nc))


def _scipy_vcycle(mesh, r_full, omega, max_coarse=4500):
    """The V-cycle of stage 1 + 2 (pre-smoothing, multigrid correction) in
    scipy, FP64, on the unknowns; returns z on the full grid."""
    d = mesh.desc
    nu, nnx, nny = d.n_unknowns, mesh.nnx, mesh.nny
    A = sp.csr_matrix((mesh.array("a_k"), mesh.array("a_jcol") - 1, mesh.array("a_srow") - 1), shape=(nu, nu))
    nt = mesh.array("node_type")
    node_of = np.zeros(nu, np.int64)
    node_of[nt[nt > 0] - 1] = np.nonzero(nt > 0)[0]
    sel = sp.csr_matrix((np.ones(nu), (np.arange(nu), node_of)), shape=(nu, nnx * nny))
    Ps = [(sel @ sp.kron(_interp1(nnx), _interp1(nny))).tocsr()]
    As = [A]
    nx, ny = nnx, nny
    while True:
        Ac = (Ps[-1].T @ As[-1] @ Ps[-1]).tocsr()
        As.append(Ac)
        nx, ny = (nx - 1) // 2 + 1, (ny - 1) // 2 + 1
        if nx * ny <= max_coarse:
            break
        Ps.append(sp.kron(_interp1(nx), _interp1(ny)).tocsr())
    act = [a.diagonal() != 0 for a in As]
    dinv = [np.where(a, 1.0 / np.where(a, A_.diagonal(), 1.0), 0.0) for a, A_ in zip(act, As)]
    dense = As[-1].toarray() + np.diag((~act[-1]).astype(float))
    inv = np.linalg.inv(dense)
    # the device applies a scaled FP16 copy of the inverse (scale: the
    # largest diagonal entry / 16384) with FP64 accumulation
    scale = np.abs(np.diag(inv)).max() / 16384.0
    inv = (inv * (1.0 / scale)).astype(np.float32).astype(np.float16).astype(np.float64) * scale
    r0 = r_full[node_of]

    def cycle(l, r):
        if l == len(As) - 1:
            return inv @ r
        z = omega * dinv[l] * r
        t = r - As[l] @ z
        e = cycle(l + 1, Ps[l].T @ t)
        y = z + Ps[l] @ e
        if l == 0:
            return y
        out = y + omega * dinv[l] * (r - As[l] @ y)
        return np.where(act[l], out, 0.0)

    z = np.zeros(nnx * nny)
    z[node_of] = cycle(0, r0)
    return z, len(As)


def _sim(cells, **over):
    from pic_b200.simulation import Simulation
    return Simulation(deck.config("cfg4", ncx=cells, ncy=cells, ppc=1, **over), load=False)


def test_vcycle_matches_scipy():
    import torch
    sim = _sim(128)
    try:
        omega = 2.0 / 3.0
        api.check(sim.lib.pic_set_precond_stages(1, omega, 0), "stages")
        api.check(sim.lib.pic_multigrid_setup(sim.mesh.ptr, 300), "mg")
        nt = sim.mesh.array("node_type")
        r = np.random.default_rng(7).standard_normal(sim.mesh.nn) * (nt > 0)
        rd = torch.tensor(r, device="cuda")
        zd = torch.zeros_like(rd)
        torch.cuda.synchronize()
        api.check(sim.lib.pic_precond_apply(0, C.c_void_p(rd.data_ptr()), C.c_void_p(zd.data_ptr())), "apply")
        torch.cuda.synchronize()
        z = zd.cpu().numpy()
        want, levels = _scipy_vcycle(sim.mesh, r, omega, 300)
        assert levels == 4  # 129^2 -> 65^2 -> 33^2 -> 17^2
        err = np.abs(z - want).max() / np.abs(want).max()
        print(f"\nV-cycle device vs scipy: max rel {err:.2e}")
        assert err <= 1e-5
        assert np.all(z[nt <= 0] == 0.0)
    finally:
        sim.close()


def _solve(sim, multigrid, omega=2.0 / 3.0, keep_phi=False):
    if not keep_phi:
        sim.set_field("phi", np.zeros(sim.mesh.nn))
        sim.set_solver("fcg", multigrid=multigrid, omega=omega)
    st = api.SolveStats()
    api.check(sim.lib.pic_ife_solve(None, 0.0, C.byref(st)), "pic_ife_solve")
    return st, sim.field("phi")


def test_multigrid_fcg_iterations():
    """cfg4 geometry (8 dielectric ellipses) at 256^2 cells, tolerance 1e-8:
    the V-cycle (256 -> 128 -> 64 -> 32 cells) needs well under the two-level
    method's iterations (scipy: 11 against 18) and reaches the same
    potential."""
    sim = _sim(256)
    try:
        sim.set_field("rho", np.random.default_rng(0).standard_normal(sim.mesh.nn))
        s2, p2 = _solve(sim, False)
        sm, pm = _solve(sim, True)
        print(f"\n256^2 FCG iterations: two-level {s2.iterations}, multigrid {sm.iterations}")
        assert s2.fallback == 0 and sm.fallback == 0
        assert sm.rel_residual <= 1e-8
        assert sm.iterations <= 14 and sm.iterations < s2.iterations
        assert np.abs(pm - p2).max() <= 1e-6 * np.abs(p2).max()
    finally:
        sim.close()


def test_multigrid_persistent_matches_launch_path():
    out = []
    for flag in ("0", "1"):
        os.environ["PIC_FCG_PERSISTENT"] = flag
        try:
            sim = _sim(256, pcg_tol=1e-10)
        finally:
            del os.environ["PIC_FCG_PERSISTENT"]
        try:
            sim.set_field("rho", np.random.default_rng(1).standard_normal(sim.mesh.nn))
            st, phi = _solve(sim, True)
            assert st.fallback == 0 and st.rel_residual <= 1e-10
            out.append((st.iterations, phi))
        finally:
            sim.close()
    print(f"\nmultigrid FCG iterations: launch path {out[0][0]}, persistent {out[1][0]}")
    assert abs(out[0][0] - out[1][0]) <= 2
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-7 * np.abs(out[0][1]).max()


@pytest.mark.parametrize("warm", [False, True])
def test_fused_setup_and_judge_match_separate_kernels(warm):
    """The persistent FCG's set-up and judge as one launch each (residual
    and norms in k_dot's order) give the same iterations and the same bits
    as the separate x0 / SpMV / residual / dot kernels (PIC_FCG_FUSED=0),
    from phi = 0 and from a warm start."""
    out = []
    for flag in ("0", "1"):
        os.environ["PIC_FCG_FUSED"] = flag
        try:
            sim = _sim(256)
        finally:
            del os.environ["PIC_FCG_FUSED"]
        try:
            sim.set_field("rho", np.random.default_rng(2).standard_normal(sim.mesh.nn))
            st, phi = _solve(sim, True)
            if warm:  # a second solve from the first one's potential, a slightly changed charge
                sim.set_field("rho", np.random.default_rng(3).standard_normal(sim.mesh.nn) * 1e-3
                              + np.random.default_rng(2).standard_normal(sim.mesh.nn))
                st, phi = _solve(sim, True, keep_phi=True)
            assert st.fallback == 0 and st.rel_residual <= 1e-8
            out.append((st.iterations, st.rel_residual, phi))
        finally:
            sim.close()
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])


def test_multigrid_rejects_grids_that_do_not_halve():
    sim = _sim(125)  # 126 nodes: 125 cells do not halve, 126^2 > 9000
    try:
        assert sim.lib.pic_multigrid_setup(sim.mesh.ptr, 4500) == api.PIC_ERR_ARG
        assert b"halve" in sim.lib.pic_last_error()
        assert sim.lib.pic_multigrid_setup(sim.mesh.ptr, 9001) == api.PIC_ERR_ARG
        # the two-level space still works on such a grid (5-cell coarse spacing)
        sim.set_field("rho", np.random.default_rng(2).standard_normal(sim.mesh.nn))
        sim.set_field("phi", np.zeros(sim.mesh.nn))
        sim.set_solver("fcg", coarse_cells=25)
        st = api.SolveStats()
        api.check(sim.lib.pic_ife_solve(None, 0.0, C.byref(st)), "pic_ife_solve")
        assert st.fallback == 0 and st.rel_residual <= 1e-8
    finally:
        sim.close()
