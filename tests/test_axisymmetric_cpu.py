"""Axisymmetric (r-z, delta = 1) assembly of the mesh builder, checked on
the CPU with a direct sparse solve: the dual volumes of the reference
(SetupGrids_2D_QLL.f90:233-289) sum to the cylinder's volume, a
manufactured solution of -(1/r) d/dr(r dphi/dr) - d2phi/dz2 = f converges
at second order through the r-weighted stiffness and load matrices, and a
dielectric slab across the whole radius gives the exact piecewise-linear
potential through the r-weighted interface-element matrices."""
import ctypes as C
import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import oracle_bind as ob
from pic_b200 import api


class _AxiMesh:
    """pic_mesh_build of an r-z box: z = x in [0, lz], r = y in [0, rr]."""

    def __init__(self, nz, nr, lz, rr, walls, wall_phi=(0.0, 0.0, 0.0, 0.0), objects=()):
        d = api.Deck()
        d.nnx, d.nny = nz + 1, nr + 1
        d.xmin, d.xmax, d.ymin, d.ymax = 0.0, lz, 0.0, rr
        d.delta = 1
        for k in range(4):
            d.wall_dirichlet[k] = walls[k]
            d.wall_phi[k] = wall_phi[k]
        d.n_objects = len(objects)
        for k, o in enumerate(objects):
            d.objects[k] = o
        self.lib = api.load()
        self.ptr = C.POINTER(api.MeshDesc)()
        api.check(self.lib.pic_mesh_build(C.byref(d), C.byref(self.ptr)), "pic_mesh_build")
        self.d = self.ptr.contents
        self.nnx, self.nny = d.nnx, d.nny
        self.nn = d.nnx * d.nny
        self.x = np.repeat(np.linspace(0.0, lz, d.nnx), d.nny)
        self.y = np.tile(np.linspace(0.0, rr, d.nny), d.nnx)

    def arr(self, name, n, dtype):
        return api.as_np(getattr(self.d, name), n, dtype)

    def solve(self, rho):
        """phi on every node: A phi_u = b_u (b from the oracle's RHS), Dirichlet values kept."""
        nu = self.d.n_unknowns
        nt = self.arr("node_type", self.nn, np.int32)
        srow = self.arr("a_srow", nu + 1, np.int32)
        nnz = int(srow[-1] - 1)
        A = sp.csr_matrix((self.arr("a_k", nnz, np.float64), self.arr("a_jcol", nnz, np.int32) - 1, srow - 1),
                          shape=(nu, nu))
        b = ob.rhs(self.ptr, np.ascontiguousarray(rho, dtype=np.float64), self.nn)
        node_of = np.zeros(nu, np.int64)
        node_of[nt[nt > 0] - 1] = np.nonzero(nt > 0)[0]
        phi = self.arr("phi_dirichlet", self.nn, np.float64).copy()
        phi[node_of] = spl.spsolve(A.tocsc(), b[node_of])
        return phi

    def close(self):
        self.lib.pic_mesh_free(self.ptr)


def test_dual_volumes_sum_to_the_cylinder():
    lz, rr = 1.7, 0.9
    m = _AxiMesh(24, 18, lz, rr, (1, 1, 0, 1))
    try:
        vol = m.arr("cell_volume", m.nn, np.float64)
        assert abs(vol.sum() - math.pi * rr * rr * lz) <= 1e-12 * math.pi * rr * rr * lz
        assert np.all(vol > 0)
        assert m.d.mass_rows  # the per-row load matrices exist for delta = 1
    finally:
        m.close()


def test_manufactured_solution_converges_at_second_order():
    """Second order in the r-weighted L2 norm and in the maximum away from
    the axis (the largest error sits on the axis, where the weight r
    vanishes; it converges there too, at about 1.7)."""
    lz, rr = 2.0, 1.0
    a, b = math.pi / lz, math.pi / (2.0 * rr)
    l2, far, axis = [], [], []
    for n in (8, 16, 32):
        m = _AxiMesh(2 * n, n, lz, rr, (1, 1, 0, 1))  # the axis r = 0 is a symmetry line
        try:
            z, r = m.x, m.y
            exact = np.sin(a * z) * np.cos(b * r)
            with np.errstate(invalid="ignore", divide="ignore"):
                radial = np.where(r > 0, b * b * np.cos(b * r) + (b / r) * np.sin(b * r), 2.0 * b * b)
            f = a * a * exact + np.sin(a * z) * radial
            e = m.solve(f) - exact
            vol = m.arr("cell_volume", m.nn, np.float64)
            l2.append(math.sqrt((vol * e * e).sum() / vol.sum()))
            far.append(np.abs(e[r > 0.25 * rr]).max())
            axis.append(np.abs(e).max())
        finally:
            m.close()
    rate = lambda v: [math.log2(v[k] / v[k + 1]) for k in range(len(v) - 1)]  # noqa: E731
    print(f"\naxisymmetric manufactured solution: L2_r {l2} rates {rate(l2)}; max r>R/4 rates {rate(far)}; "
          f"max rates {rate(axis)}")
    assert min(rate(l2)) > 1.9 and min(rate(far)) > 1.9 and min(rate(axis)) > 1.5
    assert l2[-1] < 1e-4


def test_dielectric_slab_is_exact():
    """A slab of eps = 3.9 across the whole radius between z0 and z1 (not on
    grid lines), 0 V at z = 0 and 1 V at z = lz, natural conditions on the
    axis and at r = rr: phi depends on z only and is piecewise linear with
    eps * dphi/dz continuous, which the IFE space contains."""
    lz, rr, eps, v = 1.0, 0.5, 3.9, 1.0
    z0, z1 = 0.3137, 0.5071
    slab = api.Object()
    slab.shape, slab.conductor = api.PIC_SHAPE_BOX, 0
    slab.cx, slab.cy, slab.a, slab.b = z0, -1.0, z1, rr + 1.0
    slab.eps, slab.phi, slab.angle = eps, 0.0, 0.0
    m = _AxiMesh(40, 16, lz, rr, (1, 1, 0, 0), (0.0, v, 0.0, 0.0), [slab])
    try:
        assert m.d.n_interface > 0
        phi = m.solve(np.zeros(m.nn))
        w = z1 - z0
        e1 = v / (lz - w + w / eps)  # field outside the slab; inside e1 / eps
        z = m.x
        exact = np.where(z <= z0, e1 * z, np.where(z <= z1, e1 * z0 + e1 / eps * (z - z0),
                                                    e1 * z0 + e1 / eps * w + e1 * (z - z1)))
        err = np.abs(phi - exact).max()
        print(f"\naxisymmetric dielectric slab: max |phi - exact| = {err:.2e}")
        assert err <= 1e-10
    finally:
        m.close()


def test_dielectric_rod_converges_to_the_cylindrical_solution():
    """A rod of eps = 3.9 along the axis (r < r0, every z) in uniform charge
    rho = 1, phi = 0 at r = rr, natural conditions elsewhere: phi depends on
    r only, -(1/r)(r eps phi')' = 1, so phi = (rr^2 - r^2)/4 outside and
    (rr^2 - r0^2)/4 + (r0^2 - r^2)/(4 eps) inside.  A Cartesian weighting
    would converge to twice that; the r-weighted interface-element matrices
    converge to it at second order."""
    lz, rr, eps, r0 = 0.6, 1.0, 3.9, 0.4137
    rod = api.Object()
    rod.shape, rod.conductor = api.PIC_SHAPE_BOX, 0
    rod.cx, rod.cy, rod.a, rod.b = -1.0, -1.0, lz + 1.0, r0
    rod.eps, rod.phi, rod.angle = eps, 0.0, 0.0
    l2 = []
    for n in (8, 16, 32):
        m = _AxiMesh(n, 2 * n, lz, rr, (0, 0, 0, 1), objects=[rod])
        try:
            assert m.d.n_interface > 0
            phi = m.solve(np.ones(m.nn))
            r = m.y
            exact = np.where(r >= r0, (rr * rr - r * r) / 4.0, (rr * rr - r0 * r0) / 4.0 + (r0 * r0 - r * r) / (4.0 * eps))
            vol = m.arr("cell_volume", m.nn, np.float64)
            e = phi - exact
            l2.append(math.sqrt((vol * e * e).sum() / vol.sum()))
        finally:
            m.close()
    rates = [math.log2(l2[k] / l2[k + 1]) for k in range(2)]
    print(f"\naxisymmetric dielectric rod: L2_r errors {l2}, rates {rates}")
    assert min(rates) > 1.8 and l2[-1] < 1e-4


# ---- the oracle's axisymmetric push and deposit (MoveOne.f90:213-263,
# GetParChg_2D.f90:803-821)

def _axi_parts(m, n, seed=4, lz=2.0, rr=1.0, vscale=0.02):
    """Particles well inside the domain (they stay inside over the tests' moves)."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(0.3 * lz, 0.7 * lz, n)
    r = rng.uniform(0.0, 0.6 * rr, n)
    loc = np.array([ob.load().or_locate(m.ptr, a, b) for a, b in zip(z, r)], np.int32)
    v = rng.standard_normal((3, n)) * vscale
    return {"x": z, "y": r, "vx": v[0].copy(), "vy": v[1].copy(), "vz": v[2].copy(), "loc": loc}


def test_axi_push_free_streaming_is_the_straight_line():
    """No field: every step moves the particle on its 3D straight line; the
    radius after k steps is |(r0 + t v_r0, t v_theta0)|, the speed and the
    angular momentum r v_theta are conserved."""
    lz, rr = 2.0, 1.0
    m = _AxiMesh(32, 16, lz, rr, (1, 1, 0, 1))
    try:
        p = _axi_parts(m, 400)
        p0 = {k: v.copy() for k, v in p.items()}
        zeros = np.zeros(m.nn)
        coef = np.zeros(5 * m.nn)
        dt, steps = 0.37, 12
        for _ in range(steps):
            for k in range(len(p["loc"])):  # re-locate as the step does after the push
                if p["loc"][k] >= 0:
                    p["loc"][k] = ob.load().or_locate(m.ptr, p["x"][k], p["y"][k])
            ob.move_all_axi(m.ptr, p, zeros, zeros, coef, -1.0, dt)
        live = p["loc"] >= 0
        assert live.all()
        t = dt * steps
        r_line = np.hypot(p0["y"] + t * p0["vy"], t * p0["vz"])
        assert np.allclose(p["y"], r_line, rtol=1e-12, atol=1e-14)
        assert np.allclose(p["x"], p0["x"] + t * p0["vx"], rtol=1e-13, atol=0)
        speed0 = np.sqrt(p0["vx"] ** 2 + p0["vy"] ** 2 + p0["vz"] ** 2)
        assert np.allclose(np.sqrt(p["vx"] ** 2 + p["vy"] ** 2 + p["vz"] ** 2), speed0, rtol=1e-13, atol=0)
        assert np.allclose(p["y"] * p["vz"], p0["y"] * p0["vz"], rtol=1e-11, atol=1e-15)
    finally:
        m.close()


def test_axi_push_axial_field():
    lz, rr = 2.0, 1.0
    m = _AxiMesh(32, 16, lz, rr, (1, 1, 0, 1))
    try:
        p = _axi_parts(m, 300)
        p0 = {k: v.copy() for k, v in p.items()}
        e0, qm, dt = 0.21, -1.0, 0.1
        efx, efy = np.full(m.nn, e0), np.zeros(m.nn)
        coef = np.zeros((5, m.nn))
        coef[0] = -e0
        ob.move_all_axi(m.ptr, p, efx, efy, np.ascontiguousarray(coef.ravel()), qm, dt)
        want = p0["vx"] + qm * e0 * dt
        assert np.allclose(p["vx"], want, rtol=0, atol=1e-15)
        assert np.allclose(p["x"], p0["x"] + dt * p["vx"], rtol=0, atol=1e-15)
    finally:
        m.close()


def test_axi_push_radial_field_without_swirl():
    """A uniform radial field and no azimuthal velocity: the move stays in
    the r-z plane, so it is the 1-D leapfrog v_r += qm E_r dt, r += dt v_r
    (the interface elements' PPR gradient carries the same field)."""
    lz, rr = 2.0, 1.0
    m = _AxiMesh(32, 16, lz, rr, (1, 1, 0, 1))
    try:
        p = _axi_parts(m, 300)
        p["vz"][:] = 0.0
        p["y"] = 0.2 + 0.3 * p["y"]  # off the axis: r stays positive over the step
        p["loc"] = np.array([ob.load().or_locate(m.ptr, a, b) for a, b in zip(p["x"], p["y"])], np.int32)
        p0 = {k: v.copy() for k, v in p.items()}
        e1, qm, dt = 0.17, -1.0, 0.1
        efx, efy = np.zeros(m.nn), np.full(m.nn, e1)
        coef = np.zeros((5, m.nn))
        coef[1] = -e1
        ob.move_all_axi(m.ptr, p, efx, efy, np.ascontiguousarray(coef.ravel()), qm, dt)
        assert np.all(p["loc"] >= 0)
        vr = p0["vy"] + qm * e1 * dt
        assert np.allclose(p["vy"], vr, rtol=0, atol=1e-15)
        assert np.allclose(p["y"], p0["y"] + dt * vr, rtol=0, atol=1e-15)
        assert np.all(p["vz"] == 0.0)
    finally:
        m.close()


def test_axi_deposit_splits_a_uniform_ring_evenly():
    """Particles on a node line in z and uniform in r^2 across one element
    row (equal volume each) give its lower and upper nodes half the charge
    each: the weights are linear in r^2 (the midpoint rule in r^2 is exact).
    On the axis row the lower node keeps the reference's 0.75 of its half."""
    lz, rr = 2.0, 1.0
    m = _AxiMesh(8, 8, lz, rr, (1, 1, 0, 1))
    try:
        hy = rr / 8
        npart = 1000
        for j in (0, 3):
            r1, r2 = j * hy, (j + 1) * hy
            r = np.sqrt(r1 * r1 + (np.arange(npart) + 0.5) / npart * (r2 * r2 - r1 * r1))
            z = np.full(npart, 4 * (lz / 8))  # node column i = 4
            parts = {"x": z, "y": r, "vx": np.zeros(npart), "vy": np.zeros(npart), "vz": np.zeros(npart),
                     "loc": np.zeros(npart, np.int32)}
            q, _, bad = ob.deposit(m.ptr, parts, 9.1e-31, 1.0, m.nn)
            assert bad == 0
            lower, upper = q[4 * m.nny + j] / 2.0 ** 40, q[4 * m.nny + j + 1] / 2.0 ** 40
            beta = 0.75 if j == 0 else 1.0
            assert abs(lower - beta * npart / 2) <= 1e-9 * npart
            assert abs(upper - npart / 2) <= 1e-9 * npart
    finally:
        m.close()


def test_pic_init_refuses_an_axisymmetric_mesh_off_the_axis():
    """The r-z push and deposit take the axis at y = ymin = 0: pic_init turns
    down delta = 1 with ymin != 0 before it touches the device."""
    from pic_b200 import deck
    cfg = deck.config("tiny_axi", objects=[])
    d = deck.make_deck(cfg)
    d.ymin, d.ymax = 0.5, 0.5 + d.ymax
    lib = api.load()
    ptr = C.POINTER(api.MeshDesc)()
    api.check(lib.pic_mesh_build(C.byref(d), C.byref(ptr)), "pic_mesh_build")
    try:
        p = api.Params()
        p.n_species = 1
        p.species[0].charge, p.species[0].mass, p.species[0].weight = -1.0, deck.ME, 1.0
        p.species[0].capacity = 1024
        p.dt, p.n_ref, p.T_ref_eV = cfg.dt, cfg.n0, cfg.Te_eV
        p.pcg_tol, p.pcg_maxit = cfg.pcg_tol, cfg.pcg_maxit
        assert lib.pic_init(ptr, C.byref(p)) == api.PIC_ERR_ARG
        assert b"ymin = 0" in lib.pic_last_error()
    finally:
        lib.pic_mesh_free(ptr)


def test_uniform_plasma_deposits_the_density():
    """Particles uniform in volume with weight n0 V / N deposit rho = n0
    (normalised: 1) at every node off the axis, through the r^2-linear
    weights, the L_ref^3 normalisation (GetParChg_2D.f90:900-904) and the
    axisymmetric dual volumes; the axis row reads 1.5 n0, the reference's
    axis factor beta = 0.75 applied to weights whose integral over the first
    ring is twice the axis node's dual volume."""
    lz, rr, L_ref, n0 = 2.0, 1.5, 1e-3, 1e15
    m = _AxiMesh(16, 12, lz, rr, (1, 1, 0, 1))
    try:
        rng = np.random.default_rng(17)
        N = 4_000_000
        z = rng.random(N) * lz
        r = rr * np.sqrt(rng.random(N))
        zero = np.zeros(N)
        parts = {"x": z, "y": r, "vx": zero, "vy": zero, "vz": zero, "loc": np.zeros(N, np.int32)}
        q, e, bad = ob.deposit(m.ptr, parts, 1.0, 1.0, m.nn)
        assert bad == 0
        weight = n0 * math.pi * (rr * L_ref) ** 2 * (lz * L_ref) / N
        _, rs, _ = ob.normalize(m.ptr, [q], [e], [weight], L_ref, n0, m.nn)
        rho = rs[0].reshape(m.nnx, m.nny)
        inner = rho[1:-1, 1:-1]
        assert abs(inner.mean() - 1.0) < 5e-3
        assert np.abs(inner - 1.0).max() < 0.1
        assert abs(rho[1:-1, 0].mean() - 1.5) < 0.06
    finally:
        m.close()


def test_deck_loading_is_uniform_in_volume():
    """The r-z deck loader (counts per cell by ring volume, r drawn with
    density r) with its macro-weight n0 V / N deposits rho_s = n0 off the axis
    through the oracle's deposit and normalisation."""
    from pic_b200 import deck
    cfg = deck.config("tiny_axi", objects=[], ppc=2000)
    mesh = deck.Mesh(cfg)
    try:
        x, y, vx, vy, vz = deck.load_particles(cfg, mesh, 1)
        n_mean = cfg.ncx * cfg.ncy * cfg.ppc
        assert abs(x.size - n_mean) < 5 * math.sqrt(n_mean)
        sp, L = deck.species_params(cfg)
        parts = {"x": x, "y": y, "vx": vx, "vy": vy, "vz": vz, "loc": np.zeros(x.size, np.int32)}
        q, e, bad = ob.deposit(mesh.ptr, parts, 1.0, 1.0, mesh.nn)
        assert bad == 0
        _, rs, _ = ob.normalize(mesh.ptr, [q], [e], [sp[1][2] * sp[1][0]], L, cfg.n0, mesh.nn)
        rho = rs[0].reshape(mesh.nnx, mesh.nny)
        inner = rho[1:-1, 1:-1]
        assert abs(inner.mean() - 1.0) < 5e-3
        assert np.abs(inner - 1.0).max() < 0.08
    finally:
        mesh.close()


def test_cfg5_mesh_builds():
    """The config-5 geometry (r-z, a wafer box crossing the axis) assembles;
    the wafer's elements are interface elements along its top, bottom and
    outer faces."""
    from pic_b200 import deck
    cfg = deck.config("cfg5")
    mesh = deck.Mesh(cfg)
    try:
        d = mesh.desc
        assert d.delta == 1 and d.n_interface > 0 and d.mass_rows
        nt = mesh.array("node_type").reshape(mesh.nnx, mesh.nny)
        assert np.all(nt[0] <= 0) and np.all(nt[-1] <= 0) and np.all(nt[:, -1] <= 0)
        assert np.all(nt[1:-1, 0] > 0)  # the axis is not a wall
        sp, _ = deck.species_params(cfg)
        assert abs(sp[0][2] * cfg.ncx * cfg.ncy * cfg.ppc - cfg.n0 * math.pi * 0.1 ** 2 * 0.2) < 1e-6 * cfg.n0
    finally:
        mesh.close()
