"""Input decks of the IFE-PIC step: the benchmark configurations, the
reference normalisation (Input_2D.f90:362-392), the mesh built by the
library's mesh builder, and the seeded particle loader.

All lengths handed to the library are normalised by L_ref (the Debye length
at n_ref = n0, T_ref = Te), potentials by Phi_ref = kB*T_ref/e, velocities by
v_ref = sqrt(kB*T_ref/m_e) and time by time_ref = 1/omega_pe.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import api

KB = 1.3807e-23
QE = 1.6022e-19
ME = 9.1095e-31
AMU = 1.660539040e-27
EPS0 = 8.8542e-12
EVTOK = 11605.0
AR_MASS = 39.95 * AMU


def reference_scales(n_ref: float, T_eV: float) -> dict:
    """L_ref, time_ref, v_ref, Phi_ref exactly as Input_2D.f90:362-392."""
    T_ref = T_eV * EVTOK
    return {
        "L_ref": math.sqrt(EPS0 * KB * T_ref / n_ref / QE / QE),
        "time_ref": math.sqrt(EPS0 * ME / n_ref / QE / QE),
        "v_ref": math.sqrt(KB * T_ref / ME),
        "Phi_ref": KB * T_ref / QE,
    }


@dataclass
class ObjectSpec:
    shape: int                 # api.PIC_SHAPE_*
    cx: float                  # m
    cy: float
    a: float                   # radius / semi-axis / box upper-right x (m)
    b: float = 0.0
    angle: float = 0.0
    eps: float = 1.0
    conductor: bool = False
    phi_V: float = 0.0


@dataclass
class Config:
    name: str
    Lx: float
    Ly: float
    ncx: int
    ncy: int
    objects: list = field(default_factory=list)
    wall_dirichlet: tuple = (1, 1, 1, 1)    # left, right, bottom, top
    wall_V: tuple = (0.0, 0.0, 0.0, 0.0)
    wall_particles: tuple = (0, 0, 0, 0)    # api.PIC_WALL_*
    n0: float = 1e15
    ppc: int = 50
    Te_eV: float = 2.0
    Ti_eV: float = 0.026
    gas_p_Pa: float = 1.33
    gas_T_K: float = 300.0
    dt: float = 0.05
    nt: int = 1000
    pcg_tol: float = 1e-10
    pcg_maxit: int = 50000
    seed: int = 0
    mcc: bool = True
    precision: int = api.PIC_PREC_FP64
    sort_interval: int = 10
    # 0: Cartesian x-y; 1: axisymmetric, x = z and y = r with the axis at y = 0
    delta: int = 0
    # (wall, volts, frequency_hz[, phase]): RF potential added to the Dirichlet
    # wall x = xmin (0) or x = xmax (1); None: static walls
    rf: tuple | None = None
    # per-node energy deposit (a diagnostic) only on output steps; the
    # reference writes its profiles every 1000 steps (Main_IFE_Test_2.f90:466-470)
    diag_interval: int = 1000

    @property
    def scales(self) -> dict:
        return reference_scales(self.n0, self.Te_eV)


def _seeded_disks(rng, n, Lx, Ly, rmin, rmax, margin):
    disks = []
    for _ in range(10000):
        if len(disks) == n:
            break
        r = rng.uniform(rmin, rmax)
        cx = rng.uniform(r + margin, Lx - r - margin)
        cy = rng.uniform(r + margin, Ly - r - margin)
        if all(math.hypot(cx - x, cy - y) > r + rr + margin for x, y, rr in disks):
            disks.append((cx, cy, r))
    if len(disks) < n:
        raise RuntimeError("could not place non-overlapping objects")
    return disks


def config(name: str, **over) -> Config:
    """The five benchmark decks (seeded; geometry in metres)."""
    if name == "cfg1":
        c = Config("cfg1-64x64-disk", 0.04, 0.04, 64, 64,
                   objects=[ObjectSpec(api.PIC_SHAPE_CIRCLE, 0.02, 0.02, 0.008, eps=4.0)],
                   wall_V=(50.0, 0.0, 0.0, 0.0), n0=1e15, ppc=50, Te_eV=2.0, nt=1000,
                   pcg_tol=1e-10, seed=0)
    elif name == "cfg2":
        rng = np.random.default_rng(20240602)
        disks = _seeded_disks(rng, 4, 0.16, 0.16, 0.01, 0.02, 0.004)
        eps = [2.0, 4.0, 10.0]
        objs = [ObjectSpec(api.PIC_SHAPE_CIRCLE, x, y, r, eps=eps[k]) for k, (x, y, r) in
                enumerate(disks[:3])]
        x, y, r = disks[3]
        objs.append(ObjectSpec(api.PIC_SHAPE_CIRCLE, x, y, r, conductor=True, phi_V=-20.0))
        c = Config("cfg2-512x512-4disks", 0.16, 0.16, 512, 512, objects=objs,
                   wall_V=(0.0, 0.0, 0.0, 0.0), n0=5e15, ppc=100, Te_eV=3.0, nt=2000,
                   pcg_tol=1e-10, seed=1)
    elif name == "cfg3":
        c = Config("cfg3-1024x1024-disk-mixed", 0.04, 0.04, 1024, 1024,
                   objects=[ObjectSpec(api.PIC_SHAPE_CIRCLE, 0.02, 0.02, 0.008, eps=4.0)],
                   wall_V=(50.0, 0.0, 0.0, 0.0), n0=1e15, ppc=64, Te_eV=2.0, nt=1000,
                   pcg_tol=1e-8, seed=0, precision=api.PIC_PREC_MIXED)
    elif name == "cfg4":
        rng = np.random.default_rng(20240604)
        objs = []
        placed = []
        while len(objs) < 8:
            a, b = rng.uniform(0.005, 0.03, size=2)
            ang = rng.uniform(0, math.pi)
            R = max(a, b)
            cx = rng.uniform(R + 0.004, 0.16 - R - 0.004)
            cy = rng.uniform(R + 0.004, 0.16 - R - 0.004)
            if all(math.hypot(cx - x, cy - y) > R + rr + 0.004 for x, y, rr in placed):
                placed.append((cx, cy, R))
                eps = math.exp(rng.uniform(0.0, math.log(20.0)))
                objs.append(ObjectSpec(api.PIC_SHAPE_ELLIPSE, cx, cy, a, b, ang, eps=eps))
        c = Config("cfg4-1024x1024-8ellipses", 0.16, 0.16, 1024, 1024, objects=objs,
                   wall_V=(0.0, 0.0, 0.0, 0.0), n0=5e15, ppc=64, Te_eV=3.0, nt=5000,
                   pcg_tol=1e-8, seed=4, sort_interval=20)
        # counting sort every 20 steps: 6.10 ms/step against 6.23 with 10 and
        # 6.55 with 5 (B200; the push slows only slightly as particles leave
        # their sorted cells)
    elif name == "tiny":
        c = Config("tiny-16x16-disk", 0.01, 0.01, 16, 16,
                   objects=[ObjectSpec(api.PIC_SHAPE_CIRCLE, 0.005, 0.0051, 0.0023, eps=4.0)],
                   wall_V=(5.0, 0.0, 0.0, 0.0), n0=1e15, ppc=8, Te_eV=2.0, nt=10,
                   pcg_tol=1e-10, seed=3)
    elif name == "cfg5":
        # r-z capacitively coupled cell: z = x in [0, 0.2] m (2048 cells), r =
        # y in [0, 0.1] m (1024 cells), the axis at r = 0; 200 V at 13.56 MHz
        # on the electrode z = 0, grounded z = 0.2 m and r = 0.1 m; a
        # dielectric wafer (eps 3.9, 1 mm thick, r < 0.075 m) 10 mm above the
        # electrode.  r = 0.075 m is the node line j = 768, where the interface
        # would pass through vertices: the wafer's edge sits a quarter cell
        # further out.  Mixed precision, as the benchmark decks 3 and 4.
        r_wafer = 0.075 + 0.25 * 0.1 / 1024
        c = Config("cfg5-axi-2048x1024-rf-wafer", 0.2, 0.1, 2048, 1024,
                   objects=[ObjectSpec(api.PIC_SHAPE_BOX, 0.010, -0.001, 0.011, r_wafer, eps=3.9)],
                   wall_dirichlet=(1, 1, 0, 1), wall_V=(0.0, 0.0, 0.0, 0.0), n0=1e16, ppc=32,
                   Te_eV=3.0, gas_p_Pa=2.66, nt=20000, pcg_tol=1e-8, seed=5, delta=1,
                   rf=(0, 200.0, 13.56e6), precision=api.PIC_PREC_MIXED)
    elif name == "tiny_axi":
        # r-z cylinder (z = x, r = y, axis at the bottom: a symmetry line, not
        # a wall) holding a dielectric torus; Dirichlet on the ends and the
        # outer radius
        c = Config("tiny-axi-16x16-torus", 0.01, 0.01, 16, 16,
                   objects=[ObjectSpec(api.PIC_SHAPE_CIRCLE, 0.005, 0.0055, 0.0023, eps=4.0)],
                   wall_dirichlet=(1, 1, 0, 1), wall_V=(5.0, 0.0, 0.0, 0.0), n0=1e15, ppc=8,
                   Te_eV=2.0, nt=10, pcg_tol=1e-10, seed=5, delta=1)
    else:
        raise KeyError(name)
    for k, v in over.items():
        setattr(c, k, v)
    return c


def make_deck(cfg: Config) -> api.Deck:
    sc = cfg.scales
    L, P = sc["L_ref"], sc["Phi_ref"]
    d = api.Deck()
    d.nnx, d.nny = cfg.ncx + 1, cfg.ncy + 1
    d.xmin, d.xmax, d.ymin, d.ymax = 0.0, cfg.Lx / L, 0.0, cfg.Ly / L
    d.delta = cfg.delta
    for k in range(4):
        d.wall_dirichlet[k] = int(cfg.wall_dirichlet[k])
        d.wall_phi[k] = cfg.wall_V[k] / P
    d.n_objects = len(cfg.objects)
    for k, o in enumerate(cfg.objects):
        t = d.objects[k]
        t.shape = o.shape
        t.conductor = int(o.conductor)
        t.cx, t.cy = o.cx / L, o.cy / L
        if o.shape == api.PIC_SHAPE_BOX:
            t.a, t.b = o.a / L, o.b / L
        else:
            t.a = o.a / L
            t.b = (o.b if o.b else o.a) / L
        t.angle = o.angle
        t.eps = o.eps
        t.phi = o.phi_V / P
    return d


def _cuda_visible() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


class Mesh:
    """Mesh built by the library; owns the library storage.  device: the
    interface elements' basis and element matrices computed on the CUDA device
    (pic_mesh_build_device; the same bits as the host builder); None picks
    the device when one is visible."""

    def __init__(self, cfg: Config, device: bool | None = None):
        lib = api.load()
        self.cfg = cfg
        self.deck = make_deck(cfg)
        self.ptr = C.POINTER(api.MeshDesc)()
        if device is None:
            device = _cuda_visible()
        build = lib.pic_mesh_build_device if device else lib.pic_mesh_build
        api.check(build(C.byref(self.deck), C.byref(self.ptr)),
                  "pic_mesh_build_device" if device else "pic_mesh_build")
        self.desc = self.ptr.contents
        d = self.desc
        self.nnx, self.nny = d.nnx, d.nny
        self.nn = d.nnx * d.nny
        self.ne = (d.nnx - 1) * (d.nny - 1)
        self.hx = (d.xmax - d.xmin) / (d.nnx - 1)
        self.hy = (d.ymax - d.ymin) / (d.nny - 1)

    def array(self, name: str) -> np.ndarray:
        d = self.desc
        sizes = {"node_type": self.nn, "node_index": self.nn, "element_index": self.ne,
                 "phi_dirichlet": self.nn, "cell_volume": self.nn,
                 "a_srow": d.n_unknowns + 1, "a_jcol": d.nnz, "a_k": d.nnz,
                 "xt_srow": d.n_unknowns + 1, "xt_jcol": d.nnz_xt, "xt_k": d.nnz_xt,
                 "a_diag": d.n_unknowns, "rhs_fix": d.n_unknowns, "mass_q1": 16,
                 "ife_mass": 16 * d.n_interface, "patch_ptr": self.nn + 1,
                 "mass_rows": 16 * (self.nny - 1)}
        if name == "patch_nodes":
            n = int(self.array("patch_ptr")[-1])
        else:
            n = sizes[name]
        ptr = getattr(d, name)
        dt = np.float64 if ptr._type_ is C.c_double else np.int32
        return api.as_np(ptr, int(n), dt)

    def close(self):
        if self.ptr:
            api.load().pic_mesh_free(self.ptr)
            self.ptr = C.POINTER(api.MeshDesc)()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def species_params(cfg: Config):
    """[(charge, mass, weight, sigma_v_normalised)] for e- and Ar+."""
    sc = cfg.scales
    L = sc["L_ref"]
    hx_m, hy_m = cfg.Lx / cfg.ncx, cfg.Ly / cfg.ncy
    if cfg.delta == 1:
        # real particles per macro-particle: n0 times the cylinder's volume over
        # the particle count (ppc per cell on average)
        weight = cfg.n0 * math.pi * cfg.Ly * cfg.Ly * cfg.Lx / (cfg.ncx * cfg.ncy * cfg.ppc)
    else:
        weight = cfg.n0 * hx_m * hy_m / cfg.ppc  # per unit depth
    out = []
    for q, m, T in ((-1.0, ME, cfg.Te_eV), (1.0, AR_MASS, cfg.Ti_eV)):
        sigma = math.sqrt(KB * T * EVTOK / m) / sc["v_ref"]
        out.append((q, m, weight, sigma))
    return out, L


def _inside(o, x, y):
    """Particles strictly inside object o (the test k_push and the oracle
    apply), elementwise on arrays."""
    if o.shape == api.PIC_SHAPE_CIRCLE:
        return (x - o.cx) ** 2 + (y - o.cy) ** 2 < o.a * o.a
    if o.shape == api.PIC_SHAPE_BOX:
        return (x > o.cx) & (x < o.a) & (y > o.cy) & (y < o.b)
    if o.shape == api.PIC_SHAPE_ELLIPSE:
        c, s = math.cos(o.angle), math.sin(o.angle)
        u = (x - o.cx) * c + (y - o.cy) * s
        v = -(x - o.cx) * s + (y - o.cy) * c
        return u * u / (o.a * o.a) + v * v / (o.b * o.b) < 1.0
    return np.zeros(x.shape, dtype=bool)


def _cells_box(o, mesh, ncell, ncy, ppc):
    """Indices of the loaded particles whose cell meets object o's bounding
    box (particles are generated cell by cell, ppc per cell, cell = i*ncy + j,
    so a box is one index range per cell column); only they can be inside."""
    if o.shape == api.PIC_SHAPE_BOX:
        x0, x1, y0, y1 = o.cx, o.a, o.cy, o.b
    else:
        r = o.a if o.shape == api.PIC_SHAPE_CIRCLE else max(o.a, o.b)
        x0, x1, y0, y1 = o.cx - r, o.cx + r, o.cy - r, o.cy + r
    i0 = max(int(math.floor(x0 / mesh.hx)) - 1, 0)
    i1 = int(math.floor(x1 / mesh.hx)) + 1
    j0 = max(int(math.floor(y0 / mesh.hy)) - 1, 0)
    j1 = min(int(math.floor(y1 / mesh.hy)) + 1, ncy - 1)
    parts = []
    for i in range(i0, i1 + 1):
        c0, c1 = i * ncy + j0, min(i * ncy + j1, ncell - 1)
        if c0 >= ncell or c1 < c0:
            continue
        parts.append(np.arange(c0 * ppc, (c1 + 1) * ppc, dtype=np.int64))
    return np.concatenate(parts) if parts else np.zeros(0, dtype=np.int64)


def _load_axi(cfg: Config, mesh: Mesh, rng, sigma, ncell):
    """Uniform in volume on an r-z mesh, the distribution of the reference's
    equal-weight loading (MCC_jw/code/base/ParticleOne.f90,
    PositionRandomInitializationParticleOne for delta 1: r = sqrt(r0^2 +
    u (r1^2 - r0^2))), drawn cell by cell: cell (i, j) holds ppc (2j + 1)/ncy
    particles on average (its ring's share of the cylinder; stochastic
    rounding), r drawn with density proportional to r inside the cell."""
    ncy = cfg.ncy
    cell = np.arange(ncell, dtype=np.int64)
    cj = cell % ncy
    mean = cfg.ppc * (2.0 * cj + 1.0) / ncy
    counts = np.floor(mean + rng.random(ncell)).astype(np.int64)
    cells = np.repeat(cell, counts)
    n = cells.size
    ci, cj = cells // ncy, cells % ncy
    x = (ci + rng.random(n)) * mesh.hx
    r0, r1 = cj * mesh.hy, (cj + 1) * mesh.hy
    y = np.sqrt(r0 * r0 + rng.random(n) * (r1 * r1 - r0 * r0))
    keep = np.ones(n, dtype=bool)
    dk = mesh.deck
    for k in range(dk.n_objects):
        keep &= ~_inside(dk.objects[k], x, y)
    x, y = x[keep], y[keep]
    v = rng.standard_normal((3, x.size)) * sigma
    return (np.ascontiguousarray(x), np.ascontiguousarray(y), np.ascontiguousarray(v[0]),
            np.ascontiguousarray(v[1]), np.ascontiguousarray(v[2]))


def load_particles(cfg: Config, mesh: Mesh, species: int, n_cells_limit: int | None = None):
    """Seeded uniform loading, ppc per cell, outside the objects; Maxwellian
    velocities (on an r-z mesh: uniform in volume, vz = v_theta)."""
    sp, _ = species_params(cfg)
    sigma = sp[species][3]
    rng = np.random.default_rng([cfg.seed, species, 7919])
    ncx, ncy = cfg.ncx, cfg.ncy
    ncell = ncx * ncy if n_cells_limit is None else min(n_cells_limit, ncx * ncy)
    if cfg.delta == 1:
        return _load_axi(cfg, mesh, rng, sigma, ncell)
    cell = np.arange(ncell, dtype=np.int64)
    ci, cj = cell // ncy, cell % ncy
    n = ncell * cfg.ppc
    x = (np.repeat(ci, cfg.ppc) + rng.random(n)) * mesh.hx
    y = (np.repeat(cj, cfg.ppc) + rng.random(n)) * mesh.hy
    keep = np.ones(n, dtype=bool)
    dk = mesh.deck
    for k in range(dk.n_objects):
        o = dk.objects[k]
        idx = _cells_box(o, mesh, ncell, ncy, cfg.ppc)
        xs, ys = x[idx], y[idx]
        keep[idx] &= ~_inside(o, xs, ys)
    x, y = x[keep], y[keep]
    m = x.size
    v = rng.standard_normal((3, m)) * sigma
    return (np.ascontiguousarray(x), np.ascontiguousarray(y), np.ascontiguousarray(v[0]),
            np.ascontiguousarray(v[1]), np.ascontiguousarray(v[2]))
