"""ctypes binding of the CPU oracle (oracle/liboracle.so), test infrastructure."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from pic_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")

_P = C.POINTER
_d = _P(C.c_double)
_i = _P(C.c_int32)
_u = _P(C.c_uint32)
_l = _P(C.c_int64)

_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("oracle.c", "oracle_mesh.c", "oracle_tables.c")]
    if not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < max(map(os.path.getmtime, srcs)):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    lib = C.CDLL(ORACLE_LIB)
    M = _P(api.MeshDesc)
    lib.or_reference_scales.argtypes = [C.c_double, C.c_double, _d]
    lib.or_philox.argtypes = [_u, _u, _u]
    lib.or_locate.argtypes = [M, C.c_double, C.c_double]
    lib.or_move_all.argtypes = [M, C.c_int64, _d, _d, _d, _d, _d, _i, _d, _d, _d, C.c_double,
                                C.c_double, _i]
    lib.or_move_all.restype = C.c_int64
    lib.or_deposit.argtypes = [M, C.c_int64, _d, _d, _d, _d, _d, _i, C.c_double, C.c_double, _l, _l]
    lib.or_deposit.restype = C.c_int64
    lib.or_normalize.argtypes = [M, C.c_int, _P(_l), _P(_l), _d, C.c_double, C.c_double, _d,
                                 _P(_d), _P(_d)]
    lib.or_rhs.argtypes = [M, _d, _d]
    lib.or_pcg.argtypes = [M, _d, _d, C.c_double, C.c_int, _d]
    lib.or_threads.restype = C.c_int
    lib.or_ppr.argtypes = [M, _d, _d, _d, _d]
    lib.or_sort_perm.argtypes = [C.c_int64, _i, _u, _l]
    lib.or_sort_perm.restype = C.c_int64
    lib.or_canon_dot.argtypes = [_d, _d, C.c_int64]
    lib.or_canon_dot.restype = C.c_double
    lib.or_mcc.argtypes = [_P(api.MccTable), _P(api.Gas), C.c_double, C.c_double, C.c_uint64,
                           C.c_uint64, C.c_int32, C.c_int64, _i, _u, _d, _d, _d, _l, _l, _l, _d, _d]
    lib.or_mcc.restype = C.c_int64
    lib.or_mcc_select_keys.argtypes = [C.c_uint64, C.c_uint64, C.c_int32, C.c_int64, _u, _u]
    lib.or_ife_closed_form.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                       C.c_double, _d]
    lib.or_ek_tot.argtypes = [M, _l, C.c_double, C.c_double, C.c_double, _d]
    lib.or_move_all_axi.argtypes = [M, C.c_int64, _d, _d, _d, _d, _d, _i, _d, _d, _d, C.c_double,
                                    C.c_double, _i]
    lib.or_move_all_axi.restype = C.c_int64
    lib.or_average_x.argtypes = [C.c_int, C.c_int, _d, C.c_double, _d]
    lib.or_energy_spectrum.argtypes = [C.c_int64, _d, _d, _d, _i, C.c_double, C.c_double, C.c_int,
                                       C.c_double, C.c_double, _l, _l]
    lib.or_velocity_moments.argtypes = [C.c_int64, _d, _d, _d, _d, _i, C.c_int, _l, _d, _d]
    lib.or_mesh_build.argtypes = [_P(api.Deck), C.c_int, _P(M)]
    lib.or_mesh_build.restype = C.c_int
    lib.or_mesh_free.argtypes = [M]
    lib.or_mesh_interface.argtypes = [M, C.c_int32, _i, _i, _i, _d, _d, _d]
    lib.or_quad_constants.argtypes = [C.c_int, _d]
    lib.or_mcc_sigma.argtypes = [C.c_int, _d, _d, C.c_double, C.c_double, C.c_double, C.c_int, _d]
    lib.or_mcc_sigma.restype = C.c_int
    lib.or_mcc_probability.argtypes = [C.c_int, C.c_int, _d, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_double, _d, _d]
    _lib = lib
    return lib


def d(a):
    return a.ctypes.data_as(_d)


def i32(a):
    return a.ctypes.data_as(_i)


def u32(a):
    return a.ctypes.data_as(_u)


def i64(a):
    return a.ctypes.data_as(_l)


def scales(n_ref, T_eV):
    out = np.zeros(4)
    load().or_reference_scales(n_ref, T_eV, d(out))
    return out


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    load().or_philox(c, k, o)
    return list(o)


def move_all(mesh_ptr, parts, efx, efy, coef, qm, dt, wall=(0, 0, 0, 0)):
    """parts: dict x,y,vx,vy,vz,loc (modified in place).  Returns lost count."""
    w = (C.c_int32 * 4)(*wall)
    return load().or_move_all(mesh_ptr, parts["x"].size, d(parts["x"]), d(parts["y"]),
                              d(parts["vx"]), d(parts["vy"]), d(parts["vz"]), i32(parts["loc"]),
                              d(efx), d(efy), d(coef), qm, dt, w)


def move_all_axi(mesh_ptr, parts, efx, efy, coef, qm, dt, wall=(0, 0, 0, 0)):
    """Axisymmetric push: x = z, y = r, (vx, vy, vz) = (v_z, v_r, v_theta)
    in the particle's frame (modified in place).  Returns the lost count."""
    w = (C.c_int32 * 4)(*wall)
    return load().or_move_all_axi(mesh_ptr, parts["x"].size, d(parts["x"]), d(parts["y"]),
                                  d(parts["vx"]), d(parts["vy"]), d(parts["vz"]), i32(parts["loc"]),
                                  d(efx), d(efy), d(coef), qm, dt, w)


def deposit(mesh_ptr, parts, mass, vref, nn):
    q = np.zeros(nn, np.int64)
    e = np.zeros(nn, np.int64)
    bad = load().or_deposit(mesh_ptr, parts["x"].size, d(parts["x"]), d(parts["y"]),
                            d(parts["vx"]), d(parts["vy"]), d(parts["vz"]), i32(parts["loc"]),
                            mass, vref, i64(q), i64(e))
    return q, e, bad


def normalize(mesh_ptr, qs, es, wq, L_ref, n_ref, nn):
    ns = len(qs)
    rho = np.zeros(nn)
    rho_s = [np.zeros(nn) for _ in range(ns)]
    ek_s = [np.zeros(nn) for _ in range(ns)]
    qa = (_l * ns)(*[i64(a) for a in qs])
    ea = (_l * ns)(*[i64(a) for a in es])
    ra = (_d * ns)(*[d(a) for a in rho_s])
    ka = (_d * ns)(*[d(a) for a in ek_s])
    w = np.ascontiguousarray(wq, dtype=np.float64)
    load().or_normalize(mesh_ptr, ns, qa, ea, d(w), L_ref, n_ref, d(rho), ra, ka)
    return rho, rho_s, ek_s


def rhs(mesh_ptr, rho, nn):
    b = np.zeros(nn)
    load().or_rhs(mesh_ptr, d(np.ascontiguousarray(rho)), d(b))
    return b


def pcg(mesh_ptr, b, phi0, tol, maxit):
    phi = np.ascontiguousarray(phi0, dtype=np.float64).copy()
    st = np.zeros(4)
    load().or_pcg(mesh_ptr, d(np.ascontiguousarray(b)), d(phi), tol, maxit, d(st))
    return phi, {"iterations": int(st[0]), "ierr": int(st[1]), "normR": st[2], "normRHS": st[3]}


def ppr(mesh_ptr, phi, nn):
    coef = np.zeros(5 * nn)
    efx = np.zeros(nn)
    efy = np.zeros(nn)
    load().or_ppr(mesh_ptr, d(np.ascontiguousarray(phi)), d(coef), d(efx), d(efy))
    return coef.reshape(5, nn), efx, efy


def sort_perm(loc, ids):
    perm = np.zeros(loc.size, np.int64)
    m = load().or_sort_perm(loc.size, i32(loc), u32(ids), i64(perm))
    return perm[:m]


def canon_dot(a, b):
    return load().or_canon_dot(d(a), d(b), a.size)


def mcc(table, gas, mass, vref, seed, step, species, parts):
    n = parts["x"].size
    counts = np.zeros(8, np.int64)
    n_new = np.zeros(1, np.int64)
    cap = n + 16
    par = np.zeros(cap, np.int64)
    ne = np.zeros(3 * cap)
    ni = np.zeros(3 * cap)
    ncoll = load().or_mcc(C.byref(table), C.byref(gas), mass, vref, seed, step, species, n,
                          i32(parts["loc"]), u32(parts["id"]), d(parts["vx"]), d(parts["vy"]),
                          d(parts["vz"]), i64(counts), i64(n_new), i64(par), d(ne), d(ni))
    k = int(n_new[0])
    return ncoll, counts, par[:k], ne[:3 * k].reshape(k, 3), ni[:3 * k].reshape(k, 3)


def closed_form(typ, bi, pf, a, b, R):
    C4 = np.zeros(4)
    ok = load().or_ife_closed_form(typ, bi, pf, a, b, R, d(C4))
    return C4 if ok else None


def ek_tot(mesh_ptr, e_acc, weight, L_ref, n_ref, nn):
    out = np.zeros(nn)
    load().or_ek_tot(mesh_ptr, i64(e_acc), weight, L_ref, n_ref, d(out))
    return out


def average_x(f, nnx, nny, scale):
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros(nnx)
    load().or_average_x(nnx, nny, d(f), scale, d(out))
    return out


def energy_spectrum(parts, mass, vref, nbins, e_max, v_max):
    ce, cv = np.zeros(nbins, np.int64), np.zeros(nbins, np.int64)
    n = parts["vx"].size
    load().or_energy_spectrum(n, d(parts["vx"]), d(parts["vy"]), d(parts["vz"]), i32(parts["loc"]),
                              mass, vref, nbins, e_max, v_max, i64(ce), i64(cv))
    return ce, cv


def velocity_moments(parts, nbins):
    cnt = np.zeros(nbins, np.int64)
    drift, thermal = np.zeros((3, nbins)), np.zeros((3, nbins))
    n = parts["vx"].size
    load().or_velocity_moments(n, d(parts["x"]), d(parts["vx"]), d(parts["vy"]), d(parts["vz"]),
                               i32(parts["loc"]), nbins, i64(cnt), d(drift), d(thermal))
    return cnt, drift, thermal


OR_QUAD_AS_COMPILED, OR_QUAD_EXACT = 0, 1


class OracleMesh:
    """The oracle's own mesh descriptor (or_mesh_build), built from the same
    deck as the product's pic_mesh_build; same array() accessors as
    pic_b200.deck.Mesh."""

    def __init__(self, deck, quad=OR_QUAD_AS_COMPILED):
        lib = load()
        self.deck = deck
        self.ptr = C.POINTER(api.MeshDesc)()
        rc = lib.or_mesh_build(C.byref(deck), int(quad), C.byref(self.ptr))
        if rc != 0:
            raise RuntimeError(f"or_mesh_build failed ({rc})")
        self.desc = self.ptr.contents
        d = self.desc
        self.nnx, self.nny = d.nnx, d.nny
        self.nn = d.nnx * d.nny
        self.ne = (d.nnx - 1) * (d.nny - 1)
        self.hx = (d.xmax - d.xmin) / (d.nnx - 1)
        self.hy = (d.ymax - d.ymin) / (d.nny - 1)

    def array(self, name):
        d = self.desc
        sizes = {"node_type": self.nn, "node_index": self.nn, "element_index": self.ne,
                 "phi_dirichlet": self.nn, "cell_volume": self.nn,
                 "a_srow": d.n_unknowns + 1, "a_jcol": d.nnz, "a_k": d.nnz,
                 "xt_srow": d.n_unknowns + 1, "xt_jcol": d.nnz_xt, "xt_k": d.nnz_xt,
                 "a_diag": d.n_unknowns, "rhs_fix": d.n_unknowns, "mass_q1": 16,
                 "ife_mass": 16 * d.n_interface, "patch_ptr": self.nn + 1,
                 "mass_rows": 16 * (self.nny - 1)}
        n = int(self.array("patch_ptr")[-1]) if name == "patch_nodes" else sizes[name]
        ptr = getattr(d, name)
        dt = np.float64 if ptr._type_ is C.c_double else np.int32
        return api.as_np(ptr, int(n), dt).copy()

    def interface(self, k):
        el, ty = C.c_int32(), C.c_int32()
        r2l = np.zeros(4, np.int32)
        beta, D, E = np.zeros(2), np.zeros(2), np.zeros(2)
        load().or_mesh_interface(self.ptr, int(k), C.byref(el), C.byref(ty), i32(r2l), d(beta), d(D), d(E))
        return {"element": el.value, "type": ty.value, "r2l": r2l, "beta": beta, "D": D, "E": E}

    def close(self):
        if self.ptr:
            load().or_mesh_free(self.ptr)
            self.ptr = C.POINTER(api.MeshDesc)()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def quad_constants(quad):
    out = np.zeros(9 + 18 + 9 + 18 + 4 + 8 + 1)
    load().or_quad_constants(int(quad), d(out))
    return out


def mcc_table(bundle, mass, gas_mass, n_gas, dt_s, jtoev=1.6022e-19):
    """The oracle's collision table for one raw bundle ({"model", "reactions":
    [{"threshold", "table": [[E eV, sigma cm^2], ...]}]}): (sigma [nr][ns] in
    m^2, prob [ns][nr], SigmaMax, CollisionRatio, EnergyMax).  The grid is
    MCCSigma.f90:9-11's: 10001 points, log10 E over [-3, 3] (model 1) or
    [-1, 3] (model 2)."""
    lib = load()
    emin, emax = (-3.0, 3.0) if bundle["model"] == 1 else (-1.0, 3.0)
    ns = 10001
    eint = (emax - emin) / (ns - 1)
    nr = len(bundle["reactions"])
    sig = np.zeros((nr, ns))
    for j, r in enumerate(bundle["reactions"]):
        raw = np.ascontiguousarray(np.array(r["table"], dtype=np.float64))
        e, s = np.ascontiguousarray(raw[:, 0]), np.ascontiguousarray(raw[:, 1])
        row = np.zeros(ns)
        if lib.or_mcc_sigma(len(e), d(e), d(s), float(r["threshold"]), emin, eint, ns, d(row)) != 0:
            raise RuntimeError("or_mcc_sigma")
        sig[j] = row
    prob = np.zeros((ns, nr))
    o3 = np.zeros(3)
    lib.or_mcc_probability(nr, ns, d(np.ascontiguousarray(sig)), mass, gas_mass, n_gas, emin, eint, emax,
                           dt_s, jtoev, d(prob), d(o3))
    return sig, prob, o3[0], o3[1], o3[2]


def mcc_select_keys(seed, step, species, ids):
    """The oracle's null-collision selection keys of `ids` at one step."""
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    out = np.empty_like(ids)
    load().or_mcc_select_keys(seed, step, species, ids.size, u32(ids), u32(out))
    return out
