"""Host-side mirror of the reference's explicit main loop
(code/PIC/Main_IFE_Test_2.f90:74-341) driving libpicgpu through its C-ABI.

    init:  Input_2D -> Setup_IFE_Mesh_2D/IFE_Start_2D/Get_PointPatch
           (pic_mesh_build) -> particle bundles (load_particles) -> MCC tables
           -> GetParChg_2D -> IFE_Solve_2D -> GetEField_SIDG_PPR   (Main:215-263)
    step:  MoveAll -> GetParChg_2D -> IFE_Solve_2D -> GetEField_SIDG_PPR
           (Main:329-341), MCC after the field solve (MCC_jw OneStep.F90:50-67)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api
from .deck import Config, Mesh, load_particles, species_params
from .mcc_tables import ar_tables


class Simulation:
    def __init__(self, cfg: Config, capacity_factor: float = 1.5, load: bool = True,
                 mcc: bool | None = None, capacity: list | None = None):
        """load: generate and upload the deck's initial particles.  capacity:
        particle slots per species (default: 1.5 x the initial count)."""
        self.lib = api.load()
        self.cfg = cfg
        self.mesh = Mesh(cfg)
        sp, _ = species_params(cfg)
        self.species = sp
        self.particles0 = []
        if load:
            for s in range(2):
                self.particles0.append(load_particles(cfg, self.mesh, s))
        p = api.Params()
        p.n_species = 2
        for s, (q, m, w, _) in enumerate(sp):
            n0 = self.particles0[s][0].size if load else 0
            p.species[s].charge = q
            p.species[s].mass = m
            p.species[s].weight = w
            p.species[s].capacity = max(int(n0 * capacity_factor) + 1024, 1024)
            if capacity is not None:
                p.species[s].capacity = int(capacity[s])
        p.dt = cfg.dt
        p.n_ref = cfg.n0
        p.T_ref_eV = cfg.Te_eV
        p.pcg_tol = cfg.pcg_tol
        p.pcg_maxit = cfg.pcg_maxit
        for k in range(4):
            p.wall_bc[k] = int(cfg.wall_particles[k])
        p.seed = cfg.seed
        p.precision = cfg.precision
        p.sort_interval = cfg.sort_interval
        p.diag_interval = cfg.diag_interval
        p.solver = api.PIC_SOLVER_JPCG
        self.params = p
        api.check(self.lib.pic_init(self.mesh.ptr, C.byref(p)), "pic_init")
        self.scales = cfg.scales
        if cfg.rf is not None:
            self.set_wall_rf(*cfg.rf)
        use_mcc = cfg.mcc if mcc is None else mcc
        if use_mcc:
            dt_s = cfg.dt * self.scales["time_ref"]
            gas, tabs, self._keep = ar_tables(cfg, dt_s)
            arr = (api.MccTable * len(tabs))(*tabs)
            api.check(self.lib.pic_mcc_init(C.byref(gas), len(tabs), arr), "pic_mcc_init")
            self.mcc_tables = tabs
            self.gas = gas
        for s, parts in enumerate(self.particles0):
            self.upload(s, *parts)
        self.step_index = 0

    # ---- particle I/O -------------------------------------------------
    def upload(self, s, x, y, vx, vy, vz, loc=None, ids=None):
        n = x.size
        api.check(self.lib.pic_upload_particles(s, n, api.dptr(x), api.dptr(y), api.dptr(vx),
                                                api.dptr(vy), api.dptr(vz), api.iptr(loc),
                                                api.uptr(ids)), "pic_upload_particles")

    def count(self, s) -> int:
        n = C.c_int64()
        api.check(self.lib.pic_particle_count(s, C.byref(n)), "pic_particle_count")
        return n.value

    def download(self, s):
        n = self.count(s)
        cap = max(n, 1)
        out = [np.empty(cap) for _ in range(5)] + [np.empty(cap, np.int32), np.empty(cap, np.uint32)]
        got = C.c_int64()
        api.check(self.lib.pic_download_particles(s, cap, *[api.dptr(a) for a in out[:5]],
                                                  api.iptr(out[5]), api.uptr(out[6]),
                                                  C.byref(got)), "pic_download_particles")
        k = got.value
        names = ("x", "y", "vx", "vy", "vz", "loc", "id")
        return {nm: a[:k].copy() for nm, a in zip(names, out)}

    # ---- the reference's subroutines ------------------------------------
    def particle_positioning(self, s=-1):
        api.check(self.lib.pic_particle_positioning(s), "pic_particle_positioning")

    def move_all(self, s):
        api.check(self.lib.pic_move_all(s, 0), "pic_move_all")

    def get_par_chg(self, rho_out: np.ndarray | None = None):
        api.check(self.lib.pic_get_par_chg(self.cfg.delta, api.dptr(rho_out)), "pic_get_par_chg")

    def ife_solve(self, phi: np.ndarray | None = None, time: float = 0.0) -> api.SolveStats:
        """IFE_Solve_2D at normalised time `time` (it drives a wall RF potential)."""
        st = api.SolveStats()
        api.check(self.lib.pic_ife_solve(api.dptr(phi), float(time), C.byref(st)), "pic_ife_solve")
        return st

    def set_wall_rf(self, wall: int, volts: float, frequency_hz: float, phase: float = 0.0):
        """Potential volts * sin(2 pi f t + phase) added to the Dirichlet wall
        x = xmin (0) or x = xmax (1); volts = 0 switches it off."""
        api.check(self.lib.pic_set_wall_rf(int(wall), volts / self.scales["Phi_ref"], float(frequency_hz),
                                           float(phase)), "pic_set_wall_rf")

    def get_efield_ppr(self, efx=None, efy=None):
        api.check(self.lib.pic_get_efield_ppr(api.dptr(efx), api.dptr(efy)), "pic_get_efield_ppr")

    def mcc(self, step) -> api.MccStats:
        st = api.MccStats()
        api.check(self.lib.pic_mcc(step, C.byref(st)), "pic_mcc")
        return st

    def sort(self, s):
        api.check(self.lib.pic_sort_particles(s), "pic_sort_particles")

    def initial_fields(self) -> api.SolveStats:
        """Main_IFE_Test_2.f90:215-263: charge, potential and field before the loop."""
        self.get_par_chg()
        st = self.ife_solve()
        self.get_efield_ppr()
        return st

    def step(self) -> api.StepStats:
        st = api.StepStats()
        self.step_index += 1
        api.check(self.lib.pic_step(self.step_index, C.byref(st)), "pic_step")
        return st

    # ---- Poisson solver ---------------------------------------------------
    def set_solver(self, kind: str = "jpcg", coarse_cells: int = 64, window: int = 1,
                   omega: float = 2.0 / 3.0, inner_fp32: bool = False,
                   multigrid: bool = False, max_coarse_nodes: int = 4500):
        """'jpcg': the reference's Jacobi-PCG.  'fcg': flexible CG with damped
        Jacobi smoothing and a Galerkin coarse space (no learned stage): the
        two-level space of about coarse_cells^2 cells, or with multigrid the
        V-cycle down to max_coarse_nodes; inner_fp32 (mixed precision only):
        FP32 iterations in FP64 refinement.  'fcg-learned' is set up by
        unet.LearnedPreconditioner on top of 'fcg'."""
        lib = self.lib
        if kind == "jpcg":
            api.check(lib.pic_set_solver(api.PIC_SOLVER_JPCG), "pic_set_solver")
            return
        if kind != "fcg":
            raise ValueError(kind)
        api.check(lib.pic_set_precond_stages(1, omega, 0), "pic_set_precond_stages")
        if multigrid:
            api.check(lib.pic_multigrid_setup(self.mesh.ptr, max_coarse_nodes), "pic_multigrid_setup")
        else:
            api.check(lib.pic_coarse_setup(self.mesh.ptr, coarse_cells), "pic_coarse_setup")
        api.check(lib.pic_set_fcg_window(window), "pic_set_fcg_window")
        api.check(lib.pic_set_fcg_inner(int(inner_fp32)), "pic_set_fcg_inner")
        api.check(lib.pic_set_solver(api.PIC_SOLVER_FCG_UNET), "pic_set_solver")

    # ---- fields ---------------------------------------------------------
    FIELDS = {"rho": 0, "phi": 1, "efx": 2, "efy": 3, "rho_e": 4, "rho_i": 5, "ek_e": 8,
              "ek_i": 9, "c2": 12, "c3": 13, "c4": 14, "c5": 15, "c6": 16, "b": 20,
              "ektot_e": 24, "ektot_i": 25}

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.mesh.nn)
        api.check(self.lib.pic_get_field(self.FIELDS[name], api.dptr(out)), "pic_get_field")
        return out

    def set_field(self, name: str, values: np.ndarray):
        v = np.ascontiguousarray(values, dtype=np.float64)
        api.check(self.lib.pic_set_field(self.FIELDS[name], api.dptr(v)), "pic_set_field")

    # ---- diagnostics, computed on the device ------------------------------
    SPECIES_TAGS = ("ele", "ion", "s2", "s3")

    def average_x(self) -> dict:
        """Average_x column profiles (Output_To_Tecplot_IJK_2D.f90:166-226) in
        the file's units: x [m], Phi [V], Rho, Rho_<sp> [m^-3], Ek_<sp> [eV],
        Ek_tot_<sp>."""
        ns, nnx = len(self.species), self.mesh.nnx
        out = np.empty((3 + 3 * ns) * nnx)
        api.check(self.lib.pic_average_x(api.dptr(out)), "pic_average_x")
        out = out.reshape(3 + 3 * ns, nnx)
        tags = self.SPECIES_TAGS[:ns]
        names = (["x", "Phi", "Rho"] + ["Rho_" + t for t in tags] + ["Ek_" + t for t in tags]
                 + ["Ek_tot_" + t for t in tags])
        return dict(zip(names, out))

    def energy_spectrum(self, s: int, nbins: int = 100, e_max: float = 5.0,
                        v_max: float | None = None):
        """Output_Energy.f90:41-71 counts of species s: (energy counts, vx
        counts), defaults N = 100, Ek_max = 5 eV, Vk_max = 10, 0.1, 0.01."""
        if v_max is None:
            v_max = (10.0, 0.1, 0.01, 0.01)[s]
        ce, cv = np.zeros(nbins, np.int64), np.zeros(nbins, np.int64)
        api.check(self.lib.pic_energy_spectrum(s, nbins, e_max, v_max, api.lptr(ce), api.lptr(cv)),
                  "pic_energy_spectrum")
        return ce, cv

    def velocity_moments(self, s: int, nbins: int = 1024):
        """OUTPUT_velocity.f90:48-103 of species s: per x column the count,
        drift velocity [3, nbins] and thermal velocity [3, nbins]."""
        cnt = np.zeros(nbins, np.int64)
        drift, thermal = np.zeros((3, nbins)), np.zeros((3, nbins))
        api.check(self.lib.pic_velocity_moments(s, nbins, api.lptr(cnt), api.dptr(drift),
                                                api.dptr(thermal)), "pic_velocity_moments")
        return cnt, drift, thermal

    def particle_totals(self):
        """Main_IFE_Test_2.f90:473-497 (equal weights): real particles per
        species, Npar * Weight, and their sum."""
        ns = [self.count(s) * self.species[s][2] for s in range(len(self.species))]
        return sum(ns), ns

    def close(self):
        self.lib.pic_finalize()
        self.mesh.close()
