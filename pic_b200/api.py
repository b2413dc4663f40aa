"""ctypes binding of libpicgpu.so (include/picgpu.h).

The structures mirror the C declarations field by field.  Loading fails
loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpicgpu.so")

PIC_MAX_SPECIES = 4
PIC_MAX_OBJECTS = 32
PIC_MAX_REACTIONS = 8

PIC_SHAPE_CIRCLE, PIC_SHAPE_BOX, PIC_SHAPE_ELLIPSE = 1, 3, 5
PIC_WALL_ABSORB, PIC_WALL_REFLECT = 0, 1
PIC_PREC_FP64, PIC_PREC_MIXED = 0, 1
PIC_SOLVER_JPCG, PIC_SOLVER_FCG_UNET = 0, 1
PIC_ERR_ARG, PIC_ERR_STATE = -1, -6

ERRORS = {
    -1: "PIC_ERR_ARG", -2: "PIC_ERR_CUDA", -3: "PIC_ERR_SOLVER_CAP", -4: "PIC_ERR_NAN",
    -5: "PIC_ERR_DOMAIN", -6: "PIC_ERR_STATE", -7: "PIC_ERR_CAPACITY", -8: "PIC_ERR_SETUP",
    -9: "PIC_ERR_BREAKDOWN",
}

# every entry point declared in include/picgpu.h
EXPORTS = [
    "pic_mesh_build", "pic_mesh_build_device", "pic_mesh_free", "pic_mesh_interface_info", "pic_mesh_ife_basis",
    "pic_init", "pic_finalize", "pic_last_error", "pic_mcc_init", "pic_upload_particles",
    "pic_download_particles", "pic_particle_count", "pic_particle_positioning",
    "pic_sort_particles", "pic_move_all", "pic_get_par_chg", "pic_ife_solve",
    "pic_get_efield_ppr", "pic_mcc", "pic_step", "pic_get_field", "pic_set_field",
    "pic_particle_device_ptrs", "pic_kernel_launches", "pic_device_timer",
    "pic_deposit_noalloc", "pic_set_preconditioner", "pic_set_solver", "pic_set_fcg_window",
    "pic_cuda_stream", "pic_apply_operator", "pic_solver_vectors", "pic_set_precond_stages",
    "pic_coarse_setup", "pic_precond_apply", "pic_set_fcg_inner", "pic_average_x",
    "pic_energy_spectrum", "pic_velocity_moments", "pic_multigrid_setup", "pic_get_next_id",
    "pic_set_next_id", "pic_set_wall_rf", "pic_get_fields_async", "pic_wait_fields",
    "pic_set_field_async",
]

# z = M(r) callback of flexible CG: (r_dev, z_dev, user) -> 0 or failure
PRECOND_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)


class PicError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({code}): {detail}")
        self.code = code


class Object(C.Structure):
    _fields_ = [("shape", C.c_int32), ("conductor", C.c_int32), ("cx", C.c_double),
                ("cy", C.c_double), ("a", C.c_double), ("b", C.c_double),
                ("angle", C.c_double), ("eps", C.c_double), ("phi", C.c_double)]


class Deck(C.Structure):
    _fields_ = [("nnx", C.c_int32), ("nny", C.c_int32), ("xmin", C.c_double),
                ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
                ("delta", C.c_int32), ("wall_dirichlet", C.c_int32 * 4),
                ("wall_phi", C.c_double * 4), ("n_objects", C.c_int32),
                ("objects", Object * PIC_MAX_OBJECTS)]


_P = C.POINTER


class MeshDesc(C.Structure):
    _fields_ = [("nnx", C.c_int32), ("nny", C.c_int32), ("xmin", C.c_double),
                ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
                ("delta", C.c_int32),
                ("node_type", _P(C.c_int32)), ("node_index", _P(C.c_int32)),
                ("element_index", _P(C.c_int32)), ("phi_dirichlet", _P(C.c_double)),
                ("cell_volume", _P(C.c_double)), ("n_unknowns", C.c_int32),
                ("nnz", C.c_int64), ("a_srow", _P(C.c_int32)), ("a_jcol", _P(C.c_int32)),
                ("a_k", _P(C.c_double)), ("nnz_xt", C.c_int64), ("xt_srow", _P(C.c_int32)),
                ("xt_jcol", _P(C.c_int32)), ("xt_k", _P(C.c_double)),
                ("a_diag", _P(C.c_double)), ("rhs_fix", _P(C.c_double)),
                ("mass_q1", _P(C.c_double)), ("n_interface", C.c_int32),
                ("ife_mass", _P(C.c_double)), ("patch_ptr", _P(C.c_int32)),
                ("patch_nodes", _P(C.c_int32)), ("n_objects", C.c_int32),
                ("objects", _P(Object)), ("mass_rows", _P(C.c_double))]


class SpeciesDesc(C.Structure):
    _fields_ = [("charge", C.c_double), ("mass", C.c_double), ("weight", C.c_double),
                ("capacity", C.c_int64)]


class Params(C.Structure):
    _fields_ = [("n_species", C.c_int32), ("species", SpeciesDesc * PIC_MAX_SPECIES),
                ("dt", C.c_double), ("n_ref", C.c_double), ("T_ref_eV", C.c_double),
                ("pcg_tol", C.c_double), ("pcg_maxit", C.c_int32), ("wall_bc", C.c_int32 * 4),
                ("seed", C.c_uint64), ("precision", C.c_int32), ("sort_interval", C.c_int32),
                ("solver", C.c_int32), ("diag_interval", C.c_int32)]


class MccTable(C.Structure):
    _fields_ = [("species", C.c_int32), ("n_reaction", C.c_int32), ("n_sigma", C.c_int32),
                ("energy_min", C.c_double), ("energy_interval", C.c_double),
                ("energy_max", C.c_double), ("collision_ratio", C.c_double),
                ("reaction_type", C.c_int32 * PIC_MAX_REACTIONS),
                ("threshold", C.c_double * PIC_MAX_REACTIONS),
                ("resultant", C.c_int32 * PIC_MAX_REACTIONS),
                ("probability", _P(C.c_double))]


class Gas(C.Structure):
    _fields_ = [("mass", C.c_double), ("temperature", C.c_double), ("density", C.c_double)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("ierr", C.c_int32), ("rel_residual", C.c_double),
                ("ms", C.c_double), ("fallback", C.c_int32), ("outer", C.c_int32)]


class MccStats(C.Structure):
    _fields_ = [("n_selected", C.c_int64 * PIC_MAX_SPECIES),
                ("n_by_reaction", (C.c_int64 * PIC_MAX_REACTIONS) * PIC_MAX_SPECIES),
                ("n_created", C.c_int64 * PIC_MAX_SPECIES)]


class StepStats(C.Structure):
    _fields_ = [("n_particles", C.c_int64 * PIC_MAX_SPECIES),
                ("n_lost", C.c_int64 * PIC_MAX_SPECIES), ("solve", SolveStats),
                ("mcc", MccStats), ("ms_push", C.c_double), ("ms_solve", C.c_double),
                ("ms_ppr", C.c_double), ("ms_mcc", C.c_double), ("ms_sort", C.c_double),
                ("ms_total", C.c_double), ("ms_push_kernel", C.c_double),
                ("pushed", C.c_int64)]


_lib = None


def load() -> C.CDLL:
    """Load libpicgpu.so from the package directory (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libpicgpu.so not built at {LIB_PATH}: run pic_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    lib.pic_last_error.restype = C.c_char_p
    lib.pic_kernel_launches.restype = C.c_int64
    lib.pic_mesh_build.argtypes = [_P(Deck), _P(_P(MeshDesc))]
    lib.pic_mesh_build_device.argtypes = [_P(Deck), _P(_P(MeshDesc))]
    lib.pic_mesh_free.argtypes = [_P(MeshDesc)]
    lib.pic_mesh_free.restype = None
    lib.pic_mesh_interface_info.argtypes = [_P(MeshDesc), C.c_int32, _P(C.c_int32),
                                            _P(C.c_int32), _P(C.c_int32), _P(C.c_double),
                                            _P(C.c_double), _P(C.c_double)]
    lib.pic_mesh_ife_basis.argtypes = [_P(MeshDesc), C.c_int32, C.c_int32, C.c_double,
                                       C.c_double, _P(C.c_double), _P(C.c_double),
                                       _P(C.c_double)]
    lib.pic_init.argtypes = [_P(MeshDesc), _P(Params)]
    lib.pic_finalize.restype = None
    lib.pic_mcc_init.argtypes = [_P(Gas), C.c_int32, _P(MccTable)]
    d = _P(C.c_double)
    lib.pic_upload_particles.argtypes = [C.c_int32, C.c_int64, d, d, d, d, d, _P(C.c_int32),
                                         _P(C.c_uint32)]
    lib.pic_download_particles.argtypes = [C.c_int32, C.c_int64, d, d, d, d, d,
                                           _P(C.c_int32), _P(C.c_uint32), _P(C.c_int64)]
    lib.pic_particle_count.argtypes = [C.c_int32, _P(C.c_int64)]
    lib.pic_particle_positioning.argtypes = [C.c_int32]
    lib.pic_sort_particles.argtypes = [C.c_int32]
    lib.pic_move_all.argtypes = [C.c_int32, C.c_int32]
    lib.pic_get_par_chg.argtypes = [C.c_int32, d]
    lib.pic_ife_solve.argtypes = [d, C.c_double, _P(SolveStats)]
    lib.pic_get_efield_ppr.argtypes = [d, d]
    lib.pic_mcc.argtypes = [C.c_uint64, _P(MccStats)]
    lib.pic_step.argtypes = [C.c_uint64, _P(StepStats)]
    lib.pic_get_field.argtypes = [C.c_int32, d]
    lib.pic_set_field.argtypes = [C.c_int32, d]
    lib.pic_get_fields_async.argtypes = [d, d, d, d]
    lib.pic_wait_fields.argtypes = []
    lib.pic_set_field_async.argtypes = [C.c_int32, d]
    lib.pic_device_timer.argtypes = [C.c_int32, _P(C.c_double)]
    lib.pic_set_preconditioner.argtypes = [PRECOND_FN, C.c_void_p]
    lib.pic_set_solver.argtypes = [C.c_int32]
    lib.pic_set_fcg_window.argtypes = [C.c_int32]
    lib.pic_set_fcg_inner.argtypes = [C.c_int32]
    lib.pic_cuda_stream.argtypes = [_P(C.c_void_p)]
    lib.pic_apply_operator.argtypes = [C.c_void_p, C.c_void_p]
    lib.pic_solver_vectors.argtypes = [_P(C.c_void_p), _P(C.c_void_p)]
    lib.pic_set_precond_stages.argtypes = [C.c_int32, C.c_double, C.c_int32]
    lib.pic_coarse_setup.argtypes = [_P(MeshDesc), C.c_int32]
    lib.pic_multigrid_setup.argtypes = [_P(MeshDesc), C.c_int32]
    lib.pic_get_next_id.argtypes = [C.c_int32, _P(C.c_uint32)]
    lib.pic_set_next_id.argtypes = [C.c_int32, C.c_uint32]
    lib.pic_set_wall_rf.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double]
    lib.pic_precond_apply.argtypes = [C.c_int32, C.c_void_p, C.c_void_p]
    lib.pic_deposit_noalloc.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                                        C.c_void_p]
    lib.pic_particle_device_ptrs.argtypes = [C.c_int32, _P(C.c_void_p), _P(C.c_int64)]
    lib.pic_average_x.argtypes = [d]
    lib.pic_energy_spectrum.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double,
                                        _P(C.c_int64), _P(C.c_int64)]
    lib.pic_velocity_moments.argtypes = [C.c_int32, C.c_int32, _P(C.c_int64), d, d]
    _lib = lib
    return lib


def check(rc: int, where: str) -> int:
    if rc != 0:
        raise PicError(rc, where, load().pic_last_error().decode(errors="replace"))
    return rc


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_P(C.c_double))


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_P(C.c_int32))


def uptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_P(C.c_uint32))


def lptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(_P(C.c_int64))


def as_np(ptr, n: int, dtype) -> np.ndarray:
    """Copy n elements behind a ctypes pointer into a new numpy array."""
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)
