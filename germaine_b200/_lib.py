"""ctypes binding of libgermaine_gpu.so (the C-ABI in include/germaine_gpu.h).

The library is built in-tree by germaine_b200/build.py.  There is no CPU
fallback: if the shared library is missing or a call fails, an exception is
raised.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgermaine_gpu.so")
UMFPACK_LIB_PATH = os.path.join(HERE, "libgermaine_umfpack.so")

GM_OK = 0
GM_WARNING_PERTURBED = 1
GM_WARNING_NOT_CONVERGED = 2
GM_ERROR_OUT_OF_MEMORY = -1
GM_ERROR_INVALID = -2
GM_SEIS_KEEP_LAST = 1
GM_HESS_GREEN = 1
GM_HESS_SHIN = 2
GM_ERROR_STATE = -3
GM_ERROR_CUDA = -4
GM_ERROR_NONFINITE = -5
GM_ERROR_PATTERN = -6

GM_PHYS_AC, GM_PHYS_SH, GM_PHYS_TE = 1, 2, 4
GM_PREC_FP64, GM_PREC_C64_IR = 0, 1
GM_OP_REF, GM_OP_EXACT = 0, 1
GM_SYS_A, GM_SYS_AT = 0, 1
GM_REFINE_MODE_AUTO, GM_REFINE_MODE_IR, GM_REFINE_MODE_GMRES = 0, 1, 2


class GmConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("dh", ctypes.c_float),
                ("npml", ctypes.c_int32), ("free_surf", ctypes.c_int32), ("a0_pml", ctypes.c_float),
                ("s", ctypes.c_float), ("physics", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("op_mode", ctypes.c_int32), ("leaf_max", ctypes.c_int32), ("ir_tol", ctypes.c_double),
                ("ir_max_iter", ctypes.c_int32), ("refine", ctypes.c_int32), ("gmres_restart", ctypes.c_int32),
                ("tc_min_block", ctypes.c_int32), ("pivot_tol", ctypes.c_double)]


class GmStats(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("nonzero", ctypes.c_int64), ("nnodes", ctypes.c_int32),
                ("nlevels", ctypes.c_int32), ("max_front", ctypes.c_int32), ("max_piv", ctypes.c_int32),
                ("front_entries", ctypes.c_int64), ("factor_entries", ctypes.c_int64),
                ("factor_flops", ctypes.c_double), ("solve_flops_per_rhs", ctypes.c_double),
                ("perturbed_pivots", ctypes.c_int64), ("ir_iterations", ctypes.c_int32),
                ("ir_residual", ctypes.c_double), ("ms_assemble", ctypes.c_double),
                ("ms_factor", ctypes.c_double), ("ms_solve", ctypes.c_double), ("ms_refine", ctypes.c_double),
                ("ms_subst", ctypes.c_double), ("n_subst", ctypes.c_int32), ("kernel_launches", ctypes.c_int64),
                ("u_entries", ctypes.c_int64), ("ms_subst_bwd", ctypes.c_double), ("tc_tiles", ctypes.c_int64),
                ("pivot_swaps", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GmRefineInfo(ctypes.Structure):
    _fields_ = [("first_residual", ctypes.c_double), ("final_residual", ctypes.c_double),
                ("sweeps", ctypes.c_int32), ("method", ctypes.c_int32)]


GM_REFINE_NONE, GM_REFINE_IR, GM_REFINE_GMRES = 0, 1, 2
REFINE_METHOD_NAMES = {GM_REFINE_NONE: "none", GM_REFINE_IR: "ir", GM_REFINE_GMRES: "gmres"}


# every C-ABI symbol declared in include/germaine_gpu.h
EXPORTS = [
    "gm_last_error", "gm_version", "gm_engine_create", "gm_engine_destroy", "gm_engine_stats", "gm_engine_stream",
    "gm_refine_report", "gm_autotune", "gm_autotune_table", "gm_set_model", "gm_set_models", "gm_factor", "gm_factor_models", "gm_factor_values", "gm_get_triplets", "gm_solve", "gm_forward", "gm_grad_obj", "gm_obj",
    "gm_get_gradient_fp64", "gm_get_wavefield_fp64", "gm_get_misfit_fp64", "gm_obj_each", "gm_gauss_filt", "gm_solve_noalloc", "gm_hessian", "gm_get_hessian_fp64", "gm_apply_hess", "gm_precond",
    "gm_lbfgs_create", "gm_lbfgs_destroy", "gm_lbfgs_step", "gm_lbfgs_rotate", "gm_lbfgs_zero",
    "gm_lbfgs_check_descent", "gm_lbfgs_get_old", "gm_lbfgs_set_old", "gm_mat_change",
    "gm_set_shot_taper", "gm_set_shot_block", "gm_set_refine", "gm_memory_estimate", "gm_set_invmat", "gm_set_source_wavelet", "gm_stf_dft", "gm_taper_grad_shot", "gm_taper_grad_shot1", "gm_tikhonov_cost_te", "gm_tikhonov_grad_te",
    "gm_write_seis", "gm_read_seis", "gm_write_model_true", "gm_write_model", "gm_read_model", "gm_read_grid", "gm_cgemm_sub_c64", "gm_wait_probe", "gm_peak_fp64", "gm_peak_fp64_mma",
    "gm_symbolic_create", "gm_symbolic_destroy", "gm_symbolic_sizes", "gm_symbolic_export",
    "gm_symbolic_flops",
]

# every symbol declared in include/germaine_umfpack.h (libgermaine_umfpack.so)
UMFPACK_EXPORTS = [
    "umfpack_zi_triplet_to_col", "umfpack_zi_symbolic", "umfpack_zi_numeric", "umfpack_zi_solve",
    "umfpack_zi_free_symbolic", "umfpack_zi_free_numeric", "gm_umfpack_last_error",
]
UMFPACK_A, UMFPACK_At, UMFPACK_Aat = 0, 1, 2
UMFPACK_OK, UMFPACK_WARNING_singular_matrix = 0, 1
UMFPACK_ERROR_invalid_matrix, UMFPACK_ERROR_different_pattern, UMFPACK_ERROR_invalid_system = -8, -11, -13

_lib = None


class GmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"germaine_gpu error {code}: {msg}")
        self.code = code


def load() -> ctypes.CDLL:
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python germaine_b200/build.py` "
                           "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    i32, f64 = ctypes.c_int, ctypes.c_double
    lib.gm_last_error.restype = ctypes.c_char_p
    lib.gm_version.restype = i32
    lib.gm_engine_create.argtypes = [i32, ctypes.POINTER(GmConfig), ctypes.POINTER(vp)]
    lib.gm_engine_destroy.argtypes = [vp]
    lib.gm_engine_stats.argtypes = [vp, ctypes.POINTER(GmStats)]
    lib.gm_engine_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.gm_set_model.argtypes = [vp, vp, vp]
    lib.gm_factor.argtypes = [vp, i32, vp]
    lib.gm_set_models.argtypes = [vp, i32, vp, vp]
    lib.gm_factor_models.argtypes = [vp, i32, vp, vp]
    lib.gm_obj_each.argtypes = [vp, i32, vp, vp, i32, vp, vp, vp, i32, i32, vp]
    lib.gm_factor_values.argtypes = [vp, i32, vp, vp]
    lib.gm_get_triplets.argtypes = [vp, i32, vp, vp, vp, vp]
    lib.gm_solve.argtypes = [vp, i32, i32, vp, vp]
    lib.gm_refine_report.argtypes = [vp, i32, ctypes.POINTER(GmRefineInfo)]
    lib.gm_autotune.argtypes = [vp, i32, i32]
    lib.gm_autotune_table.argtypes = [vp, ctypes.POINTER(i32), vp, i32]
    lib.gm_forward.argtypes = [vp, i32, vp, vp, i32, vp, vp, vp, vp]
    lib.gm_grad_obj.argtypes = [vp, i32, vp, vp, i32, vp, vp, vp, i32, i32, vp, vp, vp, vp]
    lib.gm_obj.argtypes = [vp, i32, vp, vp, i32, vp, vp, vp, i32, i32, vp]
    lib.gm_get_gradient_fp64.argtypes = [vp, vp, vp]
    lib.gm_get_wavefield_fp64.argtypes = [vp, i32, vp]
    lib.gm_get_misfit_fp64.argtypes = [vp, i32, vp, vp]
    f32 = ctypes.c_float
    lib.gm_gauss_filt.argtypes = [i32, i32, i32, f32, f32, f32, f32, f32, vp, vp]
    lib.gm_hessian.argtypes = [vp, i32, i32, vp, vp, i32, vp, vp, vp, vp]
    lib.gm_get_hessian_fp64.argtypes = [vp, vp, vp]
    lib.gm_apply_hess.argtypes = [i32, i32, f32, vp, vp, vp]
    lib.gm_precond.argtypes = [i32, i32, i32, i32, i32, f32, i32, f32, f32, f32, f32, i32, i32, vp, vp]
    lib.gm_lbfgs_create.argtypes = [i32, i32, i32, i32, i32, i32, i32, ctypes.POINTER(vp)]
    lib.gm_lbfgs_destroy.argtypes = [vp]
    lib.gm_lbfgs_step.argtypes = [vp, i32, i32, vp, vp, vp, vp, f32, vp]
    lib.gm_lbfgs_rotate.argtypes = [vp]
    lib.gm_lbfgs_zero.argtypes = [vp]
    lib.gm_lbfgs_check_descent.argtypes = [vp, vp, vp, vp]
    lib.gm_lbfgs_get_old.argtypes = [vp, vp, vp]
    lib.gm_lbfgs_set_old.argtypes = [vp, vp, vp]
    lib.gm_mat_change.argtypes = [i32, i32, i32, f32, f32, f32, vp, vp, vp]
    lib.gm_set_shot_taper.argtypes = [vp, i32, f32, i32]
    lib.gm_set_invmat.argtypes = [vp, i32]
    lib.gm_set_shot_block.argtypes = [vp, i32]
    lib.gm_set_refine.argtypes = [vp, i32, i32]
    lib.gm_memory_estimate.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    lib.gm_set_source_wavelet.argtypes = [vp, i32, vp]
    lib.gm_stf_dft.argtypes = [ctypes.c_char_p, i32, f32, vp]
    lib.gm_taper_grad_shot.argtypes = [i32, i32, f32, f32, i32, vp, vp, i32, vp, vp, i32, vp]
    lib.gm_taper_grad_shot1.argtypes = [i32, i32, f32, i32, i32, vp, vp, i32, vp, vp, vp]
    lib.gm_tikhonov_cost_te.argtypes = [i32, i32, i32, i32, f32, f32, f32, f32, f32, f32, f32, vp, vp, f32, vp]
    lib.gm_tikhonov_grad_te.argtypes = [i32, i32, i32, i32, f32, f32, f32, f32, f32, f32, f32, vp, vp, vp, vp]
    cp = ctypes.c_char_p
    lib.gm_write_seis.argtypes = [cp, i32, i32, i32, i32, vp]
    lib.gm_read_seis.argtypes = [cp, i32, i32, i32, vp]
    lib.gm_write_model_true.argtypes = [cp, i32, i32, i32, i32, i32, i32, vp]
    lib.gm_write_model.argtypes = [cp, i32, i32, i32, i32, vp]
    lib.gm_read_model.argtypes = [cp, i32, i32, i32, i32, vp]
    lib.gm_read_grid.argtypes = [cp, i32, i32, vp]
    lib.gm_solve_noalloc.argtypes = [vp, i32, i32, vp, vp]
    lib.gm_cgemm_sub_c64.argtypes = [i32, i32, i32, vp, vp, vp, vp]
    lib.gm_wait_probe.argtypes = [i32, ctypes.c_longlong, ctypes.POINTER(i32)]
    lib.gm_peak_fp64.argtypes = [i32, ctypes.POINTER(f64)]
    lib.gm_peak_fp64_mma.argtypes = [i32, ctypes.POINTER(f64)]
    lib.gm_symbolic_create.argtypes = [i32, i32, i32, ctypes.POINTER(vp)]
    lib.gm_symbolic_destroy.argtypes = [vp]
    lib.gm_symbolic_sizes.argtypes = [vp, vp]
    lib.gm_symbolic_export.argtypes = [vp, i32, vp]
    lib.gm_symbolic_flops.argtypes = [vp, i32]
    lib.gm_symbolic_flops.restype = f64
    _lib = lib
    return lib


_umf = None


def load_umfpack() -> ctypes.CDLL:
    """Load the in-tree UMFPACK-API shim (raises if it was not built)."""
    global _umf
    if _umf is not None:
        return _umf
    load()
    if not os.path.exists(UMFPACK_LIB_PATH):
        raise RuntimeError(f"{UMFPACK_LIB_PATH} is missing: build it with `python germaine_b200/build.py`")
    lib = ctypes.CDLL(UMFPACK_LIB_PATH)
    vp, i32 = ctypes.c_void_p, ctypes.c_int
    lib.umfpack_zi_triplet_to_col.argtypes = [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.umfpack_zi_symbolic.argtypes = [i32, i32, vp, vp, vp, vp, ctypes.POINTER(vp), vp, vp]
    lib.umfpack_zi_numeric.argtypes = [vp, vp, vp, vp, vp, ctypes.POINTER(vp), vp, vp]
    lib.umfpack_zi_solve.argtypes = [i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.umfpack_zi_free_symbolic.argtypes = [ctypes.POINTER(vp)]
    lib.umfpack_zi_free_symbolic.restype = None
    lib.umfpack_zi_free_numeric.argtypes = [ctypes.POINTER(vp)]
    lib.umfpack_zi_free_numeric.restype = None
    lib.gm_umfpack_last_error.restype = ctypes.c_char_p
    _umf = lib
    return lib


def check(rc: int, allow_warning: bool = True) -> int:
    """Raise GmError for negative status codes (and for warnings unless allowed)."""
    if rc < 0 or (rc > 0 and not allow_warning):
        msg = load().gm_last_error().decode(errors="replace")
        raise GmError(rc, msg)
    return rc


def ptr(a) -> ctypes.c_void_p:
    """Address of a numpy array (host) or a torch tensor (host or device); None -> NULL."""
    if a is None:
        return ctypes.c_void_p(0)
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)
