"""germaine_b200 -- B200 (sm_100a) per-frequency forward/adjoint engine for
GERMAINE's 2-D frequency-domain modelling and FWI.

The product is the C-ABI library ``libgermaine_gpu.so`` (include/germaine_gpu.h):
impedance-matrix assembly, nested-dissection multifrontal LU, multi-RHS
substitution with FP64 refinement, and the adjoint-state gradient stack, all
as CUDA kernels.  This package holds its in-tree build (``build.py``), the
ctypes binding (``_lib``) and the host-side mirror of the reference's
per-frequency drivers (``engine.Engine``) and of the reference's file
formats (``files``).
"""
from .engine import (GM_OP_EXACT, GM_OP_REF, GM_PHYS_AC, GM_PHYS_SH, GM_PHYS_TE, GM_PREC_C64_IR,  # noqa: F401
                     GM_PREC_FP64, GM_SYS_A, GM_SYS_AT, Engine, Lbfgs, apply_hess, gauss_filt, mat_change, precond,
                     nonzero, taper_grad_shot, taper_grad_shot1, tikhonov_cost_te, tikhonov_grad_te)
from ._lib import GM_HESS_GREEN, GM_HESS_SHIN  # noqa: F401
from ._lib import GmError  # noqa: F401
from . import files  # noqa: F401
