"""ctypes bindings of libdogpup_b200.so (the C ABI in include/dogpup_b200.h).

The library is required: importing this module raises if it is missing, and
there is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libdogpup_b200.so"

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
D = C.c_double


class SolveOpts(C.Structure):
    _fields_ = [("tol", D), ("maxit", I32), ("precision", I32), ("inner_tol", D), ("max_refine", I32),
                ("fsai_cap", I32), ("stop_rule", I32), ("check_every", I32)]


class SolveReport(C.Structure):
    _fields_ = [("iterations", I32), ("refinements", I32), ("max_rel_residual", D), ("n_not_converged", I32),
                ("d_status", P)]


PREC_FP64, PREC_MIXED, PREC_MIXED_BICGSTAB = 0, 1, 2
STOP_MAX_ALL, STOP_PER_COLUMN = 0, 1
OK, ERR_NOT_CONVERGED = 0, 5
COL_STATUS = {0: "converged", 1: "maxit", 2: "breakdown_rho", 3: "breakdown_omega", 4: "nonfinite", 5: "zero_rhs"}

# name -> (restype, argtypes)
_SIGS = {
    "dgp_last_error": (C.c_char_p, []),
    "dgp_status_string": (C.c_char_p, [C.c_int]),
    "dgp_version": (C.c_int, []),
    "dgp_kernel_launches": (I64, []),
    "dgp_device_allocations": (I64, []),
    "dgp_smv_mex": (C.c_int, [P, P, P, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, P]),
    "dgp_fsaimv_mex": (C.c_int, [P, P, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, P]),
    "dgp_fsaip_mex": (C.c_int, [P, P, P, P, P, P, P, P, C.c_int, C.c_int, P]),
    "dgp_smv_mex_ic": (C.c_int, [P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, P]),
    "dgp_fsaimv_mex_ic": (C.c_int, [P, P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, P]),
    "dgp_fsaip_mex_ic": (C.c_int, [P, P, P, P, P, P, C.c_int, C.c_int, P]),
    "dgp_fsaip_mex_noalloc": (C.c_int, [P, P, P, P, P, P, P, P, C.c_int, C.c_int, P]),
    "dgp_fem_create": (C.c_int, [C.POINTER(P), P, P, I64, I64, D, P]),
    "dgp_fem_destroy": (C.c_int, [P]),
    "dgp_fem_info": (C.c_int, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(D)]),
    "dgp_fem_pattern": (C.c_int, [P, C.POINTER(P), C.POINTER(P)]),
    "dgp_fem_boundary": (C.c_int, [P, P, P]),
    "dgp_fem_assemble": (C.c_int, [P, P, P, P, P, P]),
    "dgp_fem_adjoint_grad": (C.c_int, [P, P, P, P, P, I32, I32, P, P, P]),
    "dgp_solve_opts_default": (None, [C.POINTER(SolveOpts)]),
    "dgp_solver_create": (C.c_int, [C.POINTER(P), P, P, I64, I64, P, P, D, I32, I32, C.POINTER(SolveOpts), P]),
    "dgp_solver_create_harmonics": (C.c_int, [C.POINTER(P), P, P, I64, I64, P, P, D, P, I32, I32,
                                              C.POINTER(SolveOpts), P]),
    "dgp_solver_update": (C.c_int, [P, P, P, P]),
    "dgp_solver_destroy": (C.c_int, [P]),
    "dgp_solver_memory": (C.c_int, [P, C.POINTER(I64)]),
    "dgp_solver_autotune": (C.c_int, [P, C.POINTER(I32), C.POINTER(I32), C.POINTER(I32), C.POINTER(C.c_float), P]),
    "dgp_solver_set_spmm": (C.c_int, [P, I32, I32, I32]),
    "dgp_solver_set_spmm_kind": (C.c_int, [P, I32]),
    "dgp_solver_set_device_loop": (C.c_int, [P, I32]),
    "dgp_solver_spmm_shape": (C.c_int, [P, C.POINTER(I32), C.POINTER(I32), C.POINTER(I32), C.POINTER(I32)]),
    "dgp_solver_check_spmm": (C.c_int, [P, C.POINTER(D), P]),
    "dgp_solve": (C.c_int, [P, P, P, I32, C.POINTER(SolveOpts), C.POINTER(SolveReport), P]),
    "dgp_solve_mex": (C.c_int, [P, P, P, I32, I32, C.POINTER(SolveOpts), C.POINTER(SolveReport), P]),
    "dgp_solve_sources": (C.c_int, [P, P, P, P, I32, P, C.POINTER(SolveOpts), C.POINTER(SolveReport), P]),
    "dgp_solver_profile_kernel": (C.c_int, [P, I32, I32, C.POINTER(C.c_float), C.POINTER(D), P]),
    "dgp_spmm_A": (C.c_int, [P, P, P, P, I64, I32, I32, P, P, P]),
    "dgp_fsai_pattern": (C.c_int, [P, P, P, P, D, I64, I32, P, P, P]),
    "dgp_fsai_factor": (C.c_int, [P, P, P, P, D, I64, P, P, I32, P, P]),
    "dgp_fsai_apply": (C.c_int, [P, P, P, I64, I64, I32, I32, I32, P, P, P]),
    "dgp_meas": (C.c_int, [P, P, I32, P, I32, P, I64, I32, I32, P, P]),
    "dgp_td2fc": (C.c_int, [P, I64, I32, P, P, I32, P, P]),
    "dgp_fc2td": (C.c_int, [P, I64, I32, P, P, I32, P, P]),
    "dgp_fc2tg": (C.c_int, [P, I64, I32, P, I32, I32, P, P]),
    "dgp_csr_spmv": (C.c_int, [P, P, P, I64, I64, P, P, P]),
    "dgp_set_jacobian_engine": (C.c_int, [I32]),
    "dgp_times_jt": (C.c_int, [P, I64, I64, P, I64, P, P]),
    "dgp_tg_adjoint_rhs": (C.c_int, [P, P, I32, P, I32, P, I32, I32, P, I64, I32, I32, P, P]),
    "dgp_locate_points": (C.c_int, [P, P, I64, I64, P, I64, D, P, P, P]),
    "dgp_grid_to_mesh": (C.c_int, [P, I64, P, P, P, P, P, P, P]),
    "dgp_snap_to_surface": (C.c_int, [P, I64, P, P, I64, P, I64, P, P, P, P]),
    "dgp_solver_set_dot_rows": (C.c_int, [P, I32]),
    "dgp_normal_eq": (C.c_int, [P, I64, I64, P, P, D, I32, P, I64, P, P]),
    "dgp_cholesky_solve": (C.c_int, [P, I64, I64, P, P]),
    "dgp_cholesky_solve_many": (C.c_int, [P, I64, I64, P, I32, I64, P]),
    "dgp_row_dots": (C.c_int, [P, I64, I64, P, P, P, P, P]),
    "dgp_lm_update": (C.c_int, [P, I64, I64, P, P, D, P, I32, P, P]),
    "dgp_jacobian_complex":(C.c_int, [P, P, P, I64, P, P, I32, P, I32, I64, I32, P, P, I32, P, P]),
    "dgp_jacobian_tg": (C.c_int, [P, P, P, I64, P, P, I32, P, I32, I64, I32, P, P, I32, P, I32, I32, P, P, P]),
    "dgp_jacobian_tg_vjp": (C.c_int, [P, P, P, I64, P, P, I32, P, I32, I64, I32, P, P, I32, P, I32, I32, P, P, P,
                                      P]),
}

# every extern "C" symbol include/dogpup_b200.h declares
DECLARED = sorted(_SIGS)


class DgpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dogpup_b200 error {code}: {msg}")
        self.code = code


def load(path: Path | str | None = None) -> C.CDLL:
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build the CUDA library with `python -m dogpup_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = load()


def last_error() -> str:
    return lib.dgp_last_error().decode()


def check(rc: int, allow=()) -> int:
    if rc != OK and rc not in allow:
        raise DgpError(rc, last_error())
    return rc


def default_opts() -> SolveOpts:
    o = SolveOpts()
    lib.dgp_solve_opts_default(C.byref(o))
    return o
