"""ctypes binding of the phipict_b200 CUDA library (``include/phipict_b200.h``).

The library is built in-tree (``python -m phipict_b200.build``). Loading fails loudly
when it is missing or when no CUDA device is visible: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

import torch

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libphipict_b200.so"

PHB_F32, PHB_F64 = 0, 1
BREC, FREC, IREC, TILE = 48, 16, 8, 1024  # TILE: cells per tile (PHB_TILE_CELLS)
NOALLOC_SCRATCH_BYTES = 32 << 20  # PHB_NOALLOC_SCRATCH_BYTES
AMG_MAX_LEVELS = 12  # PHB_AMG_MAX_LEVELS

# every exported symbol of include/phipict_b200.h
EXPORTS = (
    "phb_last_error", "phb_version",
    "phb_cell_metrics", "phb_face_metrics",
    "phb_advection_matrix", "phb_advection_rhs", "phb_pressure_matrix", "phb_pressure_rhs",
    "phb_divergence", "phb_correct_velocity", "phb_epot_matrix", "phb_epot_rhs", "phb_uxb_epot_rhs",
    "phb_current_lorentz", "phb_scalar_matrix", "phb_scalar_rhs", "phb_nonortho_rhs", "phb_barrier_selftest",
    "phb_scratch_doubles", "phb_subtract_mean", "phb_rms",
    "phb_csr_row_sizes", "phb_csr_pattern", "phb_csr_gather",
    "phb_solve_work_bytes", "phb_solve_state_bytes", "phb_solve_run", "phb_solve_results",
    "phb_release_graphs", "phb_refine_work_bytes", "phb_refine_run", "phb_refine_results",
    "phb_cg_noalloc_bytes", "phb_cg_solve_noalloc", "phb_stencil_apply", "phb_projection_gram", "phb_projection_solve",
    "phb_amg_setup", "phb_amg_refresh_fine", "phb_amg_vcycle", "phb_amg_work_doubles",
    "phb_csr_pcg_work_bytes", "phb_csr_pcg_solve",
    "phb_transpose_stencil", "phb_adj_outer", "phb_adj_advection_matrix", "phb_adj_advection_rhs", "phb_adj_scalar_rhs",
    "phb_adj_pressure_rhs", "phb_adj_divergence", "phb_adj_correct_velocity", "phb_adj_pressure_matrix",
    "phb_adj_uxb_epot_rhs", "phb_adj_lorentz",
)


# phb_nonortho_rhs kinds
PHB_NONORTHO_VELOCITY, PHB_NONORTHO_SCALAR, PHB_NONORTHO_PRESSURE = 0, 1, 2


class PhbDomain(ct.Structure):
    _fields_ = [
        ("dims", ct.c_int32), ("dtype", ct.c_int32),
        ("nblocks", ct.c_int32), ("ninst", ct.c_int32), ("ntiles", ct.c_int32), ("nfixed", ct.c_int32),
        ("ncells", ct.c_int64), ("metric_stride", ct.c_int64), ("face_metric_stride", ct.c_int64),
        ("blocks", ct.c_void_p), ("tiles", ct.c_void_p), ("fixed", ct.c_void_p), ("insts", ct.c_void_p),
        ("metrics", ct.c_void_p), ("face_metrics", ct.c_void_p),
        ("fvel", ct.c_void_p), ("fpot", ct.c_void_p), ("fcw", ct.c_void_p), ("fmask", ct.c_void_p),
        ("dt", ct.c_void_p), ("nu", ct.c_void_p), ("scheme", ct.c_int32), ("nonortho", ct.c_int32),
    ]


class PhbScalar(ct.Structure):
    _fields_ = [
        ("channels", ct.c_int32), ("nu_count", ct.c_int32), ("nu", ct.c_void_p), ("types", ct.c_void_p),
        ("values", ct.c_void_p), ("offsets", ct.c_void_p), ("statics", ct.c_void_p),
    ]


class PhbTolerance(ct.Structure):
    _fields_ = [
        ("mode", ct.c_int32), ("pad", ct.c_int32),
        ("rtol", ct.c_double), ("atol", ct.c_double), ("floor_eps", ct.c_double), ("fallback", ct.c_double),
        ("values", ct.c_void_p),
    ]


class PhbSolve(ct.Structure):
    _fields_ = [
        ("kind", ct.c_int32), ("vec_dtype", ct.c_int32), ("mat_dtype", ct.c_int32), ("nrhs", ct.c_int32),
        ("maxit", ct.c_int32), ("return_best", ct.c_int32), ("use_graph", ct.c_int32), ("check_every", ct.c_int32),
        ("tol", PhbTolerance),
        ("A", ct.c_void_p), ("b", ct.c_void_p), ("x", ct.c_void_p),
        ("work", ct.c_void_p), ("state", ct.c_void_p),
        ("amg", ct.c_void_p), ("ctas_per_sm", ct.c_int32), ("pad", ct.c_int32),
    ]


class PhbSolveResult(ct.Structure):
    _fields_ = [
        ("final_residual", ct.c_double), ("used_iterations", ct.c_int32), ("converged", ct.c_int32),
        ("finite", ct.c_int32), ("status", ct.c_int32), ("inner_iterations", ct.c_int32), ("pad", ct.c_int32),
    ]


class PhbRefine(ct.Structure):
    _fields_ = [
        ("kind", ct.c_int32), ("nrhs", ct.c_int32), ("max_outer", ct.c_int32), ("inner_maxit", ct.c_int32),
        ("use_graph", ct.c_int32), ("ctas_per_sm", ct.c_int32), ("inner_rtol", ct.c_double),
        ("tol", PhbTolerance),
        ("A64", ct.c_void_p), ("A32", ct.c_void_p), ("b", ct.c_void_p), ("x", ct.c_void_p),
        ("work", ct.c_void_p), ("state", ct.c_void_p),
        ("amg", ct.c_void_p),
    ]


class PhbAmgLevel(ct.Structure):
    _fields_ = [("dom", PhbDomain), ("A", ct.c_void_p), ("b", ct.c_void_p), ("x", ct.c_void_p), ("wdinv", ct.c_void_p),
                ("inst_cells", ct.c_int32), ("pad", ct.c_int32)]


class PhbAmg(ct.Structure):
    _fields_ = [
        ("nlevels", ct.c_int32), ("coarse_n", ct.c_int32), ("omega", ct.c_float), ("coarse_scale", ct.c_float),
        ("tail_level", ct.c_int32), ("pad", ct.c_int32), ("coarse_inv", ct.c_void_p),
        ("work", ct.c_void_p), ("work_doubles", ct.c_int64),
        ("levels", PhbAmgLevel * AMG_MAX_LEVELS),
    ]


class PhbCsrLevel(ct.Structure):
    _fields_ = [
        ("a_row", ct.c_void_p), ("a_col", ct.c_void_p), ("a_val", ct.c_void_p), ("a_val_stride", ct.c_int64),
        ("dinv", ct.c_void_p), ("r_row", ct.c_void_p), ("r_col", ct.c_void_p), ("r_val", ct.c_void_p),
        ("p_row", ct.c_void_p), ("p_col", ct.c_void_p), ("p_val", ct.c_void_p), ("n", ct.c_int32), ("pad", ct.c_int32),
    ]


class PhbCsrPcg(ct.Structure):
    _fields_ = [
        ("dtype", ct.c_int32), ("hdtype", ct.c_int32),
        ("n", ct.c_int32), ("nenv", ct.c_int32), ("nlevels", ct.c_int32), ("coarse_n", ct.c_int32),
        ("coarse_batched", ct.c_int32),
        ("maxit", ct.c_int32), ("normalized", ct.c_int32), ("return_best", ct.c_int32), ("project_constant", ct.c_int32),
        ("pre_sweeps", ct.c_int32), ("post_sweeps", ct.c_int32), ("pad", ct.c_int32),
        ("tol", ct.c_double), ("omega", ct.c_double), ("tolerances", ct.c_void_p),
        ("row", ct.c_void_p), ("col", ct.c_void_p), ("val", ct.c_void_p), ("val_stride", ct.c_int64),
        ("levels", ct.c_void_p), ("coarse_pinv", ct.c_void_p), ("b", ct.c_void_p), ("x", ct.c_void_p),
        ("work", ct.c_void_p),
    ]


_lib: ct.CDLL | None = None


def load() -> ct.CDLL:
    """Load the library (building it first if this is a source checkout without it)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        if os.environ.get("PHIPICT_B200_NO_BUILD"):
            raise RuntimeError(f"phipict_b200 CUDA library missing: {LIB_PATH}")
        from phipict_b200 import build as _build

        _build.build()
    lib = ct.CDLL(str(LIB_PATH))
    P = ct.c_void_p
    I = ct.c_int
    I64 = ct.c_int64
    DP = ct.POINTER(PhbDomain)
    lib.phb_last_error.restype = ct.c_char_p
    lib.phb_version.restype = I
    sig = {
        "phb_cell_metrics": [I, I, I, I, I, P, P, I64, P],
        "phb_face_metrics": [I, I, I, I, I, P, I, P, I64, P],
        "phb_advection_matrix": [DP, P, P, P, P, P],
        "phb_advection_rhs": [DP, P, P, I, P, P],
        "phb_scalar_matrix": [DP, P, ct.POINTER(PhbScalar), I, P, P, P, P],
        "phb_scalar_rhs": [DP, P, P, ct.POINTER(PhbScalar), P, P],
        "phb_nonortho_rhs": [DP, I, P, ct.POINTER(PhbScalar), P, P, P],
        "phb_barrier_selftest": [I, I, I, ct.c_uint, P, ct.POINTER(I), ct.POINTER(I), P],
        "phb_pressure_matrix": [DP, P, P, P, P],
        "phb_pressure_rhs": [DP, P, P, P, P, P, I, P, P],
        "phb_divergence": [DP, P, P, P],
        "phb_correct_velocity": [DP, P, P, P, P, P],
        "phb_epot_matrix": [DP, P, P, P],
        "phb_epot_rhs": [DP, P, P, P],
        "phb_uxb_epot_rhs": [DP, P, P, P, P, P],
        "phb_current_lorentz": [DP, P, P, P, P, P, P, I, P],
        "phb_subtract_mean": [DP, P, I, P, P],
        "phb_rms": [DP, P, I, P, P, P],
        "phb_csr_row_sizes": [DP, P, P],
        "phb_csr_pattern": [DP, P, P, P, P],
        "phb_csr_gather": [I, I64, P, P, P, P],
        "phb_solve_run": [DP, ct.POINTER(PhbSolve), P],
        "phb_solve_results": [DP, ct.POINTER(PhbSolve), ct.POINTER(PhbSolveResult), P],
        "phb_release_graphs": [],
        "phb_refine_run": [DP, ct.POINTER(PhbRefine), ct.POINTER(PhbSolveResult), ct.POINTER(ct.c_int), P],
        "phb_refine_results": [DP, ct.POINTER(PhbRefine), ct.POINTER(PhbSolveResult), ct.POINTER(ct.c_int), P],
        "phb_cg_solve_noalloc": [DP, I, I, P, P, P, ct.POINTER(PhbTolerance), I, I, ct.POINTER(PhbSolveResult), P],
        "phb_amg_setup": [ct.POINTER(PhbAmg), P],
        "phb_amg_refresh_fine": [ct.POINTER(PhbAmg), P],
        "phb_transpose_stencil": [DP, P, P, P],
        "phb_stencil_apply": [DP, P, P, P, ct.c_int32, I64, P],
        "phb_projection_gram": [P, P, P, ct.c_int32, I64, I64, P, P, P],
        "phb_projection_solve": [P, P, ct.c_int32, ct.c_double, P, P],
        "phb_adj_outer": [DP, I, P, P, ct.c_double, P, P],
        "phb_adj_advection_matrix": [DP, P, P, P, P],
        "phb_adj_advection_rhs": [DP, P, P, P, P, P, P],
        "phb_adj_scalar_rhs": [DP, ct.POINTER(PhbScalar), P, P, P, P, P, P, P, P],
        "phb_adj_pressure_rhs": [DP, P, P, P, P, P, P, P, P, P, P, P, P, P],
        "phb_adj_divergence": [DP, P, P, P, P],
        "phb_adj_correct_velocity": [DP, P, P, P, P, P, P, P],
        "phb_adj_pressure_matrix": [DP, P, P, P, P],
        "phb_adj_uxb_epot_rhs": [DP, P, P, P, P, P],
        "phb_adj_lorentz": [DP, P, P, P, P, P, P, P, P, P],
        "phb_amg_vcycle": [ct.POINTER(PhbAmg), P, P, P],
        "phb_csr_pcg_solve": [ct.POINTER(PhbCsrPcg), ct.POINTER(PhbSolveResult), P],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = I
    for name, args in {
        "phb_scratch_doubles": [DP, I],
        "phb_solve_work_bytes": [DP, I, I, I],
        "phb_solve_state_bytes": [DP, I],
        "phb_refine_work_bytes": [DP, I, I],
        "phb_cg_noalloc_bytes": [DP, I, I],
        "phb_amg_work_doubles": [ct.POINTER(PhbAmg)],
        "phb_csr_pcg_work_bytes": [ct.POINTER(PhbCsrPcg)],
    }.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = I64
    _lib = lib
    return lib


class PhbError(RuntimeError):
    pass


def call(name: str, *args) -> int:
    """Call an entry point and raise PhbError with the library's message on failure."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.phb_last_error().decode(errors="replace")
        raise PhbError(f"{name} failed ({rc}): {msg}")
    return rc


def stream_ptr(device: torch.device | None = None) -> int:
    """The raw handle of torch's current CUDA stream."""
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float64:
        return PHB_F64
    if dtype == torch.float32:
        return PHB_F32
    raise TypeError(f"unsupported dtype {dtype}; phipict_b200 computes in float32 or float64")


def require_cuda(device: torch.device) -> None:
    if device.type != "cuda":
        raise RuntimeError(
            "phipict_b200 runs on CUDA devices only (the product path has no CPU fallback); "
            f"got device {device}"
        )
    if not torch.cuda.is_available():
        raise RuntimeError("phipict_b200 needs a CUDA device, but torch.cuda.is_available() is False")
