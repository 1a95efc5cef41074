"""ctypes binding of libaospectrum_b200.so (the C ABI in
``include/aospectrum_b200.h``).

There is no fallback: when the library is absent or fails to load, every
entry point raises ``SolverError`` naming the build command.  Device
pointers are passed as integers (``tensor.data_ptr()``), streams as the raw
``cudaStream_t`` value (``torch.cuda.current_stream().cuda_stream``).
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Any

import numpy as np

from .errors import SolverError

LIBRARY_PATH = Path(__file__).resolve().parent / "libaospectrum_b200.so"
ABI_VERSION = 1
ERROR_CAPACITY = 512

PRECISION_PLAIN = 0
PRECISION_BF16X3 = 1
PRECISION_BF16X3_FP32_PANELS = 2
PRECISION_BF16X3_ONE_STEP = 3
SOLVE_TENSOR_CORES = 1
SOLVE_GRAPH = 2

STATUS_NAMES = {
    10: "ABI mismatch", 11: "dimensions", 12: "batch", 13: "null pointer",
    14: "indptr span", 20: "CUDA error", 21: "engine", 22: "device info",
    30: "CSR not monotonic", 31: "CSR column", 32: "CSR order", 33: "missing diagonal",
    34: "size", 35: "non-finite matrix", 36: "non-finite rhs", 40: "memory",
    41: "topology", 50: "zero pivot", 51: "non-finite factor", 52: "timeout",
    53: "argument", 54: "unsupported",
}

c_i32, c_i64, c_u32, c_sz, c_vp = C.c_int32, C.c_int64, C.c_uint32, C.c_size_t, C.c_void_p


class PlanOptions(C.Structure):
    _fields_ = [("abi_version", c_u32), ("struct_size", c_u32), ("tile", c_i32),
                ("ordering", c_i32), ("leaf_dofs", c_i32), ("pad_nodes", c_i32)]


class PlanInfo(C.Structure):
    _fields_ = [("n", c_i64), ("n_pad", c_i64), ("nnz", c_i64), ("n_tiles", c_i64),
                ("n_slots", c_i64), ("n_supervariables", c_i64), ("n_nodes", c_i64),
                ("schur_tile_updates", c_i64), ("tree_levels", c_i64), ("tile", c_i32),
                ("reserved", c_i32), ("factor_flops", C.c_double),
                ("factor_flops_alg", C.c_double), ("factor_bytes", C.c_double)]


class FactorArgs(C.Structure):
    _fields_ = [("abi_version", c_u32), ("struct_size", c_u32), ("n_pencils", c_i32),
                ("precision", c_i32), ("h_values", c_vp), ("s_values", c_vp),
                ("pencil_k", c_vp), ("shifts", c_vp), ("factor", c_vp), ("pivots", c_vp),
                ("status", c_vp), ("workspace", c_vp), ("stream", c_vp)]


class SolveArgs(C.Structure):
    _fields_ = [("abi_version", c_u32), ("struct_size", c_u32), ("n_pencils", c_i32),
                ("n_rhs", c_i32), ("adjoint", c_i32), ("flags", c_i32), ("factor", c_vp),
                ("pivots", c_vp), ("work", c_vp), ("scratch", c_vp), ("stream", c_vp)]


class UbatchRequest(C.Structure):
    _fields_ = [("abi_version", c_u32), ("struct_size", c_u32), ("n", c_i64), ("nnz", c_i64),
                ("batch_count", c_i32), ("rhs_count", c_i32), ("indptr", c_vp),
                ("indices", c_vp), ("values", c_vp), ("rhs", c_vp), ("solution", c_vp)]


class UbatchResult(C.Structure):
    _fields_ = [("abi_version", c_u32), ("struct_size", c_u32), ("status", c_i32),
                ("engine_status", c_i32), ("n", c_i64), ("nnz", c_i64),
                ("diagonal_count", c_i64), ("reported_factor_nnz", c_i64),
                ("reported_pivot_count", c_i32), ("batch_count", c_i32),
                ("rhs_count", c_i32), ("iterative_refinement_steps", c_i32),
                ("upload_seconds", C.c_double), ("descriptor_setup_seconds", C.c_double),
                ("analysis_seconds", C.c_double), ("factorization_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("download_seconds", C.c_double),
                ("total_seconds", C.c_double), ("permanent_device_bytes", C.c_uint64),
                ("peak_device_bytes", C.c_uint64), ("permanent_host_bytes", C.c_uint64),
                ("peak_host_bytes", C.c_uint64), ("free_device_bytes_before", C.c_uint64),
                ("free_device_bytes_after_upload", C.c_uint64),
                ("free_device_bytes_after_factorization", C.c_uint64),
                ("free_device_bytes_after_solve", C.c_uint64),
                ("total_device_bytes", C.c_uint64),
                ("error_message", C.c_char * ERROR_CAPACITY)]


class ShiftFactorStats(C.Structure):
    _fields_ = [("upper_nnz", c_i64), ("factor_nnz", c_i64), ("pivot_count", c_i32),
                ("inertia_positive", c_i32), ("inertia_negative", c_i32),
                ("solve_calls", c_i32), ("solved_rhs", c_i64),
                ("preparation_seconds", C.c_double), ("upload_seconds", C.c_double),
                ("analysis_seconds", C.c_double), ("factorization_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("permanent_device_bytes", C.c_uint64),
                ("peak_device_bytes", C.c_uint64), ("permanent_host_bytes", C.c_uint64),
                ("peak_host_bytes", C.c_uint64),
                ("free_device_bytes_before_factorization", C.c_uint64),
                ("free_device_bytes_after_factorization", C.c_uint64)]


# name: (restype, argtypes)
_SIGNATURES: dict[str, tuple[Any, list[Any]]] = {
    "aosb_abi_version": (c_u32, []),
    "aosb_build_info": (C.c_char_p, []),
    "aosb_launch_count": (C.c_uint64, []),
    "aosb_kernel_timing": (C.c_int, [c_i32]),
    "aosb_kernel_timing_read": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.POINTER(c_i64)]),
    "aosb_kernel_timing_read_category": (C.c_int, [c_i32, C.POINTER(C.c_double),
                                                   C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                   C.POINTER(c_i64)]),
    "aospectrum_b200_solve_complex64_ubatch_v1": (C.c_int, [C.POINTER(UbatchRequest),
                                                            C.POINTER(UbatchResult)]),
    "aosb_bloch_create": (C.c_int, [c_i64, c_i64, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp,
                                    C.POINTER(c_vp), C.c_char_p, c_sz]),
    "aosb_bloch_upload": (C.c_int, [c_vp, C.c_char_p, c_sz]),
    "aosb_bloch_info": (C.c_int, [c_vp, C.POINTER(c_i64), C.POINTER(c_i64)]),
    "aosb_bloch_export": (C.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "aosb_bloch_export_groups": (C.c_int, [c_vp, C.POINTER(c_i64), C.POINTER(c_i64), c_vp, c_vp,
                                           c_vp, c_vp, c_vp]),
    "aosb_bloch_device_pattern": (C.c_int, [c_vp, C.POINTER(c_vp), C.POINTER(c_vp)]),
    "aosb_bloch_apply": (C.c_int, [c_vp, c_i32, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_vp,
                                   C.c_char_p, c_sz]),
    "aosb_bloch_destroy": (None, [c_vp]),
    "aosb_plan_create": (C.c_int, [c_i64, c_vp, c_vp, c_vp, c_i64, C.POINTER(PlanOptions),
                                   C.POINTER(c_vp), C.c_char_p, c_sz]),
    "aosb_plan_upload": (C.c_int, [c_vp, C.c_char_p, c_sz]),
    "aosb_plan_info": (C.c_int, [c_vp, C.POINTER(PlanInfo)]),
    "aosb_plan_export_perm": (C.c_int, [c_vp, c_vp]),
    "aosb_plan_export_slots": (C.c_int, [c_vp, c_vp]),
    "aosb_plan_export_super_steps": (C.c_int, [c_vp, C.POINTER(c_i64), C.POINTER(c_i64),
                                               C.POINTER(c_i64), c_vp, c_vp, c_vp, c_vp]),
    "aosb_plan_export_pair_steps": (C.c_int, [c_vp, C.POINTER(c_i64), C.POINTER(c_i64), c_vp,
                                              c_vp, c_vp, c_vp]),
    "aosb_plan_destroy": (None, [c_vp]),
    "aosb_factor_bytes": (c_sz, [c_vp, c_i32]),
    "aosb_factor_workspace_bytes": (c_sz, [c_vp, c_i32, c_i32]),
    "aosb_factor_set_lookahead_sms": (c_i32, [c_i32]),
    "aosb_tc_set_wait_limit": (c_i64, [c_i64]),
    "aosb_factor_set_schur_pairs": (c_i32, [c_i32]),
    "aosb_solve_set_ctas_per_sm": (c_i32, [c_i32]),
    "aosb_solve_set_lookahead": (c_i32, [c_i32]),
    "aosb_factor": (C.c_int, [c_vp, C.POINTER(FactorArgs), C.c_char_p, c_sz]),
    "aosb_solve": (C.c_int, [c_vp, C.POINTER(SolveArgs), C.c_char_p, c_sz]),
    "aosb_solve_scratch_bytes": (c_sz, [c_vp, c_i32, c_i32]),
    "aosb_solve_check": (C.c_int, [c_vp, C.POINTER(SolveArgs), C.c_char_p, c_sz]),
    "aosb_gather_rhs": (C.c_int, [c_vp, c_i32, c_i32, c_vp, c_i64, c_vp, c_vp, C.c_char_p, c_sz]),
    "aosb_scatter_solution": (C.c_int, [c_vp, c_i32, c_i32, c_vp, c_vp, c_i32, c_vp,
                                        C.c_char_p, c_sz]),
    "aosb_shifted_residual": (C.c_int, [c_i64, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp, c_i64,
                                        c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp,
                                        C.c_char_p, c_sz]),
    "aosb_shifted_residual_blocks": (C.c_int, [c_i64, c_i32, c_i32, c_i64, c_vp, c_i32, c_vp,
                                               c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp,
                                               c_i64, c_vp, c_vp, c_vp, C.c_char_p, c_sz]),
    "aosb_spmm_blocks": (C.c_int, [c_i64, c_i32, c_i64, c_vp, c_i32, c_vp, c_vp, c_vp, c_i64,
                                   c_vp, c_i64, c_vp, c_i64, c_vp, C.c_char_p, c_sz]),
    "aosb_spmm": (C.c_int, [c_i64, c_i32, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_i64, c_vp,
                            C.c_char_p, c_sz]),
    "aosb_moments_accumulate": (C.c_int, [c_i64, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp,
                                          C.c_char_p, c_sz]),
    "aosb_gram_scratch_bytes": (c_sz, [c_i64, c_i32, c_i32]),
    "aosb_gram": (C.c_int, [c_i64, c_i32, c_i32, c_vp, c_i64, c_vp, c_i64, c_vp, c_vp, c_vp,
                            C.c_char_p, c_sz]),
    "aosb_gram_noalloc": (C.c_int, [c_i64, c_i32, c_i32, c_vp, c_i64, c_vp, c_i64, c_vp, c_vp,
                                    C.c_char_p, c_sz]),
    "aosb_shift_factor_create_device": (C.c_int, [C.POINTER(c_vp), c_i64, c_i64, c_vp, c_vp,
                                                  c_vp, c_vp, C.c_float, c_i32, c_vp,
                                                  C.c_char_p, c_sz]),
    "aosb_shift_factor_refactor_device": (C.c_int, [c_vp, c_vp, c_vp, C.c_float, C.c_char_p,
                                                    c_sz]),
    "aosb_shift_factor_solve": (C.c_int, [c_vp, c_vp, c_i64, c_vp, c_i64, c_i32, C.c_char_p,
                                          c_sz]),
    "aosb_shift_factor_get_stats": (None, [c_vp, C.POINTER(ShiftFactorStats)]),
    "aosb_shift_factor_destroy": (None, [c_vp]),
    "aosb_dense_mul": (C.c_int, [c_i64, c_i32, c_i32, c_vp, c_i64, c_vp, c_vp, c_i64, c_vp,
                                 C.c_char_p, c_sz]),
    "aosb_column_norms": (C.c_int, [c_i64, c_i32, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp,
                                    C.c_char_p, c_sz]),
}

_lib: C.CDLL | None = None


def library() -> C.CDLL:
    """Load the library once; raise ``SolverError`` when it is unusable."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise SolverError(f"{LIBRARY_PATH.name} is not built; run "
                          "`python -m aospectrum_b200.build` (needs nvcc)")
    try:
        lib = C.CDLL(str(LIBRARY_PATH))
    except OSError as exc:
        raise SolverError(f"cannot load {LIBRARY_PATH}: {exc}") from exc
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.aosb_abi_version() != ABI_VERSION:
        raise SolverError("libaospectrum_b200 ABI version mismatch")
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


class NativeError(SolverError):
    def __init__(self, code: int, message: str) -> None:
        super().__init__(f"{message} (status {code}: {STATUS_NAMES.get(code, 'unknown')})")
        self.code = code


def call(name: str, *args: Any) -> int:
    """Call an entry point whose last two parameters are (err, err_cap)."""
    buf = C.create_string_buffer(ERROR_CAPACITY)
    rc = getattr(library(), name)(*args, buf, ERROR_CAPACITY)
    if rc != 0:
        raise NativeError(rc, f"{name} failed: {buf.value.decode(errors='replace')}")
    return rc


def ptr(a: Any) -> int | None:
    """Device or host address of a tensor / array (None for None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
