"""ctypes wrapper of oracle/bloch_ref.c -- test oracle only."""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from .bloch_ref import RefPattern, phases

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle_bloch.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        vp, i64 = C.c_void_p, C.c_int64
        _lib.oracle_bloch_sum.argtypes = [i64, i64, vp, vp, vp, C.c_int, vp, vp, vp]
        _lib.oracle_project_hermitian.argtypes = [i64, vp, vp, i64, vp, vp]
    return _lib


def bloch_values(pat: RefPattern, values: np.ndarray, k) -> np.ndarray:
    lib = _load()
    ph = phases(pat.shifts, k)
    kind = 1 if np.iscomplexobj(values) else 0
    vals = np.ascontiguousarray(values, dtype=np.complex64 if kind else np.float32)
    starts = np.ascontiguousarray(pat.starts, dtype=np.int64)
    src = np.ascontiguousarray(pat.source, dtype=np.int64)
    grp = np.ascontiguousarray(pat.group, dtype=np.int64)
    out = np.empty(starts.size, dtype=np.complex64)
    lib.oracle_bloch_sum(starts.size, src.size, starts.ctypes.data, src.ctypes.data,
                         grp.ctypes.data, kind, vals.ctypes.data, ph.ctypes.data, out.ctypes.data)
    up = np.ascontiguousarray(pat.upper, dtype=np.int64)
    lo = np.ascontiguousarray(pat.lower, dtype=np.int64)
    dg = np.ascontiguousarray(pat.diagonal, dtype=np.int64)
    lib.oracle_project_hermitian(up.size, up.ctypes.data, lo.ctypes.data, dg.size,
                                 dg.ctypes.data, out.ctypes.data)
    return out
