"""Gamma-point real symmetric shifted factorization with inertia.

The reference factors ``H - sigma S`` at the Gamma point with cuDSS's
symmetric solver and reads its inertia: the number of states below, at and
above ``sigma``.  Its ordinal locator bisects on that count to place a shift
between two requested state numbers (``src/aospectrum/primme.py:281-397``,
``native/src/aospectrum_cudss_shift_factor.c:232-742``).  Here the same
factorization runs on this library's tile engine
(``aosb_shift_factor_*``): block elimination over the symbolic plan, FP32
tile updates, and the inertia summed over Bunch-Kaufman LDL^T factors of the
eliminated diagonal tiles.

``GammaShiftFactor.update_numeric(shift_ev)`` returns the reference's
``NumericUpdate`` / ``InertiaPoint`` fields, so the reference's
``OrdinalLocator.locate_observing`` can drive it as its observer.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from time import perf_counter
from typing import Any

import numpy as np

from . import native
from .errors import InputError, SolverError


@dataclass(frozen=True, slots=True)
class InertiaPoint:
    """Eigenvalue counts of the pencil (H, S) relative to ``energy_ev``
    (reference ``primme.py:29-35``)."""

    energy_ev: float
    below: int
    zero: int
    above: int
    dimension: int


@dataclass(slots=True)
class NumericUpdate:
    """One refactorization (reference ``primme.py:37-42``)."""

    inertia: InertiaPoint
    numeric_epoch: int
    stage_seconds: dict[str, float]
    details: dict[str, Any] = field(default_factory=dict)


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise SolverError("the Gamma shift factorization needs a CUDA device")
    return torch


class GammaShiftFactor:
    """Real symmetric ``H - shift S`` factored on the device.

    ``h_values`` / ``s_values``: device float32 tensors holding the real
    CSR values of H(Gamma), S(Gamma) on the pattern (``indptr``,
    ``indices``, host arrays); only the upper triangle is read, as the
    reference's upper-triangle cuDSS view reads it."""

    def __init__(self, n: int, indptr: np.ndarray, indices: np.ndarray, h_values: Any,
                 s_values: Any, shift_ev: float, *, maximum_rhs: int = 8,
                 device: Any = None) -> None:
        torch = _torch()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else torch.device(device).index or 0)
        self.n = int(n)
        ip = np.ascontiguousarray(indptr)
        if ip[-1] > np.iinfo(np.int32).max:
            raise InputError("the shift factorization takes an int32 CSR pattern")
        self.indptr = ip.astype(np.int32)
        self.indices = np.ascontiguousarray(indices, dtype=np.int32)
        self.nnz = int(self.indices.size)
        self.maximum_rhs = int(maximum_rhs)
        self._values(h_values, s_values)
        self.epoch = 0
        self.shift_ev = float(shift_ev)
        handle = native.c_vp()
        t0 = perf_counter()
        with torch.cuda.device(self.device):
            self.stream = torch.cuda.current_stream(self.device)
            native.call("aosb_shift_factor_create_device", C.byref(handle), self.n, self.nnz,
                        self.indptr.ctypes.data, self.indices.ctypes.data,
                        self.h.data_ptr(), self.s.data_ptr(), C.c_float(self.shift_ev),
                        self.maximum_rhs, self.stream.cuda_stream)
        self.handle = handle
        self.last = self._update(perf_counter() - t0)

    @classmethod
    def from_bundle(cls, bundle: Any, shift_ev: float, *, maximum_rhs: int = 8,
                    device: Any = None) -> "GammaShiftFactor":
        """H(Gamma), S(Gamma) of a bundle from the device Bloch sum (real
        block values give exactly real Gamma values)."""
        torch = _torch()
        from .engine import BlochDevice

        dev = torch.device("cuda", torch.cuda.current_device() if device is None
                           else torch.device(device).index or 0)
        bloch = BlochDevice(bundle, dev)
        try:
            h, s = bloch.apply(np.zeros((1, 3)))
            if bool(torch.any(h.imag != 0)) or bool(torch.any(s.imag != 0)):
                raise InputError("Gamma-point values are not real (complex block values)")
            return cls(bloch.n, bloch.indptr, bloch.indices, h.real[0].contiguous(),
                       s.real[0].contiguous(), shift_ev, maximum_rhs=maximum_rhs, device=dev)
        finally:
            bloch.close()

    def _values(self, h_values: Any, s_values: Any) -> None:
        torch = _torch()
        h = torch.as_tensor(h_values, device=self.device, dtype=torch.float32).reshape(-1)
        s = torch.as_tensor(s_values, device=self.device, dtype=torch.float32).reshape(-1)
        if h.numel() != self.nnz or s.numel() != self.nnz:
            raise InputError("H/S values differ from the CSR pattern")
        self.h, self.s = h.contiguous(), s.contiguous()

    def stats(self) -> dict[str, Any]:
        st = native.ShiftFactorStats()
        native.library().aosb_shift_factor_get_stats(self.handle, C.byref(st))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def _update(self, seconds: float) -> NumericUpdate:
        st = self.stats()
        below, above = int(st["inertia_negative"]), int(st["inertia_positive"])
        zero = self.n - below - above
        if below < 0 or above < 0 or zero < 0:
            raise SolverError("inertia counts are invalid")
        self.epoch += 1
        return NumericUpdate(
            InertiaPoint(self.shift_ev, below, zero, above, self.n), self.epoch,
            {"factorization": float(st["factorization_seconds"]),
             "analysis": float(st["analysis_seconds"]), "total": seconds},
            {"factor_nnz": int(st["factor_nnz"]), "pivot_count": int(st["pivot_count"]),
             "peak_device_bytes": int(st["peak_device_bytes"])})

    def update_numeric(self, shift_ev: float, h_values: Any = None,
                       s_values: Any = None) -> NumericUpdate:
        """Refactor at ``shift_ev`` (with new values if given) and return the
        inertia there; the symbolic analysis is reused."""
        torch = _torch()
        if h_values is not None or s_values is not None:
            self._values(self.h if h_values is None else h_values,
                         self.s if s_values is None else s_values)
        self.shift_ev = float(shift_ev)
        t0 = perf_counter()
        with torch.cuda.device(self.device):
            native.call("aosb_shift_factor_refactor_device", self.handle, self.h.data_ptr(),
                        self.s.data_ptr(), C.c_float(self.shift_ev))
        self.last = self._update(perf_counter() - t0)
        return self.last

    @property
    def inertia(self) -> InertiaPoint:
        return self.last.inertia

    def solve(self, rhs: Any) -> Any:
        """x = (H - shift S)^{-1} rhs for a float32 [n] or [n, m] block
        (m <= maximum_rhs); returns a device tensor of the same shape."""
        torch = _torch()
        b = torch.as_tensor(rhs, device=self.device, dtype=torch.float32)
        vec = b.ndim == 1
        b2 = b.reshape(self.n, -1)
        m = b2.shape[1]
        if b2.shape[0] != self.n or not 1 <= m <= self.maximum_rhs:
            raise InputError("right-hand side does not match the factorization")
        cm = b2.t().contiguous()          # column-major n x m, leading dimension n
        out = torch.empty_like(cm)
        with torch.cuda.device(self.device):
            native.call("aosb_shift_factor_solve", self.handle, cm.data_ptr(), self.n,
                        out.data_ptr(), self.n, m)
        x = out.t()
        return x.reshape(self.n) if vec else x

    def close(self) -> None:
        if getattr(self, "handle", None):
            native.library().aosb_shift_factor_destroy(self.handle)
            self.handle = None

    def __enter__(self) -> "GammaShiftFactor":
        return self

    def __exit__(self, *exc: Any) -> None:
        self.close()
