"""Drop-ins for the reference's solver objects on the Band path.

* ``B200ShiftSession`` replaces ``_aospectrum_cuda.CudssShiftSession``
  (``native/src/bindings.cpp:71-252``): bound to one CSR pattern, it packs
  ``H - z S`` per shift and a column-major right-hand side exactly as the
  reference binding does and calls ``aospectrum_b200_solve_complex64_ubatch_v1``
  (host buffers; factorization, FP64 refinement and solves on the GPU).
* ``NativeB200ShiftSolver`` replaces ``NativeCudssShiftSolver``
  (``src/aospectrum/ciss.py:180-250``): ``solve_shifted(SparsePair, shifts,
  rhs) -> ShiftedResult``.
* ``B200CissSolver`` replaces ``CudssCissSolver`` (``ciss.py:253-391``):
  ``solve_interval(SparsePair, EnergyInterval) -> CissResult`` runs the whole
  CISS step on the GPU for the given CSR matrices (the pattern is analysed
  once and reused while it does not change).
"""

from __future__ import annotations

import ctypes as C
from time import perf_counter
from typing import Any

import numpy as np

from . import native
from .ciss import CissResult, CissSettings, EngineSettings, ShiftedResult, require_shared_pattern
from .data import EnergyInterval
from .errors import InputError, SolverError
from .sparse import SparsePair


class ShiftSolveResult:
    """What ``CudssShiftSession.solve`` returns (bindings.cpp:595-603)."""

    def __init__(self, solutions, stage_seconds, peak, details):
        self.solutions = solutions
        self.stage_seconds = stage_seconds
        self.peak_gpu_memory_bytes = peak
        self.details = details


class B200ShiftSession:
    def __init__(self, indptr, indices, n: int, scalar_dtype: str = "complex64") -> None:
        self._indptr = np.array(indptr, dtype=np.int32, copy=True)
        self._indices = np.array(indices, dtype=np.int32, copy=True)
        self._n = int(n)
        if self._n <= 0 or self._indptr.size != self._n + 1:
            raise ValueError("CSR dimension and indptr differ")
        if self._indptr[0] != 0 or self._indptr[-1] != self._indices.size:
            raise ValueError("CSR indptr endpoints are invalid")
        if scalar_dtype != "complex64":
            raise ValueError("B200ShiftSession supports complex64 only")
        self._closed = False

    def solve(self, hamiltonian, overlap, shifts, rhs) -> ShiftSolveResult:
        if self._closed:
            raise RuntimeError("B200ShiftSession is closed")
        h = np.ascontiguousarray(hamiltonian, dtype=np.complex64)
        s = np.ascontiguousarray(overlap, dtype=np.complex64)
        z = np.ascontiguousarray(shifts, dtype=np.complex64)
        b = np.ascontiguousarray(rhs, dtype=np.complex64)
        nnz = self._indices.size
        if h.ndim != 1 or s.ndim != 1 or h.size != nnz or s.size != nnz:
            raise ValueError("shifted H/S values differ from CSR pattern")
        if z.ndim != 1 or not 1 <= z.size <= 64:
            raise ValueError("shift batch must contain 1 through 64 values")
        if b.ndim != 2 or b.shape[0] != self._n or not 1 <= b.shape[1] <= 256:
            raise ValueError("RHS must have shape (n, 1..256)")
        batch, nrhs = z.size, b.shape[1]
        values = np.ascontiguousarray(h[None, :] - z[:, None] * s[None, :], dtype=np.complex64)
        packed = np.ascontiguousarray(np.broadcast_to(b.T, (batch, nrhs, self._n)))
        out = np.empty_like(packed)
        started = perf_counter()
        req = native.UbatchRequest(native.ABI_VERSION, C.sizeof(native.UbatchRequest), self._n,
                                   nnz, batch, nrhs, self._indptr.ctypes.data,
                                   self._indices.ctypes.data, values.ctypes.data,
                                   packed.ctypes.data, out.ctypes.data)
        res = native.UbatchResult()
        rc = native.library().aospectrum_b200_solve_complex64_ubatch_v1(C.byref(req),
                                                                       C.byref(res))
        if rc != 0 or res.status != 0:
            raise RuntimeError(f"B200 shifted solve failed: return={rc}, status={res.status}, "
                               f"message={res.error_message.decode(errors='replace')}")
        stages = {"device_upload": res.upload_seconds,
                  "descriptor_setup": res.descriptor_setup_seconds,
                  "symbolic_analysis": res.analysis_seconds,
                  "numeric_factorization": res.factorization_seconds,
                  "multi_rhs_solve": res.solve_seconds,
                  "device_download": res.download_seconds,
                  "native_total": res.total_seconds,
                  "binding_wall": perf_counter() - started}
        details = {"batch_count": res.batch_count, "rhs_count": res.rhs_count,
                   "reported_factor_nnz": res.reported_factor_nnz,
                   "reported_pivot_count": res.reported_pivot_count,
                   "permanent_device_bytes": res.permanent_device_bytes,
                   "iterative_refinement_steps": res.iterative_refinement_steps}
        return ShiftSolveResult(np.ascontiguousarray(out.transpose(0, 2, 1)), stages,
                                int(res.peak_device_bytes), details)

    def close(self) -> None:
        self._closed = True


class NativeB200ShiftSolver:
    """``solve_shifted`` seam of the reference CISS solver on the B200 ABI."""

    def __init__(self) -> None:
        self._session: B200ShiftSession | None = None
        self._token: tuple[Any, ...] | None = None

    @staticmethod
    def _pattern_token(m: SparsePair) -> tuple[Any, ...]:
        h = m.hamiltonian
        return (h.shape, h.indptr.size, h.indices.size, int(h.indptr[-1]),
                hash(h.indices.tobytes()))

    def solve_shifted(self, matrices: SparsePair, shifts_ev, rhs) -> ShiftedResult:
        token = self._pattern_token(matrices)
        if self._session is not None and token != self._token:
            raise SolverError("shift session cannot change its CSR pattern")
        try:
            if self._session is None:
                h = matrices.hamiltonian
                self._session = B200ShiftSession(h.indptr, h.indices, h.shape[0])
                self._token = token
            started = perf_counter()
            res = self._session.solve(matrices.hamiltonian.data, matrices.overlap.data,
                                      shifts_ev, rhs)
        except (RuntimeError, ValueError) as exc:
            raise SolverError(f"B200 shifted solve failed: {exc}") from exc
        return ShiftedResult(res.solutions,
                             {"native_total": perf_counter() - started, **res.stage_seconds},
                             res.peak_gpu_memory_bytes)

    def close(self) -> None:
        if self._session is not None:
            self._session.close()
        self._session = None
        self._token = None


class B200CissSolver:
    """``solve_interval`` on host CSR matrices, computed on the GPU."""

    def __init__(self, settings: CissSettings | None = None,
                 engine: EngineSettings | None = None, device: Any = None) -> None:
        self.settings = settings or CissSettings()
        self.engine_settings = engine or EngineSettings()
        self.device = device
        self._engine = None
        self._token: tuple[Any, ...] | None = None

    def solve_interval(self, matrices: SparsePair, interval: EnergyInterval) -> CissResult:
        require_shared_pattern(matrices)
        if self.settings.search_dimension >= matrices.n_orbitals:
            raise SolverError("CISS search dimension must be smaller than matrix dimension")
        h = matrices.hamiltonian
        token = (h.shape, h.indices.size, hash(h.indptr.tobytes()), hash(h.indices.tobytes()))
        if self._engine is None or token != self._token:
            from .engine import BandEngine

            if self._engine is not None:
                self._engine.close()
            self._engine = BandEngine(None, self.settings, self.engine_settings, self.device,
                                      csr=(h.shape[0], h.indptr, h.indices))
            self._token = token
        return self._engine.solve_values(h.data, matrices.overlap.data, interval)[0]

    def close(self) -> None:
        if self._engine is not None:
            self._engine.close()
        self._engine = None
