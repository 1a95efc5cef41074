"""GPU Band engine: device-resident bundle, Bloch sums and batched CISS.

One ``BandEngine`` per (bundle, process, GPU).  Construction uploads the
operator block values once, builds the CSR pattern (``aosb_bloch_create``)
and the symbolic plan (``aosb_plan_create``, once per bundle).  Each call of
``solve_kpoints`` then runs, for a group of k points:

1. Bloch sums H(k), S(k) on the device (bit-identical to the reference
   numpy path for real block values);
2. rhs = S(k) Q in FP64 with the reference's probe block Q;
3. every (k, contour node) pencil through batched tile factorizations; in
   "mixed" precision a node and its conjugate partner share one
   factorization (A^H = H - conj(z) S), the Schur updates run on the tensor
   cores in split BF16, and every solve gets FP64 iterative refinement;
4. moment accumulation, S-Gram rank truncation, Rayleigh-Ritz, ghost
   filter and FP64 residuals.

This replaces ``BlochWorkspace.update`` + ``CudssCissSolver.solve_interval``
of the reference (``src/aospectrum/sparse.py:199-245``,
``src/aospectrum/ciss.py:266-391``).
"""

from __future__ import annotations

import math
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from time import perf_counter
from typing import Any, Sequence

import numpy as np

from . import native
from .ciss import (
    CissResult,
    CissSettings,
    EngineSettings,
    contour_geometry,
    interval_mask,
    moment_coefficients,
    nonspurious_mask,
    probe_block,
    projected_eigh,
    result_warnings,
    small_lapack,
    truncate_gram,
)
from .data import EnergyInterval, LocalizedOperatorBundle
from .errors import InputError, SolverError
from .sparse import SparsePair


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise SolverError("the B200 Band engine needs a CUDA device")
    return torch


def row_blocks(indptr: np.ndarray, indices: np.ndarray, max_rows: int = 16,
               starts: np.ndarray | None = None) -> np.ndarray:
    """Start rows of blocks of consecutive rows with identical column sets
    (at most ``max_rows`` rows each), closed by n.  ``starts`` (e.g. the atom
    offsets of a bundle) are trusted; otherwise runs are detected."""
    n = indptr.size - 1
    if starts is None:
        lens = np.diff(indptr)
        same = np.zeros(n, dtype=bool)
        for r in range(1, n):
            if lens[r] == lens[r - 1] and np.array_equal(
                    indices[indptr[r]:indptr[r + 1]], indices[indptr[r - 1]:indptr[r]]):
                same[r] = True
        starts = np.flatnonzero(~same)
    out = []
    bounds = list(np.asarray(starts, dtype=np.int64)) + [n]
    for a, b in zip(bounds[:-1], bounds[1:]):
        out.extend(range(int(a), int(b), max_rows))
    out.append(n)
    return np.asarray(out, dtype=np.int32)


def choose_tile(n: int) -> int:
    if n <= 256:
        return 32
    if n <= 4096:
        return 64
    return 128


@dataclass
class PlanSummary:
    n: int
    n_pad: int
    nnz: int
    tile: int
    n_tiles: int
    n_slots: int
    n_nodes: int
    tree_levels: int
    factor_flops: float
    factor_flops_alg: float
    factor_bytes: float


class BlochDevice:
    """CSR pattern of a bundle plus device-resident block values.

    With ``upload=False`` only the host side is built (pattern, tables);
    ``upload`` then copies the tables and block values to the device."""

    def __init__(self, bundle: LocalizedOperatorBundle, device: Any, *,
                 upload: bool = True) -> None:
        torch = _torch()
        lib = native.library()
        ops = bundle.operators
        self.bundle = bundle
        self.n = bundle.n_orbitals
        offsets = np.ascontiguousarray(bundle.basis.atom_offsets, dtype=np.int64)
        rows = np.ascontiguousarray(ops.row_atom, dtype=np.int32)
        cols = np.ascontiguousarray(ops.col_atom, dtype=np.int32)
        shifts = np.ascontiguousarray(ops.lattice_shift, dtype=np.int32)
        boff = np.ascontiguousarray(ops.block_offsets, dtype=np.int64)
        handle = native.c_vp()
        with torch.cuda.device(device):
            native.call("aosb_bloch_create", self.n, bundle.basis.n_atoms, offsets.ctypes.data,
                        ops.n_blocks, rows.ctypes.data, cols.ctypes.data, shifts.ctypes.data,
                        boff.ctypes.data, native.C.byref(handle))
        self.handle = handle
        nnz, nsh = native.c_i64(), native.c_i64()
        lib.aosb_bloch_info(handle, native.C.byref(nnz), native.C.byref(nsh))
        self.nnz, self.n_shifts = int(nnz.value), int(nsh.value)
        self.indptr = np.empty(self.n + 1, dtype=np.int64)
        self.indices = np.empty(self.nnz, dtype=np.int32)
        self.shifts = np.empty((self.n_shifts, 3), dtype=np.int32)
        self.block_shift = np.empty(ops.n_blocks, dtype=np.int32)
        lib.aosb_bloch_export(handle, self.indptr.ctypes.data, self.indices.ctypes.data,
                              self.shifts.ctypes.data, self.block_shift.ctypes.data)
        complex_values = np.iscomplexobj(ops.h_values) or np.iscomplexobj(ops.s_values)
        self.value_kind = 1 if complex_values else 0
        self.device = device
        self.uploaded = False
        if upload:
            self.upload()

    def value_bytes(self) -> int:
        ops = self.bundle.operators
        item = 8 if self.value_kind else 4
        return int((np.asarray(ops.h_values).size + np.asarray(ops.s_values).size) * item)

    def upload(self) -> None:
        if self.uploaded:
            return
        torch = _torch()
        lib = native.library()
        with torch.cuda.device(self.device):
            native.call("aosb_bloch_upload", self.handle)
        dptr, dind = native.c_vp(), native.c_vp()
        lib.aosb_bloch_device_pattern(self.handle, native.C.byref(dptr), native.C.byref(dind))
        self.d_indptr, self.d_indices = int(dptr.value), int(dind.value)
        ops = self.bundle.operators
        dtype = np.complex64 if self.value_kind else np.float32
        hv = np.array(ops.h_values, dtype=dtype, copy=True)
        sv = np.array(ops.s_values, dtype=dtype, copy=True)
        tdt = torch.complex64 if self.value_kind else torch.float32
        self.h_values = torch.from_numpy(hv).to(device=self.device, dtype=tdt)
        self.s_values = torch.from_numpy(sv).to(device=self.device, dtype=tdt)
        self.uploaded = True

    def phases(self, kpoints: np.ndarray) -> np.ndarray:
        """exp(2 pi i R.k) per k and distinct shift, with the reference's
        complex64 arithmetic (sparse.py:207-213)."""
        out = np.empty((len(kpoints), self.n_shifts), dtype=np.complex64)
        r = self.shifts.astype(np.float32)
        for i, k in enumerate(kpoints):
            arg = r @ np.asarray(k, dtype=np.float32)
            out[i] = np.exp(np.asarray(2.0j * np.pi, dtype=np.complex64) * arg)
        return out

    def apply(self, kpoints: np.ndarray, stream: Any = None):
        """Device H(k), S(k) values [n_k, nnz] complex64."""
        torch = _torch()
        nk = len(kpoints)
        ph = torch.from_numpy(self.phases(kpoints)).to(self.device, non_blocking=False)
        h = torch.empty((nk, self.nnz), dtype=torch.complex64, device=self.device)
        s = torch.empty_like(h)
        st = torch.cuda.current_stream(self.device).cuda_stream if stream is None else stream
        native.call("aosb_bloch_apply", self.handle, self.value_kind, self.h_values.data_ptr(),
                    self.s_values.data_ptr(), ph.data_ptr(), nk, h.data_ptr(), s.data_ptr(), st)
        return h, s

    def close(self) -> None:
        if getattr(self, "handle", None):
            native.library().aosb_bloch_destroy(self.handle)
            self.handle = None


class SymbolicPlan:
    """Symbolic analysis of one CSR pattern (aosb_plan_create).

    ``ordering="auto"`` analyses the pattern with nested dissection and with
    the natural order and keeps the one with fewer factorization flops (for
    3D lattices whose interaction range is long compared with the cell,
    the banded natural order wins).  Creation is host-only; ``upload`` copies
    the tables to the device.
    """

    def __init__(self, n: int, indptr: np.ndarray, indices: np.ndarray, *, tile: int,
                 supervariables: np.ndarray | None = None, ordering: str = "auto",
                 device: Any = None, upload: bool = True) -> None:
        ip = np.ascontiguousarray(indptr, dtype=np.int64)
        ix = np.ascontiguousarray(indices, dtype=np.int32)
        sv = None if supervariables is None else np.ascontiguousarray(supervariables, np.int64)
        modes = {"nested_dissection": [1], "natural": [0], "auto": [1, 0]}[ordering]
        best = None
        for mode in modes:
            opts = native.PlanOptions(native.ABI_VERSION, native.C.sizeof(native.PlanOptions),
                                      tile, mode, 4 * tile, 1)
            handle = native.c_vp()
            native.call("aosb_plan_create", n, ip.ctypes.data, ix.ctypes.data,
                        None if sv is None else sv.ctypes.data,
                        0 if sv is None else sv.size - 1, native.C.byref(opts),
                        native.C.byref(handle))
            info = native.PlanInfo()
            native.library().aosb_plan_info(handle, native.C.byref(info))
            if best is None or info.factor_flops < best[1].factor_flops:
                if best is not None:
                    native.library().aosb_plan_destroy(best[0])
                best = (handle, info, mode)
            else:
                native.library().aosb_plan_destroy(handle)
        self.handle, info, mode = best
        self.ordering = "nested_dissection" if mode == 1 else "natural"
        self.info = PlanSummary(info.n, info.n_pad, info.nnz, info.tile, info.n_tiles,
                                info.n_slots, info.n_nodes, info.tree_levels, info.factor_flops,
                                info.factor_flops_alg, info.factor_bytes)
        self.device = device
        if upload:
            self.upload()

    def upload(self) -> None:
        torch = _torch()
        with torch.cuda.device(self.device):
            native.call("aosb_plan_upload", self.handle)

    def perm(self) -> np.ndarray:
        out = np.empty(self.info.n_pad, dtype=np.int32)
        native.library().aosb_plan_export_perm(self.handle, out.ctypes.data)
        return out

    def slots(self) -> np.ndarray:
        nb = self.info.n_tiles
        out = np.empty(nb * nb, dtype=np.int32)
        native.library().aosb_plan_export_slots(self.handle, out.ctypes.data)
        return out.reshape(nb, nb)

    def close(self) -> None:
        if getattr(self, "handle", None):
            native.library().aosb_plan_destroy(self.handle)
            self.handle = None


class CsrPattern:
    """A user CSR pattern on the device (for CISS on given H, S matrices)."""

    def __init__(self, n: int, indptr: np.ndarray, indices: np.ndarray, device: Any) -> None:
        torch = _torch()
        self.n = int(n)
        self.indptr = np.ascontiguousarray(indptr, dtype=np.int64)
        self.indices = np.ascontiguousarray(indices, dtype=np.int32)
        if self.indptr.shape != (self.n + 1,) or self.indptr[0] != 0 or \
                self.indptr[-1] != self.indices.size:
            raise InputError("CSR indptr endpoints are invalid")
        self.nnz = int(self.indices.size)
        self._ip = torch.from_numpy(self.indptr).to(device)
        self._ix = torch.from_numpy(self.indices).to(device)
        self.d_indptr, self.d_indices = self._ip.data_ptr(), self._ix.data_ptr()

    def close(self) -> None:
        self._ip = self._ix = None


@dataclass
class PencilWork:
    """One factorization: k row, shift, and the nodes it serves."""

    k: int
    node: int           # node solved with A = H - z S
    partner: int | None  # node solved with A^H (conjugate shift), if any


def pencil_schedule(n_k: int, shifts: np.ndarray, pair: bool) -> list[PencilWork]:
    """All (k, node) work items; with ``pair`` node j and node N-1-j share
    one factorization when z_{N-1-j} == conj(z_j)."""
    n = shifts.size
    items: list[PencilWork] = []
    for k in range(n_k):
        if pair:
            for j in range((n + 1) // 2):
                partner = n - 1 - j
                close = abs(complex(shifts[partner]) - complex(shifts[j]).conjugate())
                if partner != j and close <= 1e-5 * max(1.0, abs(complex(shifts[j]))):
                    items.append(PencilWork(k, j, partner))
                else:
                    items.append(PencilWork(k, j, None))
                    if partner != j:
                        items.append(PencilWork(k, partner, None))
        else:
            items.extend(PencilWork(k, j, None) for j in range(n))
    return items


class BundleResources:
    """Device state of one bundle that several engines (requests) can share:
    the Bloch tables with the resident block values, the CSR pattern, the
    symbolic plan and the row blocks.  Construction is host-only (pattern,
    analysis), so the footprint is known before any device memory is
    taken; ``upload`` moves everything to the device."""

    def __init__(self, bundle: LocalizedOperatorBundle, device: Any, *, tile: int,
                 ordering: str = "auto") -> None:
        torch = _torch()
        self.device = torch.device(device)
        self.bundle = bundle
        self.bloch = BlochDevice(bundle, self.device, upload=False)
        supervariables = np.asarray(bundle.basis.atom_offsets)
        self.plan = SymbolicPlan(self.bloch.n, self.bloch.indptr, self.bloch.indices, tile=tile,
                                 supervariables=supervariables, ordering=ordering,
                                 device=self.device, upload=False)
        self._rb = row_blocks(self.bloch.indptr, self.bloch.indices, starts=supervariables[:-1])
        self.max_block_rows = int(np.diff(self._rb).max())
        self.row_blocks = None
        self.uploaded = False

    def upload(self) -> None:
        if self.uploaded:
            return
        torch = _torch()
        self.bloch.upload()
        self.plan.upload()
        self.row_blocks = torch.from_numpy(self._rb).to(self.device)
        self.uploaded = True

    def resident_bytes(self) -> int:
        """Device bytes held while the bundle stays resident."""
        b = self.bloch
        pattern = 8 * (b.n + 1) + 4 * b.nnz
        info = self.plan.info
        plan = 4 * (3 * info.n_pad + 4 * info.n_tiles * info.n_tiles) + 4 * info.n_slots
        return int(b.value_bytes() + 2 * pattern + plan + 4 * self._rb.size)

    def close(self) -> None:
        self.bloch.close()
        self.plan.close()


class BandEngine:
    """Device-resident Band solver for one bundle."""

    def __init__(self, bundle: LocalizedOperatorBundle | None,
                 settings: CissSettings | None = None, engine: EngineSettings | None = None,
                 device: Any = None, *, csr: tuple[int, np.ndarray, np.ndarray] | None = None,
                 resources: BundleResources | None = None) -> None:
        torch = _torch()
        self.bundle = bundle
        self.settings = settings or CissSettings()
        self.engine = engine or EngineSettings()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else torch.device(device).index or 0)
        self._owns = resources is None
        if resources is not None:
            resources.upload()
            self.bundle = resources.bundle
            self.n = resources.bloch.n
            self.bloch = self.pattern = resources.bloch
            self.plan = resources.plan
            self.row_blocks = resources.row_blocks
            self.max_block_rows = resources.max_block_rows
            self.pattern_seconds = self.analysis_seconds = 0.0
            self.tuning = None
            if self.settings.search_dimension >= self.n:
                raise SolverError("CISS search dimension must be smaller than matrix dimension")
            self._init_buffers()
            return
        t0 = perf_counter()
        if bundle is not None:
            self.n = bundle.n_orbitals
            self.bloch = BlochDevice(bundle, self.device)
            self.pattern = self.bloch
            supervariables = np.asarray(bundle.basis.atom_offsets)
        else:
            if csr is None:
                raise InputError("BandEngine needs a bundle or a CSR pattern")
            self.n = int(csr[0])
            self.bloch = None
            self.pattern = CsrPattern(csr[0], csr[1], csr[2], self.device)
            supervariables = None
        if self.settings.search_dimension >= self.n:
            raise SolverError("CISS search dimension must be smaller than matrix dimension")
        self.pattern_seconds = perf_counter() - t0
        rb = row_blocks(self.pattern.indptr, self.pattern.indices,
                        starts=None if supervariables is None else supervariables[:-1])
        self.row_blocks = torch.from_numpy(rb).to(self.device)
        self.max_block_rows = int(np.diff(rb).max())
        t0 = perf_counter()
        use_tc = self.engine.precision == "mixed" and self.engine.tensor_cores
        tile = self.engine.tile or (128 if use_tc else choose_tile(self.n))
        self.tuning = None
        if self.engine.autotune and not self.engine.tile and self.bloch is not None:
            from .autotune import tune_plan

            h, s = self.bloch.apply(np.zeros((1, 3)))
            self.plan, self.tuning = tune_plan(
                self.n, self.pattern.indptr, self.pattern.indices, supervariables, h, s,
                precision=self.precision_id(), device=self.device)
            del h, s
        else:
            self.plan = SymbolicPlan(self.n, self.pattern.indptr, self.pattern.indices,
                                     tile=tile, supervariables=supervariables,
                                     ordering=self.engine.ordering, device=self.device)
        self.analysis_seconds = perf_counter() - t0
        self._init_buffers()

    def _init_buffers(self) -> None:
        torch = _torch()
        q = probe_block(self.n, self.settings)
        self.probes = torch.from_numpy(q.astype(np.complex128)).to(self.device)
        self._gram_scratch = None
        self._solve_scratch = None
        self._lapack_pool: ThreadPoolExecutor | None = None
        self.last_stats: dict[str, Any] = {}
        # optional device timing of every factorization call (CUDA events)
        self.profile_factor = False
        # with keep_vectors, the last call's selected Ritz vectors (device
        # complex128 [n][m] per k point, columns in the order of the
        # returned energies) and their FP64 energies are kept
        self.keep_vectors = False
        self.last_vectors: list[Any] = []
        self.last_energies: list[np.ndarray] = []
        self.factor_times_ms: list[float] = []
        self.factor_pencils: list[int] = []

    # ------------------------------------------------------------------ utils
    def precision_id(self) -> int:
        """The aosb_factor precision this engine's settings select."""
        if self.engine.precision == "mixed" and self.engine.tensor_cores:
            if not self.engine.tensor_core_panels:
                return native.PRECISION_BF16X3_FP32_PANELS
            return (native.PRECISION_BF16X3 if self.engine.schur_depth == 2
                    else native.PRECISION_BF16X3_ONE_STEP)
        return native.PRECISION_PLAIN

    def _stream(self):
        torch = _torch()
        return torch.cuda.current_stream(self.device).cuda_stream

    def _spmm(self, values, x, y) -> None:
        """y = A x for one k (values [nnz] complex64)."""
        n, m = x.shape
        native.call("aosb_spmm_blocks", n, m, self.row_blocks.numel() - 1,
                    self.row_blocks.data_ptr(), self.max_block_rows, self.pattern.d_indptr,
                    self.pattern.d_indices, values.data_ptr(), self.pattern.nnz, x.data_ptr(),
                    x.stride(0), y.data_ptr(), y.stride(0), self._stream())

    def _gram(self, x, y):
        """x^H y (p x q) in FP64 on the device."""
        torch = _torch()
        n, p = x.shape
        q = y.shape[1]
        need = native.library().aosb_gram_scratch_bytes(n, p, q)
        if self._gram_scratch is None or self._gram_scratch.numel() < need:
            self._gram_scratch = torch.empty(max(need, 16), dtype=torch.uint8, device=self.device)
        g = torch.empty((p, q), dtype=torch.complex128, device=self.device)
        native.call("aosb_gram", n, p, q, x.data_ptr(), x.stride(0), y.data_ptr(), y.stride(0),
                    g.data_ptr(), self._gram_scratch.data_ptr(), self._stream())
        return g

    def _dense_mul(self, x, t):
        torch = _torch()
        n, p = x.shape
        r = t.shape[1]
        t = t.contiguous()
        y = torch.empty((n, r), dtype=torch.complex128, device=self.device)
        native.call("aosb_dense_mul", n, p, r, x.data_ptr(), x.stride(0), t.data_ptr(),
                    y.data_ptr(), y.stride(0), self._stream())
        return y

    def pencil_bytes(self, n_rhs: int) -> int:
        info = self.plan.info
        lib = native.library()
        per = lib.aosb_factor_bytes(self.plan.handle, 1) + 4 * info.n_pad + 4
        per += 8 * info.n_pad * n_rhs * 2          # normal + adjoint solve blocks (complex64)
        per += 16 * self.n * n_rhs * 3             # x, r and adjoint x (complex128)
        per += lib.aosb_factor_workspace_bytes(self.plan.handle, 1, native.PRECISION_BF16X3)
        return int(per)

    def max_pencils(self, n_rhs: int) -> int:
        torch = _torch()
        if self.engine.max_pencils:
            return self.engine.max_pencils
        free, _ = torch.cuda.mem_get_info(self.device)
        # blocks the caching allocator holds but nobody uses are free for us
        free += torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        budget = int(free * self.engine.memory_fraction)
        return max(1, min(4096, budget // max(1, self.pencil_bytes(n_rhs))))

    # ------------------------------------------------------------- public API
    def load_values(self, h_values, s_values) -> None:
        """Replace the resident block values (same pattern) from host
        tensors/arrays; pinned host memory gives an asynchronous copy."""
        torch = _torch()
        for dst, src in ((self.bloch.h_values, h_values), (self.bloch.s_values, s_values)):
            t = src if isinstance(src, torch.Tensor) else torch.from_numpy(np.asarray(src))
            if t.numel() != dst.numel():
                raise InputError("block values do not match the bundle pattern")
            dst.copy_(t.reshape(dst.shape).to(dst.dtype), non_blocking=True)

    def host_pair(self, k: Sequence[float]) -> SparsePair:
        """H(k), S(k) as host scipy CSR (for user-supplied solvers)."""
        from scipy import sparse

        torch = _torch()
        kp = tuple(float(v) for v in k)
        if len(kp) != 3:
            raise InputError("k point must contain three values")
        h, s = self.bloch.apply(np.asarray([kp]))
        torch.cuda.current_stream(self.device).synchronize()
        hv, sv = h[0].cpu().numpy(), s[0].cpu().numpy()
        ip = self.bloch.indptr
        ix = self.bloch.indices
        if ip[-1] <= np.iinfo(np.int32).max:
            ip = ip.astype(np.int32)
        shape = (self.n, self.n)
        return SparsePair(sparse.csr_matrix((hv, ix, ip), shape=shape, copy=False),
                          sparse.csr_matrix((sv, ix, ip), shape=shape, copy=False), kp)

    def solve_values(self, h_values, s_values, interval: EnergyInterval) -> list[CissResult]:
        """CISS on given H, S value rows (complex64, [n_k, nnz] or [nnz]) of
        this engine's pattern; host arrays are uploaded."""
        torch = _torch()
        h = torch.as_tensor(np.asarray(h_values, dtype=np.complex64)).to(self.device)
        s = torch.as_tensor(np.asarray(s_values, dtype=np.complex64)).to(self.device)
        h = h.reshape(-1, self.pattern.nnz).contiguous()
        s = s.reshape(-1, self.pattern.nnz).contiguous()
        if h.shape != s.shape:
            raise InputError("H and S values differ in shape")
        with torch.cuda.device(self.device):
            torch.cuda.reset_peak_memory_stats(self.device)
            return self._ciss(h, s, interval, {}, perf_counter())

    def solve_kpoints(self, kpoints: Sequence[Sequence[float]], interval: EnergyInterval):
        """CISS for several k points; returns (results, assembly_seconds)."""
        torch = _torch()
        if len(kpoints) == 0:
            return [], []
        kp = np.asarray([[float(v) for v in k] for k in kpoints], dtype=np.float64)
        if kp.ndim != 2 or kp.shape[1] != 3:
            raise InputError("k point must contain three values")
        with torch.cuda.device(self.device):
            return self._solve(kp, interval)

    def _solve(self, kp: np.ndarray, interval: EnergyInterval):
        torch = _torch()
        dev = self.device
        torch.cuda.reset_peak_memory_stats(dev)
        t0 = perf_counter()
        hvals, svals = self.bloch.apply(kp)
        torch.cuda.current_stream(dev).synchronize()
        assembly = perf_counter() - t0
        results = self._ciss(hvals, svals, interval, {"bloch_assembly": assembly}, t0)
        return results, [assembly / kp.shape[0]] * kp.shape[0]

    def _ciss(self, hvals, svals, interval: EnergyInterval, stages: dict[str, float],
              total0: float) -> list[CissResult]:
        """CISS for the n_k value rows of (hvals, svals) on self.pattern."""
        torch = _torch()
        st = self.settings
        mixed = self.engine.precision == "mixed"
        n, L, M = self.n, st.block_size, st.moment_size
        nk = hvals.shape[0]
        dev = self.device

        def tick(name: str, t0: float) -> float:
            torch.cuda.current_stream(dev).synchronize()
            t1 = perf_counter()
            stages[name] = stages.get(name, 0.0) + (t1 - t0)
            return t1

        t = perf_counter()
        shifts, nodes, weights = contour_geometry(interval, st)
        coef = moment_coefficients(shifts, nodes, weights, M)
        rhs = torch.empty((nk, n, L), dtype=torch.complex128, device=dev)
        for k in range(nk):
            self._spmm(svals[k], self.probes, rhs[k])
        mom = torch.zeros((nk, n, L * M), dtype=torch.complex128, device=dev)
        t = tick("probe_setup", t)

        work = pencil_schedule(nk, shifts, pair=mixed)
        cap = min(self.max_pencils(L), len(work))
        # equal batches: 64 pencils under a cap of 48 run as 32 + 32, not 48 + 16
        n_batches = -(-len(work) // cap)
        cap = -(-len(work) // n_batches)
        info = self.plan.info
        lib = native.library()
        precision = self.precision_id()
        fbytes = lib.aosb_factor_bytes(self.plan.handle, cap)
        factor = torch.empty(fbytes // 4, dtype=torch.float32, device=dev)
        pivots = torch.empty((cap, info.n_pad), dtype=torch.int32, device=dev)
        status = torch.zeros(cap, dtype=torch.int32, device=dev)
        wbytes = lib.aosb_factor_workspace_bytes(self.plan.handle, cap, precision)
        workspace = torch.empty(max(wbytes, 16), dtype=torch.uint8, device=dev)
        wn = torch.empty((cap, info.n_pad, L), dtype=torch.complex64, device=dev)
        xn = torch.empty((cap, n, L), dtype=torch.complex128, device=dev)
        rr = torch.empty((cap, n, L), dtype=torch.complex128, device=dev)
        coef_d = torch.from_numpy(coef).to(dev)
        steps = self.engine.refinement_steps if mixed else 0
        n_factor = 0
        for b0 in range(0, len(work), cap):
            batch = work[b0:b0 + cap]
            np_ = len(batch)
            pk = torch.tensor([w.k for w in batch], dtype=torch.int32, device=dev)
            z = torch.from_numpy(shifts[[w.node for w in batch]].astype(np.complex128)).to(dev)
            status.zero_()
            fa = native.FactorArgs(native.ABI_VERSION, native.C.sizeof(native.FactorArgs), np_,
                                   precision, hvals.data_ptr(), svals.data_ptr(), pk.data_ptr(),
                                   z.data_ptr(), factor.data_ptr(), pivots.data_ptr(),
                                   status.data_ptr(), workspace.data_ptr(), self._stream())
            if self.profile_factor:
                ev0 = torch.cuda.Event(enable_timing=True)
                ev1 = torch.cuda.Event(enable_timing=True)
                ev0.record()
            native.call("aosb_factor", self.plan.handle, native.C.byref(fa))
            if self.profile_factor:
                ev1.record()
                ev1.synchronize()
                self.factor_times_ms.append(ev0.elapsed_time(ev1))
                self.factor_pencils.append(np_)
            n_factor += np_
            t = tick("native_numeric_factorization", t)
            bad = status[:np_].cpu().numpy()
            if np.any(bad != 0):
                code = int(bad[bad != 0][0])
                raise SolverError(f"shifted factorization failed with device status {code} "
                                  f"({native.STATUS_NAMES.get(code, 'unknown')})")
            # normal solves (node), then adjoint solves (conjugate partner);
            # a batch without partners skips the adjoint pass
            for adjoint in (0, 1):
                if adjoint and all(w.partner is None for w in batch):
                    continue
                zz = z if not adjoint else torch.conj_physical(z)
                self._solve_refined(batch, pk, zz, hvals, svals, rhs, factor, pivots, wn, xn,
                                    rr, adjoint, steps)
                t = tick("native_multi_rhs_solve", t)
                for i, w in enumerate(batch):
                    node = w.node if adjoint == 0 else w.partner
                    if node is None:
                        continue
                    native.call("aosb_moments_accumulate", n, L, M, xn[i].data_ptr(),
                                coef_d[node].data_ptr(), mom[w.k].data_ptr(), self._stream())
                t = tick("moment_accumulation", t)
        stages["shifted_solves"] = (stages.get("native_numeric_factorization", 0.0)
                                    + stages.get("native_multi_rhs_solve", 0.0)
                                    + stages.get("moment_accumulation", 0.0))
        del factor, pivots, wn, xn, rr, workspace
        results = self._subspace_batch(hvals, svals, mom, interval, stages, nk)
        peak = int(torch.cuda.max_memory_allocated(dev))
        total = perf_counter() - total0
        for res in results:
            res.stage_seconds["solver_total"] = total / nk
            res.peak_gpu_memory_bytes = peak
        self.last_stats = {"factorizations": n_factor, "pencil_batch": cap,
                           "stage_seconds": dict(stages)}
        return results

    def _solve_refined(self, batch, pk, z, hvals, svals, rhs, factor, pivots, wn, xn, rr,
                       adjoint: int, steps: int) -> None:
        """x = A^{-1} b (or A^{-H} b) for every pencil of the batch with
        ``steps`` FP64 refinement sweeps."""
        torch = _torch()
        n, L = self.n, self.settings.block_size
        np_ = len(batch)
        st = self._stream()
        # gather the rhs of each pencil's k into the pencil-major residual buffer
        kidx = torch.tensor([w.k for w in batch], dtype=torch.long, device=self.device)
        b = rhs.index_select(0, kidx).contiguous()
        need = native.library().aosb_solve_scratch_bytes(self.plan.handle, np_, L)
        if self._solve_scratch is None or self._solve_scratch.numel() < need:
            self._solve_scratch = torch.empty(max(need, 16), dtype=torch.uint8, device=self.device)
        mixed_tc = (self.engine.precision == "mixed" and self.engine.tensor_cores
                    and self.engine.tensor_core_solves and self.plan.info.tile == 128)
        flags = native.SOLVE_TENSOR_CORES if mixed_tc else 0
        if self.engine.cuda_graphs:
            flags |= native.SOLVE_GRAPH
        sa = native.SolveArgs(native.ABI_VERSION, native.C.sizeof(native.SolveArgs), np_, L,
                              adjoint, flags, factor.data_ptr(), pivots.data_ptr(), wn.data_ptr(),
                              self._solve_scratch.data_ptr(), st)
        for it in range(steps + 1):
            src = b if it == 0 else rr
            native.call("aosb_gather_rhs", self.plan.handle, np_, L, src.data_ptr(), n * L,
                        wn.data_ptr(), st)
            native.call("aosb_solve", self.plan.handle, native.C.byref(sa))
            native.call("aosb_scatter_solution", self.plan.handle, np_, L, wn.data_ptr(),
                        xn.data_ptr(), 1 if it > 0 else 0, st)
            if it < steps:
                self._residual(n, L, np_, hvals, svals, pk, z, b, xn, rr, st)
        if flags & native.SOLVE_TENSOR_CORES:
            native.call("aosb_solve_check", self.plan.handle, native.C.byref(sa))

    residual_kernel = "blocks"   # "blocks" (rows of one atom share x loads) or "rows"

    def _residual(self, n, L, np_, hvals, svals, pk, z, b, xn, rr, st) -> None:
        """FP64 r = b - (H - z S) x for every pencil of the batch."""
        if self.residual_kernel == "blocks":
            native.call("aosb_shifted_residual_blocks", n, L, np_, self.row_blocks.numel() - 1,
                        self.row_blocks.data_ptr(), self.max_block_rows, self.pattern.d_indptr,
                        self.pattern.d_indices, hvals.data_ptr(), svals.data_ptr(),
                        self.pattern.nnz, pk.data_ptr(), z.contiguous().data_ptr(),
                        b.data_ptr(), n * L, xn.data_ptr(), rr.data_ptr(), st)
        else:
            native.call("aosb_shifted_residual", n, L, np_, self.pattern.d_indptr,
                        self.pattern.d_indices, hvals.data_ptr(), svals.data_ptr(),
                        self.pattern.nnz, pk.data_ptr(), z.contiguous().data_ptr(),
                        b.data_ptr(), n * L, xn.data_ptr(), rr.data_ptr(), st)

    def _host_map(self, fn, items: list) -> list:
        """fn over items: the small FP64 eigenproblems of the batch's k points
        run in parallel threads, each on one BLAS thread (numpy and scipy
        release the GIL inside LAPACK)."""
        if len(items) <= 1:
            return [fn(x) for x in items]
        if self._lapack_pool is None:
            self._lapack_pool = ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1))
        with small_lapack():
            return list(self._lapack_pool.map(fn, items))

    def _subspace_batch(self, hvals, svals, mom, interval: EnergyInterval,
                        stages: dict[str, float], nk: int) -> list[CissResult]:
        """Rank truncation, Rayleigh-Ritz, ghost filter and residuals for the
        batch's k points, in lockstep: each phase enqueues the device work of
        every k point, reads the small results back once and solves the k
        points' host eigenproblems in parallel.  Per k point the arithmetic
        is that of the reference's solve_interval (ciss.py:320-372)."""
        torch = _torch()
        st = self.settings
        dev = self.device
        local = [{k: v / nk for k, v in stages.items()} for _ in range(nk)]
        # compression: G = M^H S M, truncation, B = M V / sqrt(lambda)
        t = perf_counter()
        grams = []
        for k in range(nk):
            sm = torch.empty_like(mom[k])
            self._spmm(svals[k], mom[k], sm)
            grams.append(self._gram(mom[k], sm))
        grams = torch.stack(grams).cpu().numpy()
        tol = st.rank_relative_tolerance
        trunc = self._host_map(lambda g: truncate_gram(g, tol, limit_threads=False), list(grams))
        basis = [self._dense_mul(mom[k], torch.from_numpy(trunc[k][0]).to(dev)) for k in range(nk)]
        torch.cuda.current_stream(dev).synchronize()
        dt = (perf_counter() - t) / nk
        for d in local:
            d["subspace_compression"] = dt
        # Rayleigh-Ritz: B^H H B, B^H S B, generalized eigh in FP64
        t = perf_counter()
        pairs = []
        for k in range(nk):
            hb = torch.empty_like(basis[k])
            sb = torch.empty_like(basis[k])
            self._spmm(hvals[k], basis[k], hb)
            self._spmm(svals[k], basis[k], sb)
            pairs.append((self._gram(basis[k], hb), self._gram(basis[k], sb)))
        pairs = [(hr.cpu().numpy(), sr.cpu().numpy()) for hr, sr in pairs]
        eig = self._host_map(lambda p: projected_eigh(p[0], p[1], limit_threads=False), pairs)
        dt = (perf_counter() - t) / nk
        for d in local:
            d["rayleigh_ritz"] = dt
        # ghost filter, interval selection, FP64 eigenpair residuals
        sel = []
        for k in range(nk):
            energies, coeffs = eig[k]
            keep = nonspurious_mask(coeffs, trunc[k][1], st.spurious_relative_threshold)
            inside = interval_mask(energies, interval)
            sel.append(np.flatnonzero(keep & inside))
        t = perf_counter()
        norms = [None] * nk
        self.last_vectors = [None] * nk if self.keep_vectors else []
        self.last_energies = [eig[k][0][sel[k]] for k in range(nk)] if self.keep_vectors else []
        for k in range(nk):
            if not sel[k].size:
                continue
            energies, coeffs = eig[k]
            csel = torch.from_numpy(np.ascontiguousarray(coeffs[:, sel[k]])).to(dev)
            vec = self._dense_mul(basis[k], csel)
            if self.keep_vectors:
                self.last_vectors[k] = vec
            hv = torch.empty_like(vec)
            sv = torch.empty_like(vec)
            self._spmm(hvals[k], vec, hv)
            self._spmm(svals[k], vec, sv)
            e_d = torch.from_numpy(np.ascontiguousarray(energies[sel[k]])).to(dev)
            norms[k] = torch.empty(sel[k].size, dtype=torch.float64, device=dev)
            native.call("aosb_column_norms", self.n, int(sel[k].size), hv.data_ptr(),
                        sv.data_ptr(), hv.stride(0), e_d.data_ptr(), norms[k].data_ptr(),
                        self._stream())
        max_res = [float(x.max().item()) if x is not None else 0.0 for x in norms]
        n_res = sum(1 for x in norms if x is not None)
        if n_res:
            dt = (perf_counter() - t) / n_res
            for k in range(nk):
                if norms[k] is not None:
                    local[k]["residual"] = dt
        results = []
        for k in range(nk):
            saturated = basis[k].shape[1] == st.search_dimension
            selected = np.asarray(eig[k][0][sel[k]], dtype=np.float32)
            results.append(CissResult(selected, max_res[k], local[k], None,
                                      result_warnings(max_res[k], saturated), not saturated))
        return results

    def close(self) -> None:
        if self._lapack_pool is not None:
            self._lapack_pool.shutdown(wait=True)
            self._lapack_pool = None
        if self._owns:
            self.pattern.close()
            self.plan.close()
