"""CISS (contour-integral Sakurai-Sugiura) settings, contour and the small
projected problems.

``CissSettings`` keeps exactly the nine fields of the reference
(``src/aospectrum/ciss.py:35-62``) so ``run.json`` specifications stay
comparable; engine-only knobs live in ``EngineSettings``.  The contour
geometry and the probe block are computed on the host with the same numpy
operations as the reference (``ciss.py:81-104`` and ``:284-295``), so the
shifts, weights and probes are bit-identical.  The small projected problems
(rank truncation, Rayleigh-Ritz, ghost filter; ``ciss.py:107-177``) are
solved in FP64 on the host from FP64 device products.
"""

from __future__ import annotations

import contextlib
import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from .data import EnergyInterval
from .errors import InputError, SolverError


@dataclass(slots=True)
class CissResult:
    energies_ev: np.ndarray
    maximum_residual_ev: float
    stage_seconds: dict[str, float]
    peak_gpu_memory_bytes: int | None
    warnings: tuple[str, ...]
    complete: bool


@dataclass(slots=True)
class ShiftedResult:
    solutions: np.ndarray
    stage_seconds: dict[str, float]
    peak_gpu_memory_bytes: int | None


@dataclass(frozen=True, slots=True)
class CissSettings:
    integration_points: int = 32
    contour_batch_size: int = 1
    block_size: int = 32
    moment_size: int = 4
    ellipse_vertical_scale: float = 0.1
    endpoint_guard_ev: float = 1.0e-5
    rank_relative_tolerance: float = 1.0e-5
    spurious_relative_threshold: float = 1.0e-4
    random_seed: int = 20260727

    def __post_init__(self) -> None:
        sizes_ok = (
            self.integration_points >= 1
            and self.contour_batch_size >= 1
            and self.integration_points % self.contour_batch_size == 0
            and self.block_size >= 1
            and self.moment_size >= 1
        )
        if not sizes_ok:
            raise InputError("CISS sizes must be positive and contour_batch_size "
                             "must divide integration_points")

    @property
    def search_dimension(self) -> int:
        return self.block_size * self.moment_size


PRECISIONS = ("mixed", "plain")


@dataclass(frozen=True, slots=True)
class EngineSettings:
    """Knobs of the GPU engine (no counterpart in the reference).

    precision: "mixed" = split-BF16 tensor-core tile updates, FP32 panels,
        FP64 iterative refinement, conjugate node pairs share one
        factorization; "plain" = complex64 FP32 updates, one factorization
        per node, no refinement (the drop-in baseline).
    refinement_steps: FP64 refinement sweeps of every mixed solve.
    tile: tile edge (32, 64, 128) or 0 to let the autotuner choose.
    max_pencils: cap on pencils factored together (0 = by memory).
    memory_fraction: share of free device memory the pencil pool may use.
    ordering: "auto" (fewest factorization flops), "nested_dissection" or
        "natural".
    tensor_cores: with precision "mixed", False keeps the FP32 SIMT tile
        updates (FP32 factor + FP64 refinement + node pairing).
    tensor_core_panels: with tensor cores, also form the panel tiles
        L_ik = A_ik inv(U_kk) and U_kj = inv(L_kk) P_k A_kj in split BF16;
        False keeps them in FP32 SIMT.
    tensor_core_solves: with tensor cores, run the off-diagonal tile
        updates of the triangular sweeps in split BF16 too (FP64
        refinement recovers the accuracy); False keeps them in FP32 SIMT.
    schur_depth: 2 applies the Schur updates of two tile steps in one
        tensor-core pass (K = 256: each target tile read and written once per
        two steps); 1 updates after every step.
    cuda_graphs: capture each batch's triangular sweeps (hundreds of
        launches per solve) into a CUDA graph on first use and replay it.
    autotune: with tile 0, time the candidate tile plans (tile edge x
        ordering) on the device for this pattern and keep the fastest
        (aospectrum_b200.autotune); False picks by size and flop count.
    """

    precision: str = "mixed"
    refinement_steps: int = 1
    tile: int = 0
    max_pencils: int = 0
    memory_fraction: float = 0.6
    ordering: str = "auto"
    tensor_cores: bool = True
    tensor_core_panels: bool = True
    tensor_core_solves: bool = True
    autotune: bool = False
    schur_depth: int = 2
    cuda_graphs: bool = False

    def __post_init__(self) -> None:
        if self.precision not in PRECISIONS:
            raise InputError(f"precision must be one of {PRECISIONS}")
        if self.tile not in (0, 32, 64, 128):
            raise InputError("tile must be 0, 32, 64 or 128")
        if self.refinement_steps < 0 or self.max_pencils < 0:
            raise InputError("refinement_steps and max_pencils must be >= 0")
        if not 0.0 < self.memory_fraction <= 0.95:
            raise InputError("memory_fraction must be in (0, 0.95]")
        if self.schur_depth not in (1, 2):
            raise InputError("schur_depth must be 1 or 2")
        if self.ordering not in ("auto", "nested_dissection", "natural"):
            raise InputError("ordering must be auto, nested_dissection or natural")


def contour_geometry(interval: EnergyInterval, settings: CissSettings):
    """Shifts z_j, normalised nodes zeta_j and weights w_j (complex64) of the
    ellipse around the interval; the same float32/complex64 arithmetic as
    the reference (ciss.py:81-104)."""
    lo = interval.lower_ev - 2.0 * settings.endpoint_guard_ev
    hi = interval.upper_ev + 2.0 * settings.endpoint_guard_ev
    centre = 0.5 * (lo + hi)
    rx = 0.5 * (hi - lo)
    ry = rx * settings.ellipse_vertical_scale
    n = settings.integration_points
    theta = 2.0 * np.pi * (np.arange(n, dtype=np.float32) + 0.5) / n
    nodes = np.cos(theta) + (1j * settings.ellipse_vertical_scale * np.sin(theta))
    shifts = centre + rx * nodes
    weights = (ry * np.cos(theta) + 1j * rx * np.sin(theta)) / n
    return (np.asarray(shifts, dtype=np.complex64), np.asarray(nodes, dtype=np.complex64),
            np.asarray(weights, dtype=np.complex64))


def probe_block(n: int, settings: CissSettings) -> np.ndarray:
    """Orthonormal complex64 probe block Q (n x L) from the seeded generator,
    drawn and orthonormalised with the reference's numpy calls
    (ciss.py:284-295)."""
    rng = np.random.default_rng(settings.random_seed)
    shape = (n, settings.block_size)
    raw = (rng.standard_normal(shape, dtype=np.float32)
           + 1j * rng.standard_normal(shape, dtype=np.float32))
    raw = np.asarray(raw / np.asarray(math.sqrt(2.0), dtype=np.float32), dtype=np.complex64)
    q, _ = np.linalg.qr(raw, mode="reduced")
    return q


def moment_coefficients(shifts: np.ndarray, nodes: np.ndarray, weights: np.ndarray,
                        moments: int) -> np.ndarray:
    """c[j, m] = -w_j zeta_j^m as complex128 (the reference forms the same
    products in complex64, ciss.py:324-333)."""
    w = weights.astype(np.complex128)
    z = nodes.astype(np.complex128)
    return np.stack([-w * z ** m for m in range(moments)], axis=1)


def hermitize(a: np.ndarray) -> np.ndarray:
    return 0.5 * (a + a.conj().T)


def small_lapack():
    """Context that runs host LAPACK on one thread.  The projected problems
    are at most a few hundred wide; on hosts with many cores a BLAS pool
    sized to the machine spends far longer waking and synchronising its
    threads than the factorization itself takes."""
    from threadpoolctl import threadpool_limits

    return threadpool_limits(limits=1)


def truncate_gram(gram: np.ndarray, tolerance: float, *,
                  limit_threads: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """Rank truncation of the S-Gram matrix of the moments (reference
    ``_compress_moments``, ciss.py:107-126): returns the transform
    V_keep / sqrt(lambda) and the singular values sqrt(lambda).
    ``limit_threads=False`` leaves the BLAS thread limit to the caller (a
    caller running several of these in threads sets it once around them)."""
    with small_lapack() if limit_threads else contextlib.nullcontext():
        values, vectors = np.linalg.eigh(hermitize(gram))
    scale = float(np.max(np.abs(values), initial=0.0))
    if scale == 0.0 or not math.isfinite(scale):
        raise SolverError("CISS contour moments have zero numerical rank")
    keep = values > scale * tolerance
    if not np.any(keep):
        raise SolverError("CISS contour moments have no positive stable subspace")
    lam = values[keep]
    return vectors[:, keep] / np.sqrt(lam)[None, :], np.sqrt(lam)


def projected_eigh(hr: np.ndarray, sr: np.ndarray, *,
                   limit_threads: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """Generalized Hermitian eigenproblem of the projected pencil (reference
    ``_rayleigh_ritz``, ciss.py:129-150), solved in FP64."""
    from scipy import linalg

    try:
        with small_lapack() if limit_threads else contextlib.nullcontext():
            e, c = linalg.eigh(hermitize(hr), hermitize(sr), check_finite=False, driver="gvd")
    except linalg.LinAlgError as exc:
        raise SolverError("CISS reduced overlap is not positive definite") from exc
    return e, c


def nonspurious_mask(coefficients: np.ndarray, singular_values: np.ndarray,
                     threshold: float) -> np.ndarray:
    """Ghost filter (reference ``_nonspurious_mask``, ciss.py:153-177)."""
    amp = np.abs(coefficients) ** 2
    num = amp.sum(axis=0)
    den = (amp / singular_values[:, None]).sum(axis=0)
    scores = np.divide(num, den, out=np.zeros(num.shape, dtype=num.dtype), where=den > 0.0)
    top = float(np.max(scores, initial=0.0))
    if top == 0.0 or not math.isfinite(top):
        raise SolverError("CISS ghost filter produced no positive finite score")
    return np.isfinite(scores) & (scores >= threshold * top)


def interval_mask(energies: np.ndarray, interval: EnergyInterval) -> np.ndarray:
    """Strict interval test on the energies as the reference emits them:
    cast to float32 first (``_rayleigh_ritz`` returns float32 energies,
    ciss.py:145-150) and compared with the bounds as numpy compares a
    float32 array with Python floats (ciss.py:355-358).  An FP64 energy a
    float32 ulp inside a bound that rounds onto it is therefore dropped, as
    the reference drops it."""
    e32 = np.asarray(energies, dtype=np.float32)
    return (e32 > interval.lower_ev) & (e32 < interval.upper_ev)


def result_warnings(max_residual: float, saturated: bool) -> tuple[str, ...]:
    out = []
    if max_residual > 1.0e-3:
        out.append(f"maximum eigenpair residual is {max_residual:.3e} eV")
    if saturated:
        out.append("CISS search subspace is saturated; the returned interval "
                   "spectrum may be incomplete")
    return tuple(out)


def require_shared_pattern(matrices: Any) -> None:
    """CSR H and S on one pattern, complex64 (reference ciss.py:65-78)."""
    from scipy import sparse

    h, s = matrices.hamiltonian, matrices.overlap
    if not (sparse.issparse(h) and h.format == "csr" and sparse.issparse(s) and s.format == "csr"):
        raise InputError("CISS requires CSR H and S")
    if not (np.array_equal(h.indptr, s.indptr) and np.array_equal(h.indices, s.indices)):
        raise InputError("CISS requires one shared H/S CSR pattern")
    if h.dtype != np.complex64 or s.dtype != np.complex64:
        raise InputError("CISS requires complex64 H/S")


@dataclass
class StageClock:
    """Accumulates named stage durations (seconds)."""

    seconds: dict[str, float] = field(default_factory=dict)

    def add(self, name: str, value: float) -> None:
        self.seconds[name] = self.seconds.get(name, 0.0) + float(value)
