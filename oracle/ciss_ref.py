"""numpy/scipy restatement of the reference CISS interval solver -- test
oracle and CPU baseline only.

Follows src/aospectrum/ciss.py of yumiaoyi-o/AOSpectrum:
  contour       _contour_geometry   ciss.py:81-104
  probes        solve_interval      ciss.py:284-295
  moments       solve_interval      ciss.py:296-333
  compression   _compress_moments   ciss.py:107-126
  Rayleigh-Ritz _rayleigh_ritz      ciss.py:129-150
  ghost filter  _nonspurious_mask   ciss.py:153-177
  selection + residual              ciss.py:350-372
all in the reference's complex64 arithmetic.  The shifted solves, which
the reference sends to cuDSS (general complex64 LU with two refinement
steps), are done here on the host cores by LAPACK: ``dense`` factors each
complex64 pencil with cgetrf; ``splu`` uses scipy's SuperLU in complex128
(closest to exact solves).  BandEngine-independent.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
from scipy import linalg, sparse
from scipy.sparse import linalg as splinalg


@dataclass
class RefCissResult:
    energies: np.ndarray
    max_residual: float
    saturated: bool
    rank: int


def contour(lower: float, upper: float, n_points: int = 32, scale: float = 0.1,
            guard: float = 1.0e-5):
    # Python floats, as the reference's EnergyInterval stores them (numpy
    # float64 scalars would change the float32/complex64 promotion below).
    lower, upper = float(lower), float(upper)
    lo = lower - 2.0 * guard
    hi = upper + 2.0 * guard
    centre = 0.5 * (lo + hi)
    rx = 0.5 * (hi - lo)
    ry = rx * scale
    idx = np.arange(n_points, dtype=np.float32)
    theta = 2.0 * np.pi * (idx + 0.5) / n_points
    nodes = np.cos(theta) + (1j * scale * np.sin(theta))
    shifts = centre + rx * nodes
    weights = (ry * np.cos(theta) + 1j * rx * np.sin(theta)) / n_points
    return (np.asarray(shifts, dtype=np.complex64), np.asarray(nodes, dtype=np.complex64),
            np.asarray(weights, dtype=np.complex64))


def probes(n: int, block: int, seed: int = 20260727) -> np.ndarray:
    rng = np.random.default_rng(seed)
    a = (rng.standard_normal((n, block), dtype=np.float32)
         + 1j * rng.standard_normal((n, block), dtype=np.float32))
    a = np.asarray(a / np.asarray(math.sqrt(2.0), dtype=np.float32), dtype=np.complex64)
    q, _ = np.linalg.qr(a, mode="reduced")
    return q


def shifted_solve(h: sparse.csr_matrix, s: sparse.csr_matrix, z, rhs: np.ndarray,
                  method: str = "splu") -> np.ndarray:
    if method == "splu":
        a = (h.astype(np.complex128) - complex(z) * s.astype(np.complex128)).tocsc()
        return splinalg.splu(a).solve(rhs.astype(np.complex128)).astype(np.complex64)
    a = (h - np.complex64(z) * s).toarray().astype(np.complex64)
    lu = linalg.lu_factor(a, check_finite=False)
    return linalg.lu_solve(lu, rhs, check_finite=False).astype(np.complex64)


def solve_interval(h: sparse.csr_matrix, s: sparse.csr_matrix, lower: float, upper: float, *,
                   n_points: int = 32, block: int = 32, moments: int = 4,
                   method: str = "splu", rank_tol: float = 1.0e-5,
                   ghost_tol: float = 1.0e-4, seed: int = 20260727) -> RefCissResult:
    n = h.shape[0]
    shifts, nodes, weights = contour(lower, upper, n_points)
    q = probes(n, block, seed)
    rhs = np.asarray(s @ q, dtype=np.complex64)
    mom = np.zeros((n, block * moments), dtype=np.complex64)
    for j in range(n_points):
        x = shifted_solve(h, s, shifts[j], rhs, method)
        accumulate_moments(mom, x, weights[j], nodes[j], block, moments)
    return subspace(h, s, mom, lower, upper, block=block, moments=moments, rank_tol=rank_tol,
                    ghost_tol=ghost_tol)


def accumulate_moments(mom: np.ndarray, x: np.ndarray, weight, node, block: int,
                       moments: int) -> None:
    """mom[:, m L:(m+1) L] += -w_j zeta_j^m X_j in complex64 (ciss.py:324-333)."""
    for m in range(moments):
        mom[:, m * block:(m + 1) * block] += -weight * node ** m * x


def subspace(h: sparse.csr_matrix, s: sparse.csr_matrix, mom: np.ndarray, lower: float,
             upper: float, *, block: int, moments: int, rank_tol: float = 1.0e-5,
             ghost_tol: float = 1.0e-4) -> RefCissResult:
    """Compression, Rayleigh-Ritz, ghost filter, selection and residuals of
    the moment block (ciss.py:107-177, :334-372)."""
    gram = mom.conj().T @ (s @ mom)
    gram = 0.5 * (gram + gram.conj().T)
    lam, vec = np.linalg.eigh(gram)
    scale = float(np.max(np.abs(lam), initial=0.0))
    keep = lam > scale * rank_tol
    pos = lam[keep]
    basis = np.asarray(mom @ (vec[:, keep] / np.sqrt(pos)[None, :]), dtype=np.complex64)
    sigma = np.sqrt(pos)
    hr = basis.conj().T @ (h @ basis)
    sr = basis.conj().T @ (s @ basis)
    hr = 0.5 * (hr + hr.conj().T)
    sr = 0.5 * (sr + sr.conj().T)
    e, c = linalg.eigh(hr, sr, check_finite=False, driver="gvd")
    e = np.asarray(e, dtype=np.float32)
    v = np.asarray(basis @ c, dtype=np.complex64)
    c = np.asarray(c, dtype=np.complex64)
    amp = np.abs(c) ** 2
    num, den = amp.sum(axis=0), (amp / sigma[:, None]).sum(axis=0)
    score = np.divide(num, den, out=np.zeros(num.shape, dtype=num.dtype), where=den > 0.0)
    good = np.isfinite(score) & (score >= ghost_tol * float(np.max(score, initial=0.0)))
    sel = good & (e > lower) & (e < upper)
    es, vs = e[sel], v[:, sel]
    if es.size:
        res = h @ vs - (s @ vs) * es[None, :]
        maxres = float(np.max(np.linalg.norm(res, axis=0)))
    else:
        maxres = 0.0
    return RefCissResult(es, maxres, int(keep.sum()) == block * moments, int(keep.sum()))
