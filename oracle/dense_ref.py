"""FP64 dense generalized eigenvalue oracle -- test infrastructure only.

Solves H(k) c = E S(k) c with the supplied overlap (never the identity),
through a Cholesky factor of S, for small systems.
"""

from __future__ import annotations

import numpy as np
from scipy import linalg


def dense_pair(indptr, indices, h, s, n):
    hd = np.zeros((n, n), dtype=np.complex128)
    sd = np.zeros((n, n), dtype=np.complex128)
    rows = np.repeat(np.arange(n), np.diff(indptr))
    hd[rows, indices] = h
    sd[rows, indices] = s
    return hd, sd


def eigenvalues(hd: np.ndarray, sd: np.ndarray) -> np.ndarray:
    hh = 0.5 * (hd + hd.conj().T)
    ss = 0.5 * (sd + sd.conj().T)
    return linalg.eigh(hh, ss, eigvals_only=True)


def window(e: np.ndarray, lo: float, hi: float) -> np.ndarray:
    return np.sort(e[(e > lo) & (e < hi)])
