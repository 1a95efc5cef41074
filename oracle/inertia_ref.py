"""numpy restatement of the Gamma-point inertia count -- test oracle only.

The reference reads the inertia of H - sigma S from cuDSS's symmetric
factorization (native/src/aospectrum_cudss_shift_factor.c:232-329) and its
ordinal locator compares the count of states below sigma with the requested
state numbers (src/aospectrum/primme.py:281-397).  The library computes it
tile by tile: symmetric block elimination over T-wide diagonal tiles, and a
Bunch-Kaufman LDL^T (partial pivoting, alpha = (1 + sqrt(17)) / 8; Bunch and
Kaufman, Math. Comp. 31 (1977)) of each eliminated diagonal tile, summed
(Haynsworth inertia additivity of Schur complements).  These functions do
the same in FP64 on the host so the tests can check the method against
eigenvalue counts.
"""

from __future__ import annotations

import math

import numpy as np

ALPHA = (1.0 + math.sqrt(17.0)) / 8.0


def bunch_kaufman_inertia(a: np.ndarray) -> tuple[int, int, int, int]:
    """(negative, zero, positive, interchanges) of a symmetric matrix from
    its Bunch-Kaufman LDL^T."""
    a = np.array(a, dtype=np.float64, copy=True)
    n = a.shape[0]
    neg = zero = pos = swaps = 0
    j = 0
    while j < n:
        col = np.abs(a[j + 1:, j])
        lam = float(col.max()) if col.size else 0.0
        r = j + 1 + int(np.argmax(col)) if col.size else j
        ajj = abs(a[j, j])
        kind, frm, to = 1, -1, -1
        if lam <= 0.0 and ajj == 0.0:
            kind = 0
        elif ajj >= ALPHA * lam:
            kind = 1
        else:
            row = np.abs(a[r, j:])
            row[r - j] = -1.0
            sig = float(row.max())
            if ajj * sig >= ALPHA * lam * lam:
                kind = 1
            elif abs(a[r, r]) >= ALPHA * sig:
                kind, frm, to = 1, j, r
            else:
                kind, frm, to = 2, j + 1, r
        if frm >= 0 and frm != to:
            swaps += 1
            a[[frm, to], j:] = a[[to, frm], j:]
            a[j:, [frm, to]] = a[j:, [to, frm]]
        if kind == 0:
            zero += 1
            j += 1
        elif kind == 1:
            d = a[j, j]
            neg += d < 0
            pos += d > 0
            zero += d == 0
            if d != 0:
                a[j + 1:, j + 1:] -= np.outer(a[j + 1:, j], a[j, j + 1:]) / d
            j += 1
        else:
            dblk = a[j:j + 2, j:j + 2]
            det = float(np.linalg.det(dblk))
            tr = float(np.trace(dblk))
            if det < 0:
                neg += 1
                pos += 1
            elif det > 0:
                if tr > 0:
                    pos += 2
                else:
                    neg += 2
            else:
                zero += 1
                pos += tr > 0
                neg += tr < 0
                zero += tr == 0
            if det != 0:
                c = a[j + 2:, j:j + 2]
                a[j + 2:, j + 2:] -= c @ np.linalg.solve(dblk, a[j:j + 2, j + 2:])
            j += 2
    return int(neg), int(zero), int(pos), int(swaps)


def tiled_inertia(a: np.ndarray, tile: int) -> tuple[int, int, int]:
    """Inertia of symmetric ``a`` by block elimination over ``tile``-wide
    diagonal blocks (padding the last block with identity rows, removed from
    the positive count): the sum of the Bunch-Kaufman inertias of the Schur
    complements of the diagonal blocks."""
    n = a.shape[0]
    npad = -(-n // tile) * tile
    m = np.eye(npad)
    m[:n, :n] = a
    neg = zero = pos = 0
    for k0 in range(0, npad, tile):
        k1 = k0 + tile
        skk = m[k0:k1, k0:k1]
        dn, dz, dp, _ = bunch_kaufman_inertia(skk)
        neg, zero, pos = neg + dn, zero + dz, pos + dp
        if k1 < npad:
            m[k1:, k1:] -= m[k1:, k0:k1] @ np.linalg.solve(skk, m[k0:k1, k1:])
    return neg, zero, pos - (npad - n)
