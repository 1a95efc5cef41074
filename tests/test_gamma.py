"""Gamma-point real symmetric shifted factorization with inertia (the
reference's cuDSS shift factor, native/src/aospectrum_cudss_shift_factor.c,
whose inertia drives its ordinal locator, src/aospectrum/primme.py:281-397).

CPU: the method -- Bunch-Kaufman inertia of a symmetric matrix, and its sum
over the Schur complements of the diagonal tiles of a block elimination --
against eigenvalue counts.  GPU: the library's aosb_shift_factor_* on the
64-atom sheet at Gamma against FP64 dense generalized eigenvalue counts at
several shifts, refactorization, and the solve against scipy."""

from __future__ import annotations

import numpy as np
import pytest

import bundles
from oracle import dense_ref, inertia_ref


def _counts(a, sigma=0.0):
    e = np.linalg.eigvalsh(a)
    return int(np.sum(e < sigma)), int(np.sum(e == sigma)), int(np.sum(e > sigma))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_bunch_kaufman_inertia_matches_eigenvalue_counts(seed):
    rng = np.random.default_rng(seed)
    for n in (1, 2, 7, 40):
        a = rng.standard_normal((n, n))
        a = a + a.T
        neg, zero, pos, _ = inertia_ref.bunch_kaufman_inertia(a)
        assert (neg, zero, pos) == _counts(a)
    # zero diagonal forces 2x2 pivots
    a = np.kron(np.eye(5), np.array([[0.0, 1.0], [1.0, 0.0]]))
    neg, zero, pos, swaps = inertia_ref.bunch_kaufman_inertia(a)
    assert (neg, zero, pos) == (5, 0, 5)
    # exactly singular: one zero count
    b = np.diag([1.0, -2.0, 0.0, 3.0])
    assert inertia_ref.bunch_kaufman_inertia(b)[:3] == (1, 1, 2)


@pytest.mark.parametrize("tile", [4, 8, 16])
def test_tiled_inertia_is_the_sum_over_diagonal_schur_complements(tile):
    """Haynsworth additivity: block elimination over diagonal tiles, as the
    device factorization does it, gives the inertia of the whole matrix
    (padding identity rows removed) -- here for shifted generalized pencils
    H - sigma S with S positive definite, counted against eig(H, S)."""
    from scipy import linalg

    rng = np.random.default_rng(tile)
    n = 45
    h = rng.standard_normal((n, n))
    h = h + h.T
    g = rng.standard_normal((n, n)) * 0.1
    s = np.eye(n) + g @ g.T
    e = linalg.eigh(h, s, eigvals_only=True)
    for sigma in (-3.0, 0.1, 2.5):
        neg, zero, pos = inertia_ref.tiled_inertia(h - sigma * s, tile)
        assert zero == 0
        assert neg == int(np.sum(e < sigma)) and pos == int(np.sum(e > sigma))


def _gamma_pair(b):
    from oracle import bloch_ref

    pat = bloch_ref.build_pattern(b)
    h, s = bloch_ref.bloch_pair(pat, b, (0.0, 0.0, 0.0))
    assert not np.any(np.imag(h)) and not np.any(np.imag(s))
    return pat, np.real(h).astype(np.float32), np.real(s).astype(np.float32)


@pytest.mark.gpu
def test_gamma_shift_factor_inertia_matches_fp64_counts():
    import torch

    from aospectrum_b200.gamma import GammaShiftFactor

    torch.cuda.set_device(0)
    b = bundles.c1()
    pat, h, s = _gamma_pair(b)
    n = b.n_orbitals
    hd, sd = dense_ref.dense_pair(pat.indptr, pat.indices, h.astype(np.complex64),
                                  s.astype(np.complex64), n)
    exact = np.sort(dense_ref.eigenvalues(hd, sd))
    # shifts midway between neighbouring FP64 eigenvalues (well away from both)
    picks = [n // 5, n // 2, (4 * n) // 5]
    shifts = [0.5 * (exact[i - 1] + exact[i]) for i in picks]
    dev = torch.device("cuda", 0)
    hv = torch.from_numpy(h).to(dev)
    sv = torch.from_numpy(s).to(dev)
    f = GammaShiftFactor(n, pat.indptr, pat.indices, hv, sv, shifts[0], maximum_rhs=4)
    try:
        for i, sigma in zip(picks, shifts):
            up = f.update_numeric(sigma) if sigma != shifts[0] else f.last
            assert up.inertia.below == i, (sigma, up.inertia)
            assert up.inertia.zero == 0 and up.inertia.above == n - i
            assert up.inertia.dimension == n and up.inertia.energy_ev == pytest.approx(sigma)
        st = f.stats()
        assert st["upper_nnz"] == (pat.indices.size + n) // 2
        assert st["factor_nnz"] > 0
        # solve against scipy (FP64) at the last shift: backward error of the
        # FP32 factorization without refinement
        from scipy import sparse
        from scipy.sparse import linalg as splinalg

        a = (sparse.csr_matrix((h.astype(np.float64), pat.indices, pat.indptr), shape=(n, n))
             - shifts[-1] * sparse.csr_matrix((s.astype(np.float64), pat.indices, pat.indptr),
                                              shape=(n, n)))
        rng = np.random.default_rng(3)
        rhs = rng.standard_normal((n, 3)).astype(np.float32)
        x = f.solve(torch.from_numpy(rhs).to(dev)).cpu().numpy().astype(np.float64)
        ref = splinalg.spsolve(a.tocsc(), rhs.astype(np.float64))
        res = np.linalg.norm(rhs - a @ x, axis=0)
        scale = splinalg.norm(a, 1) * np.linalg.norm(x, axis=0)
        assert np.max(res / scale) < 1e-5
        rel = np.linalg.norm(x - ref) / np.linalg.norm(ref)
        assert rel < 1e-3, rel
        assert f.stats()["solve_calls"] == 1 and f.stats()["solved_rhs"] == 3
    finally:
        f.close()


@pytest.mark.gpu
def test_gamma_shift_factor_from_bundle_and_errors():
    import torch

    from aospectrum_b200.errors import InputError, SolverError
    from aospectrum_b200.gamma import GammaShiftFactor

    torch.cuda.set_device(0)
    b = bundles.small2d()
    pat, h, s = _gamma_pair(b)
    hd, sd = dense_ref.dense_pair(pat.indptr, pat.indices, h.astype(np.complex64),
                                  s.astype(np.complex64), b.n_orbitals)
    exact = np.sort(dense_ref.eigenvalues(hd, sd))
    sigma = 0.5 * (exact[99] + exact[100])
    with GammaShiftFactor.from_bundle(b, sigma) as f:
        assert f.inertia.below == 100 and f.inertia.zero == 0
        with pytest.raises(InputError):
            f.solve(np.zeros((b.n_orbitals, 9), np.float32))    # more than maximum_rhs
    with pytest.raises(SolverError, match="status"):
        GammaShiftFactor(3, np.array([0, 1, 2, 3]), np.array([0, 1, 1]), np.ones(3),
                         np.ones(3), 0.0)   # row 2 has no diagonal entry
