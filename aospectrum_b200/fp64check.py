"""FP64 check of CISS eigenvalues where a dense FP64 eigensolver does not fit.

At n = 53,248 (the 4096-atom cubic bundle) or n = 260,000 (the 20,000-atom
slab) a dense FP64 generalized eigensolve of H(k), S(k) needs tens to
hundreds of GB and hours; a sparse complex128 LU on the host needs hours per
shift.  This check refines the engine's own eigenpairs instead, with solves
whose accuracy is measured, and bounds what is left:

1. the engine's eigenpairs (E_i, v_i) in the interval (mixed precision);
2. one shift-invert step per eigenpair: x_i = (H - s S)^{-1} S v_i with a
   complex shift s = c + i eta near E_i (shifts are shared by the
   eigenvalues within eta of a centre c), each solve iteratively refined
   in FP64 until ||b - (H - s S) x|| <= tol ||b|| for every right-hand
   side (the sweep count and the reached tolerance are reported);
3. a Rayleigh-Ritz step in FP64 on span[V, X]: refined pairs (E'_i, v'_i)
   and their FP64 residuals r_i = H v'_i - E'_i S v'_i.

Only converged refined pairs are compared (residual at most 1e-3 eV, or
twice the engine's own largest residual): the enriched space also yields
Ritz values that approximate no eigenpair.  Reported per k point: the
engine's values paired one to one with the converged refined values
(minimum total distance), max |E_i - E'_i| over the pairs -- the eigenvalue
error of the engine's values as far as the refined ones resolve it -- the
count difference, and the residual /
gap estimate ||r_i||^2 / gap_i of the refined values' own error (gap_i: the
distance from E'_i to the nearest other Ritz value of the enriched space),
the Kato-Temple form of the a-posteriori bound for Hermitian pencils with
the Euclidean residual norm.
"""

from __future__ import annotations

from typing import Any, Sequence

import numpy as np

from . import native
from .ciss import hermitize, projected_eigh
from .data import EnergyInterval
from .errors import SolverError


def shift_centres(energies: np.ndarray, eta: float) -> list[tuple[float, list[int]]]:
    """Greedy cover of the sorted energies by centres: every energy lies
    within eta of its centre; returns (centre, indices) pairs."""
    order = np.argsort(energies)
    out: list[tuple[float, list[int]]] = []
    i = 0
    while i < order.size:
        first = float(energies[order[i]])
        members = [int(order[i])]
        j = i + 1
        while j < order.size and float(energies[order[j]]) - first <= 2.0 * eta:
            members.append(int(order[j]))
            j += 1
        centre = 0.5 * (first + float(energies[order[j - 1]]))
        out.append((centre, members))
        i = j
    return out


def compare_refined(energies: np.ndarray, refined: np.ndarray, residuals: np.ndarray,
                    engine_residual: float) -> tuple[np.ndarray, float | None, int]:
    """Which refined pairs count, and the engine's error against them.

    Only converged refined pairs count: the enriched space also yields Ritz
    values that approximate no eigenpair (their residuals are of the order
    of the interval width).  Converged: residual at most 1e-3 eV (the
    reference's warning level) or twice the engine's own largest residual.
    The engine's values are paired one to one with the converged refined
    values at the least total distance; returns (converged mask, max
    distance over the pairs or None, number of pairs)."""
    conv = np.asarray(residuals) <= max(1e-3, 2.0 * engine_residual)
    ref_conv = np.asarray(refined)[conv]
    energies = np.asarray(energies, dtype=np.float64)
    if ref_conv.size == 0 or energies.size == 0:
        return conv, None, 0
    from scipy.optimize import linear_sum_assignment

    dist = np.abs(energies[:, None] - ref_conv[None, :])
    rows, cols = linear_sum_assignment(dist)
    return conv, float(dist[rows, cols].max()), int(rows.size)


def fp64_check(engine: Any, kpoint: Sequence[float], interval: EnergyInterval, *,
               eta_ev: float | None = None, tol: float = 1e-9, max_sweeps: int = 30) -> dict:
    """Refine the engine's eigenpairs at one k point (see the module text)
    and return the comparison.  ``engine`` is a BandEngine on a bundle."""
    import torch

    dev = engine.device
    keep = engine.keep_vectors
    engine.keep_vectors = True
    try:
        res, _ = engine.solve_kpoints([kpoint], interval)
        energies = np.asarray(engine.last_energies[0], dtype=np.float64)
        vec = engine.last_vectors[0]
    finally:
        engine.keep_vectors = keep
    m = int(energies.size)
    if m == 0 or vec is None:
        return {"count": 0}
    n = engine.n
    with torch.cuda.device(dev):
        hvals, svals = engine.bloch.apply(np.asarray([kpoint], dtype=np.float64))
        sv = torch.empty_like(vec)
        engine._spmm(svals[0], vec, sv)
        if eta_ev is None:
            spacing = float(np.median(np.diff(np.sort(energies)))) if m > 1 else 1e-3
            eta_ev = max(2e-3, 4.0 * spacing)
        centres = shift_centres(energies, eta_ev)
        L = max(len(mem) for _, mem in centres)
        L += L & 1   # an even column count keeps the solves on their TMA epilogue
        xs = torch.zeros((n, m), dtype=torch.complex128, device=dev)
        sweeps_used, worst_rel = 0, 0.0
        lib = native.library()
        info = engine.plan.info
        precision = engine.precision_id()
        cap = max(1, min(engine.max_pencils(L), len(centres)))
        # the engine's own factor storage of the last solve may still sit in
        # the allocator's cache
        torch.cuda.empty_cache()
        fbytes = lib.aosb_factor_bytes(engine.plan.handle, cap)
        factor = torch.empty(fbytes // 4, dtype=torch.float32, device=dev)
        pivots = torch.empty((cap, info.n_pad), dtype=torch.int32, device=dev)
        status = torch.zeros(cap, dtype=torch.int32, device=dev)
        wbytes = lib.aosb_factor_workspace_bytes(engine.plan.handle, cap, precision)
        workspace = torch.empty(max(wbytes, 16), dtype=torch.uint8, device=dev)
        wn = torch.empty((cap, info.n_pad, L), dtype=torch.complex64, device=dev)
        scratch = torch.empty(max(16, lib.aosb_solve_scratch_bytes(engine.plan.handle, cap, L)),
                              dtype=torch.uint8, device=dev)
        st = engine._stream()
        flags = native.SOLVE_TENSOR_CORES if (precision != native.PRECISION_PLAIN and
                                               info.tile == 128) else 0
        for b0 in range(0, len(centres), cap):
            batch = centres[b0:b0 + cap]
            np_ = len(batch)
            pk = torch.zeros(np_, dtype=torch.int32, device=dev)
            z = torch.tensor([complex(c, eta_ev) for c, _ in batch], dtype=torch.complex128,
                             device=dev)
            b = torch.zeros((np_, n, L), dtype=torch.complex128, device=dev)
            for p, (_, mem) in enumerate(batch):
                b[p, :, :len(mem)] = sv[:, mem]
            status.zero_()
            fa = native.FactorArgs(native.ABI_VERSION, native.C.sizeof(native.FactorArgs), np_,
                                   precision, hvals.data_ptr(), svals.data_ptr(), pk.data_ptr(),
                                   z.data_ptr(), factor.data_ptr(), pivots.data_ptr(),
                                   status.data_ptr(), workspace.data_ptr(), st)
            native.call("aosb_factor", engine.plan.handle, native.C.byref(fa))
            bad = status[:np_].cpu().numpy()
            if np.any(bad != 0):
                raise SolverError(f"FP64 check factorization failed with status {int(bad[bad != 0][0])}")
            xn = torch.zeros((np_, n, L), dtype=torch.complex128, device=dev)
            rr = b.clone()
            sa = native.SolveArgs(native.ABI_VERSION, native.C.sizeof(native.SolveArgs), np_, L,
                                  0, flags, factor.data_ptr(), pivots.data_ptr(), wn.data_ptr(),
                                  scratch.data_ptr(), st)
            bnorm = torch.linalg.vector_norm(b, dim=1).clamp_min(1e-300)
            rel = float("inf")
            sweeps = 0
            while sweeps < max_sweeps:
                native.call("aosb_gather_rhs", engine.plan.handle, np_, L, rr.data_ptr(), n * L,
                            wn.data_ptr(), st)
                native.call("aosb_solve", engine.plan.handle, native.C.byref(sa))
                native.call("aosb_scatter_solution", engine.plan.handle, np_, L, wn.data_ptr(),
                            xn.data_ptr(), 1 if sweeps else 0, st)
                if flags:
                    native.call("aosb_solve_check", engine.plan.handle, native.C.byref(sa))
                engine._residual(n, L, np_, hvals, svals, pk, z, b, xn, rr, st)
                sweeps += 1
                rnorm = torch.linalg.vector_norm(rr, dim=1)
                used = torch.zeros_like(rnorm, dtype=torch.bool)
                for p, (_, mem) in enumerate(batch):
                    used[p, :len(mem)] = True
                rel = float(torch.where(used, rnorm / bnorm, torch.zeros_like(rnorm)).max())
                if rel <= tol:
                    break
            sweeps_used = max(sweeps_used, sweeps)
            worst_rel = max(worst_rel, rel)
            for p, (_, mem) in enumerate(batch):
                xs[:, mem] = xn[p, :, :len(mem)]
        del factor, workspace, wn, scratch
        # FP64 Rayleigh-Ritz on span[V, X]
        space = torch.cat([vec, xs], dim=1).contiguous()
        ss = torch.empty_like(space)
        engine._spmm(svals[0], space, ss)
        g = engine._gram(space, ss).cpu().numpy()
        lam, w = np.linalg.eigh(hermitize(g))
        keep_cols = lam > lam.max() * 1e-13
        tr = w[:, keep_cols] / np.sqrt(lam[keep_cols])
        basis = engine._dense_mul(space, torch.from_numpy(np.ascontiguousarray(tr)).to(dev))
        hb = torch.empty_like(basis)
        sb = torch.empty_like(basis)
        engine._spmm(hvals[0], basis, hb)
        engine._spmm(svals[0], basis, sb)
        hr = engine._gram(basis, hb).cpu().numpy()
        sr = engine._gram(basis, sb).cpu().numpy()
        e2, c2 = projected_eigh(hr, sr)
        inside = (e2 > interval.lower_ev) & (e2 < interval.upper_ev)
        sel = np.flatnonzero(inside)
        refined = e2[sel]
        norms = np.zeros(sel.size)
        if sel.size:
            vv = engine._dense_mul(basis, torch.from_numpy(np.ascontiguousarray(c2[:, sel])).to(dev))
            hv = torch.empty_like(vv)
            svv = torch.empty_like(vv)
            engine._spmm(hvals[0], vv, hv)
            engine._spmm(svals[0], vv, svv)
            e_d = torch.from_numpy(np.ascontiguousarray(refined)).to(dev)
            nd = torch.empty(sel.size, dtype=torch.float64, device=dev)
            native.call("aosb_column_norms", n, int(sel.size), hv.data_ptr(), svv.data_ptr(),
                        hv.stride(0), e_d.data_ptr(), nd.data_ptr(), st)
            norms = nd.cpu().numpy()
    gaps = np.array([np.min(np.abs(np.delete(e2, i) - e2[i])) for i in sel]) if sel.size else \
        np.zeros(0)
    bound = norms ** 2 / np.maximum(gaps, 1e-300)
    engine_res = float(res[0].maximum_residual_ev)
    conv, err, paired = compare_refined(energies, refined, norms, engine_res)
    ref_conv = refined[conv]
    return {"count": m, "refined_count": int(refined.size), "converged_count": int(ref_conv.size),
            "count_diff": int(m - ref_conv.size), "paired": paired,
            "max_eig_error_ev": err,
            "engine_max_residual_ev": engine_res,
            "refined_max_residual_ev": float(norms[conv].max()) if conv.any() else 0.0,
            "refined_error_bound_ev": float(bound[conv].max()) if conv.any() else 0.0,
            "shifts": len(centres), "eta_ev": float(eta_ev), "rhs_per_shift": L,
            "refinement_sweeps": sweeps_used, "solve_relative_residual": worst_rel,
            "tolerance": tol}
