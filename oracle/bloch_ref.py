"""numpy restatement of the reference Bloch assembly -- test oracle only.

Follows src/aospectrum/sparse.py of yumiaoyi-o/AOSpectrum:
  pattern   from_bundle       sparse.py:64-140  (entry expansion, stable
                                                 argsort on row*n+col,
                                                 dedup, Hermitian check)
  values    _fill             sparse.py:181-197 (gather, phase multiply,
                                                 reduceat)
            update            sparse.py:199-245 (complex64 phases)
  projection _project_hermitian sparse.py:25-36
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


class TopologyError(ValueError):
    pass


@dataclass
class RefPattern:
    n: int
    indptr: np.ndarray
    indices: np.ndarray
    source: np.ndarray      # value index of every expanded entry, sorted
    group: np.ndarray       # lattice-shift index of every expanded entry
    starts: np.ndarray      # segment starts (one segment per CSR entry)
    shifts: np.ndarray      # distinct lattice shifts (int32, n_shifts x 3)
    upper: np.ndarray
    lower: np.ndarray
    diagonal: np.ndarray


def build_pattern(bundle) -> RefPattern:
    """sparse.py:64-140."""
    ops = bundle.operators
    off = np.asarray(bundle.basis.atom_offsets, dtype=np.int64)
    n = bundle.n_orbitals
    shifts, grp_of_block = np.unique(np.asarray(ops.lattice_shift), axis=0, return_inverse=True)
    grp_of_block = np.asarray(grp_of_block).reshape(-1)
    rows, cols, src, grp = [], [], [], []
    for b in range(ops.n_blocks):
        nr, nc = (int(v) for v in ops.block_shapes[b])
        r0, c0 = int(off[ops.row_atom[b]]), int(off[ops.col_atom[b]])
        rows.append(r0 + np.repeat(np.arange(nr, dtype=np.int64), nc))
        cols.append(c0 + np.tile(np.arange(nc, dtype=np.int64), nr))
        s = np.arange(int(ops.block_offsets[b]), int(ops.block_offsets[b + 1]), dtype=np.int64)
        src.append(s)
        grp.append(np.full(s.size, grp_of_block[b], dtype=np.int64))
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    src, grp = np.concatenate(src), np.concatenate(grp)
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    skey = key[order]
    first = np.ones(skey.size, dtype=bool)
    first[1:] = skey[1:] != skey[:-1]
    starts = np.flatnonzero(first)
    uniq = skey[starts]
    ur, uc = uniq // n, uniq % n
    mkey = uc * n + ur
    mirror = np.searchsorted(uniq, mkey)
    if np.any(mirror >= uniq.size) or not np.array_equal(uniq[mirror], mkey):
        raise TopologyError("operator topology is not Hermitian")
    upper = np.flatnonzero(ur < uc)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(ur, minlength=n), out=indptr[1:])
    return RefPattern(n, indptr, uc.astype(np.int64), src[order], grp[order], starts,
                      np.asarray(shifts, dtype=np.int32), upper, mirror[upper],
                      np.flatnonzero(ur == uc))


def phases(shifts: np.ndarray, k) -> np.ndarray:
    """complex64 exp(2 pi i R.k) with a float32 argument (sparse.py:207-213)."""
    arg = shifts.astype(np.float32) @ np.asarray(tuple(float(v) for v in k), dtype=np.float32)
    return np.exp(np.asarray(2.0j * np.pi, dtype=np.complex64) * arg).astype(np.complex64)


def project_hermitian(values: np.ndarray, pat: RefPattern) -> None:
    """sparse.py:25-36."""
    if pat.upper.size:
        mean = (values[pat.upper] + np.conjugate(values[pat.lower])) * 0.5
        values[pat.upper] = mean
        values[pat.lower] = np.conjugate(mean)
    if np.iscomplexobj(values) and pat.diagonal.size:
        values[pat.diagonal] = np.real(values[pat.diagonal])


def bloch_values(pat: RefPattern, values: np.ndarray, k) -> np.ndarray:
    """One of H(k) or S(k) as complex64 CSR data (sparse.py:181-245)."""
    ph = phases(pat.shifts, k)
    scratch = np.empty(pat.source.size, dtype=np.complex64)
    scratch[...] = np.asarray(values)[pat.source]
    np.multiply(scratch, ph[pat.group], out=scratch)
    out = np.empty(pat.starts.size, dtype=np.complex64)
    np.add.reduceat(scratch, pat.starts, out=out)
    project_hermitian(out, pat)
    return out


def bloch_pair(pat: RefPattern, bundle, k) -> tuple[np.ndarray, np.ndarray]:
    ops = bundle.operators
    return bloch_values(pat, ops.h_values, k), bloch_values(pat, ops.s_values, k)
