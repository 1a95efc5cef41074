"""Seeded bundles shared by the tests and the golden-vector generator."""

from __future__ import annotations

from dataclasses import replace

import numpy as np

from aospectrum_b200 import synth
from aospectrum_b200.data import LocalizedOperatorBlocks, LocalizedOperatorBundle


def tiny2d():
    return synth.generate_bundle(synth.small_spec("tiny2d", side=3, orbitals=5, seed=7, dims=2))


def tiny3d():
    return synth.generate_bundle(synth.small_spec("tiny3d", side=3, orbitals=5, seed=11, dims=3))


def small2d():
    """6x6 sheet, 13 orbitals (n = 468)."""
    spec = replace(synth.SPEC_C1, name="small2d", grid=(6, 6, 1), cell=(15.0, 15.0, 15.0),
                   seed=5)
    return synth.generate_bundle(spec)


def c1():
    return synth.generate_bundle(synth.SPEC_C1)


def complexified(bundle: LocalizedOperatorBundle, seed: int = 3) -> LocalizedOperatorBundle:
    """Adds an imaginary part i*A_b with A_mirror = -A_b^T so the topology
    stays Hermitian (H_{j0,i(-R)} = conj(H_{i0,jR})^T)."""
    ops = bundle.operators
    rng = np.random.default_rng(seed)
    rows, cols, sh = ops.row_atom, ops.col_atom, ops.lattice_shift
    key = {(int(r), int(c), tuple(int(v) for v in s)): b
           for b, (r, c, s) in enumerate(zip(rows, cols, sh))}
    hv = np.asarray(ops.h_values, dtype=np.complex64).copy()
    sv = np.asarray(ops.s_values, dtype=np.complex64).copy()
    done = set()
    for b, (r, c, s) in enumerate(zip(rows, cols, sh)):
        if b in done:
            continue
        m = key[(int(c), int(r), tuple(-int(v) for v in s))]
        nr, nc = (int(v) for v in ops.block_shapes[b])
        lo, hi = int(ops.block_offsets[b]), int(ops.block_offsets[b + 1])
        mlo, mhi = int(ops.block_offsets[m]), int(ops.block_offsets[m + 1])
        ah = (0.3 * rng.standard_normal((nr, nc))).astype(np.float32)
        as_ = (0.01 * rng.standard_normal((nr, nc))).astype(np.float32)
        if m == b:
            ah = 0.5 * (ah - ah.T)
            as_ = 0.5 * (as_ - as_.T)
        hv[lo:hi] += 1j * ah.reshape(-1)
        sv[lo:hi] += 1j * as_.reshape(-1)
        if m != b:
            hv[mlo:mhi] += 1j * (-ah.T).reshape(-1)
            sv[mlo:mhi] += 1j * (-as_.T).reshape(-1)
        done.update((b, m))
    blocks = LocalizedOperatorBlocks(rows, cols, sh, ops.block_offsets, ops.block_shapes, hv, sv)
    return LocalizedOperatorBundle(bundle.structure, bundle.basis, blocks, bundle.filling,
                                   bundle.provenance)


KPOINTS = [(0.0, 0.0, 0.0), (0.1, 0.27, 0.0), (0.5, 0.5, 0.0), (0.3, -0.2, 0.45)]
