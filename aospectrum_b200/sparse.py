"""Sparse H(k), S(k) containers shared with user-supplied solvers.

``SparsePair`` is the object the reference passes to
``solve_interval`` (``src/aospectrum/sparse.py:39-47``): scipy CSR H and S on
one pattern plus the fractional k point.
"""

from __future__ import annotations

from dataclasses import dataclass

from scipy import sparse


@dataclass(slots=True)
class SparsePair:
    hamiltonian: sparse.csr_matrix
    overlap: sparse.csr_matrix
    k_fractional: tuple[float, float, float]

    @property
    def n_orbitals(self) -> int:
        return int(self.hamiltonian.shape[0])
