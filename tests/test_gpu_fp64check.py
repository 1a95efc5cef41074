"""The FP64 eigenvalue check used where a dense FP64 eigensolver does not
fit (aospectrum_b200.fp64check), validated where one does: on the 64-atom
sheet its refined eigenvalues must agree with FP64 dense generalized eigh
far below the 1e-4 eV target, its solves must reach the requested
refinement tolerance, and the error it reports for the engine's values
must be the true error against the dense oracle."""

from __future__ import annotations

import json

import numpy as np
import pytest

import bundles
from oracle import dense_ref

pytestmark = pytest.mark.gpu


def test_fp64_check_agrees_with_dense_fp64(golden):
    import torch

    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine
    from aospectrum_b200.fp64check import fp64_check

    torch.cuda.set_device(0)
    case = json.loads((golden / "manifest.json").read_text())["ciss"]["c1_k0"]
    interval = EnergyInterval(*case["interval"])
    k = bundles.KPOINTS[case["k_index"]]
    eng = BandEngine(bundles.c1(), CissSettings(), EngineSettings(precision="mixed"))
    try:
        eng.keep_vectors = True
        res, _ = eng.solve_kpoints([k], interval)
        mine = np.sort(np.asarray(eng.last_energies[0], np.float64))
        eng.keep_vectors = False
        chk = fp64_check(eng, k, interval)
        pair = eng.host_pair(k)
        hd, sd = dense_ref.dense_pair(pair.hamiltonian.indptr, pair.hamiltonian.indices,
                                      pair.hamiltonian.data, pair.overlap.data, eng.n)
        exact = dense_ref.window(dense_ref.eigenvalues(hd, sd), *case["interval"])
    finally:
        eng.close()
    assert chk["count"] == mine.size == exact.size and chk["count_diff"] == 0
    assert chk["solve_relative_residual"] <= chk["tolerance"]
    true_err = float(np.max(np.abs(mine - exact)))
    # the reported error is the true error, up to the refined values' own error
    assert abs(chk["max_eig_error_ev"] - true_err) < 1e-7
    assert chk["refined_error_bound_ev"] < 1e-6
    assert chk["refined_max_residual_ev"] < res[0].maximum_residual_ev
