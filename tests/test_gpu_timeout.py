"""Bounded waits of the tensor-core kernels, made to run out on purpose.

The wait limit of the tcgen05 kernels is a process-wide setting
(aosb_tc_set_wait_limit); the test runs with one-CTA and with two-CTA
(cluster) Schur updates.  With it cut to one poll, the mbarrier waits of
the split-BF16 factorization give up long before their copies and MMAs
land: each CTA that gives up records AOSB_ERR_TIMEOUT (52) in the pencil's
status word, drains its own copies and MMAs in flight, frees its TMEM and
returns.  The engine must report the status as a SolverError, and with the
default limit restored the next solve on the same context must succeed and
match the reference.  Nothing here faults, traps or hangs the GPU: the only
failure is a wait that stops polling early.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

import bundles

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pairs", [False, True])
def test_wait_limit_expiry_reports_timeout_and_context_survives(golden, pairs):
    import torch

    from aospectrum_b200 import native
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine
    from aospectrum_b200.errors import SolverError

    torch.cuda.set_device(0)
    lib = native.library()
    case = json.loads((golden / "manifest.json").read_text())["ciss"]["c1_k0"]
    ref = np.sort(np.load(golden / "ciss.npz")["c1_k0_energies"].astype(np.float64))
    eng = BandEngine(bundles.c1(), CissSettings(),
                     EngineSettings(precision="mixed", tensor_cores=True))
    assert eng.plan.info.tile == 128
    interval = EnergyInterval(*case["interval"])
    k = [bundles.KPOINTS[case["k_index"]]]
    prev_pairs = lib.aosb_factor_set_schur_pairs(1 if pairs else 0)
    try:
        prev = lib.aosb_tc_set_wait_limit(1)
        try:
            with pytest.raises(SolverError, match="status 52"):
                eng.solve_kpoints(k, interval)
            torch.cuda.synchronize()
        finally:
            lib.aosb_tc_set_wait_limit(prev)
        assert lib.aosb_tc_set_wait_limit(0) == prev
        res, _ = eng.solve_kpoints(k, interval)
        got = np.sort(res[0].energies_ev.astype(np.float64))
        assert got.size == ref.size
        assert np.max(np.abs(got - ref)) < 1e-4
        torch.cuda.synchronize()
    finally:
        lib.aosb_factor_set_schur_pairs(prev_pairs)
        eng.close()
