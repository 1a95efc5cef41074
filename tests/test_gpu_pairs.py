"""Two-CTA (cta_group::2, M = 256) Schur updates against the one-CTA
two-step updates they replace: the same targets get the same split-BF16
products (FP32 accumulation in the same K order), so the factorizations
and solves agree to rounding, and CISS eigenvalues match the reference's.
Covers the static schedule (cross items) and the shared item counter of the
main and lookahead launches (rest items), pairs and singles, odd pencil
counts, and a 2808-orbital cubic bundle with many pairs per super-step."""

from __future__ import annotations

import json
from dataclasses import replace

import numpy as np
import pytest

import bundles
from test_gpu_parity import _factor_solve, _pencil_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    t.cuda.set_device(0)
    return t


def _with_pairs(lib, on):
    prev = lib.aosb_factor_set_schur_pairs(1 if on else 0)
    assert prev in (0, 1)
    return prev


def _cubic6():
    from aospectrum_b200 import synth

    return synth.generate_bundle(replace(synth.SPEC_C2, name="cubic6", grid=(6, 6, 6),
                                         cell=(14.4, 14.4, 14.4), seed=17))


@pytest.mark.parametrize("case,ordering,pencils", [("c1", "natural", 3), ("c1", "nested_dissection", 2),
                                                   ("cubic6", "natural", 5)])
def test_pair_factor_matches_single_cta(case, ordering, pencils, torch):
    from aospectrum_b200 import native

    lib = native.library()
    b = bundles.c1() if case == "c1" else _cubic6()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[1], torch, 128, ordering)
    rng = np.random.default_rng(9)
    rhs = rng.standard_normal((dev.n, 8)) + 1j * rng.standard_normal((dev.n, 8))
    shifts = [-2.6 + 0.02j * (p + 1) + 0.3 * p for p in range(pencils)]
    prev = _with_pairs(lib, False)
    try:
        one = _factor_solve(dev, plan, h, s, shifts, rhs, torch,
                            precision=native.PRECISION_BF16X3)
        _with_pairs(lib, True)
        two = _factor_solve(dev, plan, h, s, shifts, rhs, torch,
                            precision=native.PRECISION_BF16X3)
        two_again = _factor_solve(dev, plan, h, s, shifts, rhs, torch,
                                  precision=native.PRECISION_BF16X3)
    finally:
        lib.aosb_factor_set_schur_pairs(prev)
        dev.close()
        plan.close()
    for p in range(pencils):
        rel = np.linalg.norm(two[p] - one[p]) / np.linalg.norm(one[p])
        assert rel < 1e-5, (p, rel)
        rel2 = np.linalg.norm(two_again[p] - two[p]) / np.linalg.norm(two[p])
        assert rel2 < 1e-5, (p, rel2)


def test_pair_engine_ciss_matches_reference(golden, torch):
    from aospectrum_b200 import native
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine

    lib = native.library()
    case = json.loads((golden / "manifest.json").read_text())["ciss"]["c1_k0"]
    ref = np.sort(np.load(golden / "ciss.npz")["c1_k0_energies"].astype(np.float64))
    prev = _with_pairs(lib, True)
    eng = BandEngine(bundles.c1(), CissSettings(), EngineSettings(precision="mixed"))
    try:
        res, _ = eng.solve_kpoints([bundles.KPOINTS[case["k_index"]]],
                                   EnergyInterval(*case["interval"]))
        got = np.sort(res[0].energies_ev.astype(np.float64))
        assert got.size == ref.size
        assert np.max(np.abs(got - ref)) < 1e-4
        assert res[0].maximum_residual_ev <= case["max_residual_ev"] * 1.01
    finally:
        eng.close()
        lib.aosb_factor_set_schur_pairs(prev)
