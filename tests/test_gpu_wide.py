"""Wide Schur and panel products (aosb_factor_set_schur_wide: U tiles staged
as the operand rows [-Ui; Ur; Ui], six M = 128, N = 256 MMAs per K slab
each writing both halves of the accumulator) against the N = 128 form.
The MMAs take the same split-BF16 products in the same order per element,
so factorizations and solves agree to rounding; covered for the two-step
updates with lookahead (static cross items and the shared rest-item
counter), the one-step updates, several pencils and a 2808-orbital cubic
bundle, and CISS eigenvalues against the reference's.  With two-CTA pairs
on, the switch is ignored (pairs read the plain staging layout)."""

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


def _cubic6():
    from aospectrum_b200 import synth

    return synth.generate_bundle(replace(synth.SPEC_C2, name="cubic6", grid=(6, 6, 6),
                                         cell=(14.4, 14.4, 14.4), seed=17))


@pytest.mark.parametrize("case,ordering,pencils,mode", [
    ("c1", "natural", 3, "two_step"), ("c1", "nested_dissection", 2, "one_step"),
    ("cubic6", "natural", 5, "two_step"), ("c1", "natural", 2, "pairs")])
def test_wide_factor_matches_n128_form(case, ordering, pencils, mode, torch):
    from aospectrum_b200 import native

    lib = native.library()
    precision = (native.PRECISION_BF16X3_ONE_STEP if mode == "one_step"
                 else native.PRECISION_BF16X3)
    b = bundles.c1() if case == "c1" else _cubic6()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[1], torch, 128, ordering)
    rng = np.random.default_rng(13)
    rhs = rng.standard_normal((dev.n, 8)) + 1j * rng.standard_normal((dev.n, 8))
    shifts = [-2.6 + 0.02j * (p + 1) + 0.3 * p for p in range(pencils)]
    prev = lib.aosb_factor_set_schur_wide(0)
    prev_pairs = lib.aosb_factor_set_schur_pairs(1 if mode == "pairs" else 0)
    assert prev in (0, 1) and prev_pairs in (0, 1)
    try:
        narrow = _factor_solve(dev, plan, h, s, shifts, rhs, torch, precision=precision)
        lib.aosb_factor_set_schur_wide(1)
        wide = _factor_solve(dev, plan, h, s, shifts, rhs, torch, precision=precision)
        wide_again = _factor_solve(dev, plan, h, s, shifts, rhs, torch, precision=precision)
    finally:
        lib.aosb_factor_set_schur_wide(prev)
        lib.aosb_factor_set_schur_pairs(prev_pairs)
        dev.close()
        plan.close()
    for p in range(pencils):
        rel = np.linalg.norm(wide[p] - narrow[p]) / np.linalg.norm(narrow[p])
        assert rel < 1e-5, (p, rel)
        rel2 = np.linalg.norm(wide_again[p] - wide[p]) / np.linalg.norm(wide[p])
        assert rel2 < 1e-5, (p, rel2)


def test_wide_engine_ciss_matches_reference(golden, torch):
    from aospectrum_b200 import native
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine

    lib = native.library()
    case = json.loads((golden / "manifest.json").read_text())["ciss"]["c1_k0"]
    ref = np.sort(np.load(golden / "ciss.npz")["c1_k0_energies"].astype(np.float64))
    prev = lib.aosb_factor_set_schur_wide(1)
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
        lib.aosb_factor_set_schur_wide(prev)
