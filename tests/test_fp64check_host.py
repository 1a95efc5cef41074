"""The pairing rule of the FP64 check (aospectrum_b200.fp64check), on the
host: refined Ritz values whose residual shows they approximate no
eigenpair are left out, and the engine's values are paired one to one with
the converged ones."""

from __future__ import annotations

import numpy as np

from aospectrum_b200.fp64check import compare_refined


def test_unconverged_ritz_values_are_left_out():
    engine = np.array([-2.50, -2.49, -2.48])
    refined = np.array([-2.50002, -2.4951, -2.49001, -2.48003])
    residuals = np.array([1e-6, 0.6, 2e-6, 1e-6])   # -2.4951 is spurious
    conv, err, paired = compare_refined(engine, refined, residuals, 1e-4)
    assert conv.tolist() == [True, False, True, True]
    assert paired == 3
    assert abs(err - 3e-5) < 1e-12


def test_pairing_is_one_to_one():
    # two engine values near one refined value: the second pairs with the
    # next refined value, not the same one
    engine = np.array([-1.0, -0.9999])
    refined = np.array([-1.0, -0.9990])
    conv, err, paired = compare_refined(engine, refined, np.zeros(2), 0.0)
    assert paired == 2 and abs(err - 9e-4) < 1e-12


def test_engine_residual_widens_the_converged_threshold():
    refined = np.array([0.0, 1.0])
    residuals = np.array([4e-3, 6e-3])
    conv, _, _ = compare_refined(np.array([0.0]), refined, residuals, 2.5e-3)
    assert conv.tolist() == [True, False]
    conv, err, paired = compare_refined(np.array([]), refined, residuals, 0.0)
    assert not conv.any() and err is None and paired == 0
