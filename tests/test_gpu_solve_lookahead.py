"""Lookahead in the tensor-core triangular sweeps: the next step's tile is
updated first and the next diagonal solve runs on a side stream beside the
rest of the current step's updates, with double-buffered diagonal results.
The arithmetic is unchanged, so the solutions must equal the in-order
sweeps bit for bit (normal and adjoint sweeps, 32 and 40 right-hand sides,
and graph-captured sweeps)."""

from __future__ import annotations

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


@pytest.mark.parametrize("case", ["c1", "cubic6"])
@pytest.mark.parametrize("adjoint", [0, 1])
@pytest.mark.parametrize("L", [32, 40])
def test_lookahead_sweeps_equal_in_order_sweeps(case, adjoint, L, torch):
    from aospectrum_b200 import native

    lib = native.library()
    b = bundles.c1() if case == "c1" else _cubic6()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[2], torch, 128, "natural")
    rng = np.random.default_rng(4)
    rhs = rng.standard_normal((dev.n, L)) + 1j * rng.standard_normal((dev.n, L))
    shifts = [-2.5 + 0.03j, -1.2 + 0.4j, 0.3 + 0.01j]
    prev = lib.aosb_solve_set_lookahead(0)
    try:
        ref = _factor_solve(dev, plan, h, s, shifts, rhs, torch, precision=native.PRECISION_BF16X3,
                            adjoint=adjoint, flags=native.SOLVE_TENSOR_CORES)
        lib.aosb_solve_set_lookahead(1)
        got = _factor_solve(dev, plan, h, s, shifts, rhs, torch, precision=native.PRECISION_BF16X3,
                            adjoint=adjoint, flags=native.SOLVE_TENSOR_CORES)
        graph = _factor_solve(dev, plan, h, s, shifts, rhs, torch,
                              precision=native.PRECISION_BF16X3, adjoint=adjoint,
                              flags=native.SOLVE_TENSOR_CORES | native.SOLVE_GRAPH)
    finally:
        lib.aosb_solve_set_lookahead(prev)
        dev.close()
        plan.close()
    assert np.array_equal(got, ref)
    assert np.array_equal(graph, ref)
