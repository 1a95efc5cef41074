"""The project-written autotuner: candidate enumeration and the batch
choice (CPU, with a fake engine whose call cost is known), and on the GPU a
tuned tile plan that gives the eigenvalues of the default plan."""

from __future__ import annotations

import json
import time
from types import SimpleNamespace

import numpy as np
import pytest

import bundles
from aospectrum_b200 import autotune, native
from aospectrum_b200.ciss import CissSettings


def test_plan_candidates_follow_the_precision_and_size():
    tc = autotune.plan_candidates(13000, native.PRECISION_BF16X3)
    assert tc == [(128, "natural"), (128, "nested_dissection")]
    assert autotune.plan_candidates(13000, native.PRECISION_BF16X3_FP32_PANELS) == tc
    small = autotune.plan_candidates(200, native.PRECISION_PLAIN)
    assert sorted({t for t, _ in small}) == [32, 64]
    mid = autotune.plan_candidates(2000, native.PRECISION_PLAIN)
    assert sorted({t for t, _ in mid}) == [32, 64, 128]
    big = autotune.plan_candidates(13000, native.PRECISION_PLAIN)
    assert sorted({t for t, _ in big}) == [64, 128]
    for cands in (tc, small, mid, big):
        assert {o for _, o in cands} == {"natural", "nested_dissection"}


class FakeEngine:
    """solve_kpoints costs overhead + per_k seconds per k point; the pencil
    budget caps the batch."""

    def __init__(self, overhead: float, per_k: float, cap_pencils: int):
        import torch

        self.device = torch.device("cpu")
        self.settings = CissSettings(integration_points=8, block_size=4)
        self.engine = SimpleNamespace(precision="mixed")
        self.plan = object()
        self.cost = (overhead, per_k)
        self.cap = cap_pencils
        self.calls: list[int] = []

    def max_pencils(self, n_rhs: int) -> int:
        return self.cap

    def solve_kpoints(self, kpoints, interval):
        self.calls.append(len(kpoints))
        time.sleep(self.cost[0] + self.cost[1] * len(kpoints))
        return [], []


def test_tune_batch_picks_the_best_rate_within_the_pencil_budget():
    kpts = [(0.0, 0.0, 0.1 * i) for i in range(8)]
    # fixed cost per call dominates: the largest batch that fits wins
    eng = FakeEngine(overhead=0.03, per_k=0.002, cap_pencils=4 * 4)
    best, rates = autotune.tune_batch(eng, kpts, None, sizes=(1, 2, 4, 8), repeats=2)
    assert set(rates) == {1, 2, 4}          # 8 k x 4 pencil pairs exceeds the budget
    assert best == 4
    assert eng.calls[0] == 1 and eng.calls.count(4) == 2   # warm-up, then 2 rounds
    # cached per plan: no further calls
    n = len(eng.calls)
    assert autotune.tune_batch(eng, kpts, None, sizes=(1, 2, 4, 8), repeats=2)[0] == 4
    assert len(eng.calls) == n
    # a budget below one k point's pencils still runs one k point per call
    eng2 = FakeEngine(overhead=0.0, per_k=0.001, cap_pencils=2)
    assert autotune.tune_batch(eng2, kpts, None, sizes=(2, 4))[0] == 1


@pytest.mark.gpu
def test_tuned_plan_gives_the_default_plans_eigenvalues(golden):
    import torch

    from aospectrum_b200.ciss import EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine

    torch.cuda.set_device(0)
    case = json.loads((golden / "manifest.json").read_text())["ciss"]["c1_k0"]
    ref = np.sort(np.load(golden / "ciss.npz")["c1_k0_energies"].astype(np.float64))
    interval = EnergyInterval(*case["interval"])
    k = [bundles.KPOINTS[case["k_index"]]]
    got = {}
    for tuned in (False, True):
        eng = BandEngine(bundles.c1(), CissSettings(), EngineSettings(autotune=tuned))
        try:
            if tuned:
                t = eng.tuning.as_dict()
                assert t["tile"] == 128
                assert set(t["factor_ms_per_pencil"]) == {"T128-natural",
                                                          "T128-nested_dissection"}
                assert all(v > 0 for v in t["factor_ms_per_pencil"].values())
                assert eng.plan.ordering == t["ordering"]
            res, _ = eng.solve_kpoints(k, interval)
            got[tuned] = np.sort(res[0].energies_ev.astype(np.float64))
        finally:
            eng.close()
    assert got[True].size == got[False].size == ref.size
    assert np.max(np.abs(got[True] - got[False])) < 1e-4
    assert np.max(np.abs(got[True] - ref)) < 1e-4
