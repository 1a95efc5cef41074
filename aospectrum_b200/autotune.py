"""Project-written autotuner for the tile plan and the pencil batch.

Two choices decide how the shifted factorizations map onto the GPU:

* the tile plan -- the tile edge T (the "supernode" tile shape: 128 for the
  tensor-core path, 32/64/128 for the FP32 SIMT path) and the ordering
  (natural/banded or nested dissection).  Flop counts alone mislead here:
  the tensor-core Schur update is bound by target-tile traffic, the
  diagonal LU by latency, and the fill differs between orderings;
* the number of k points per batch -- every k point brings its
  (contour-node-pair) pencils, and a batch runs their diagonal LU, panel,
  Schur and sweep launches together, so small per-step launches fill more
  of the machine while the working set grows with the batch.

``tune_plan`` builds every candidate plan on the host, times one
factorization launch of a probe batch on the device with CUDA events (after
one untimed launch) and keeps the fastest per pencil.  ``tune_batch`` times
``BandEngine.solve_kpoints`` for growing batches that fit the memory budget
and keeps the best k points per second.  Results are cached per (pattern
digest, precision, candidates) for the life of the process.
"""

from __future__ import annotations

import hashlib
from dataclasses import dataclass, field
from time import perf_counter
from typing import Any, Sequence

import numpy as np

from . import native

_PLAN_CACHE: dict[tuple, tuple[int, str, dict]] = {}
_BATCH_CACHE: dict[tuple, tuple[int, dict]] = {}


@dataclass
class TuneResult:
    tile: int
    ordering: str
    ms_per_pencil: dict[str, float] = field(default_factory=dict)
    kpoints_per_batch: int = 1
    kpoints_per_s: dict[int, float] = field(default_factory=dict)

    def as_dict(self) -> dict[str, Any]:
        return {"tile": self.tile, "ordering": self.ordering,
                "factor_ms_per_pencil": {k: round(v, 3) for k, v in self.ms_per_pencil.items()},
                "kpoints_per_batch": self.kpoints_per_batch,
                "kpoints_per_s_by_batch": {str(k): round(v, 4)
                                           for k, v in self.kpoints_per_s.items()}}


def pattern_digest(indptr: np.ndarray, indices: np.ndarray) -> str:
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(indptr, dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(indices, dtype=np.int32).tobytes())
    return h.hexdigest()


def plan_candidates(n: int, precision: int) -> list[tuple[int, str]]:
    """(tile, ordering) pairs to time: the tensor-core path needs T = 128."""
    orderings = ["natural", "nested_dissection"]
    if precision in (native.PRECISION_BF16X3, native.PRECISION_BF16X3_FP32_PANELS):
        tiles = [128]
    elif n <= 256:
        tiles = [32, 64]
    elif n <= 2048:
        tiles = [32, 64, 128]
    else:
        tiles = [64, 128]
    return [(t, o) for t in tiles for o in orderings]


def time_factorization(plan: Any, h_values: Any, s_values: Any, shift: complex, pencils: int,
                       precision: int, device: Any) -> float:
    """Device milliseconds of one aosb_factor launch of ``pencils`` pencils
    (all on value row 0 and ``shift``), after one untimed launch."""
    import torch

    lib = native.library()
    info = plan.info
    factor = torch.empty(lib.aosb_factor_bytes(plan.handle, pencils) // 4, dtype=torch.float32,
                         device=device)
    piv = torch.empty((pencils, info.n_pad), dtype=torch.int32, device=device)
    status = torch.zeros(pencils, dtype=torch.int32, device=device)
    ws = torch.empty(max(16, lib.aosb_factor_workspace_bytes(plan.handle, pencils, precision)),
                     dtype=torch.uint8, device=device)
    pk = torch.zeros(pencils, dtype=torch.int32, device=device)
    z = torch.full((pencils,), complex(shift), dtype=torch.complex128, device=device)
    stream = torch.cuda.current_stream(device)
    fa = native.FactorArgs(native.ABI_VERSION, native.C.sizeof(native.FactorArgs), pencils,
                           precision, h_values.data_ptr(), s_values.data_ptr(), pk.data_ptr(),
                           z.data_ptr(), factor.data_ptr(), piv.data_ptr(), status.data_ptr(),
                           ws.data_ptr(), stream.cuda_stream)
    native.call("aosb_factor", plan.handle, native.C.byref(fa))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    native.call("aosb_factor", plan.handle, native.C.byref(fa))
    ev1.record(stream)
    ev1.synchronize()
    ms = float(ev0.elapsed_time(ev1))
    del factor, piv, status, ws
    return ms


def tune_plan(n: int, indptr: np.ndarray, indices: np.ndarray,
              supervariables: np.ndarray | None, h_values: Any, s_values: Any, *,
              precision: int, device: Any, probe_pencils: int = 2, shift: complex = 0.05j,
              candidates: Sequence[tuple[int, str]] | None = None):
    """The fastest SymbolicPlan per pencil among ``candidates`` and a
    TuneResult with every timing.  h_values / s_values: device complex64
    [1][nnz] values of one k point on this pattern."""
    from .engine import SymbolicPlan

    cands = list(candidates or plan_candidates(n, precision))
    key = (pattern_digest(indptr, indices), precision, tuple(cands))
    if key in _PLAN_CACHE:
        tile, ordering, timings = _PLAN_CACHE[key]
        plan = SymbolicPlan(n, indptr, indices, tile=tile, supervariables=supervariables,
                            ordering=ordering, device=device)
        return plan, TuneResult(tile, ordering, dict(timings))
    best = None
    timings: dict[str, float] = {}
    for tile, ordering in cands:
        plan = SymbolicPlan(n, indptr, indices, tile=tile, supervariables=supervariables,
                            ordering=ordering, device=device)
        ms = time_factorization(plan, h_values, s_values, shift, probe_pencils, precision,
                                device) / probe_pencils
        timings[f"T{tile}-{ordering}"] = ms
        if best is None or ms < best[0]:
            if best is not None:
                best[1].close()
            best = (ms, plan, tile, ordering)
        else:
            plan.close()
    _, plan, tile, ordering = best
    _PLAN_CACHE[key] = (tile, ordering, timings)
    return plan, TuneResult(tile, ordering, timings)


def tune_batch(engine: Any, kpoints: Sequence[Sequence[float]], interval: Any,
               sizes: Sequence[int] = (1, 2, 4), repeats: int = 2) -> tuple[int, dict[int, float]]:
    """k points per ``solve_kpoints`` call with the best k points per second
    among ``sizes`` whose pencils fit the engine's pencil budget.  After one
    warm-up call of the smallest size, the sizes are timed in ``repeats``
    interleaved rounds and each keeps its fastest round (the clock of a
    power-capped GPU moves between calls; one slow sample must not decide)."""
    import torch

    def sync() -> None:
        if torch.device(engine.device).type == "cuda":
            torch.cuda.current_stream(engine.device).synchronize()

    st = engine.settings
    pairs = (st.integration_points + 1) // 2 if engine.engine.precision == "mixed" \
        else st.integration_points
    cap = engine.max_pencils(st.block_size)
    sizes = [s for s in sizes if s * pairs <= cap and s <= len(kpoints)] or [1]
    key = (id(engine.plan), tuple(sizes), st.integration_points, st.block_size)
    if key in _BATCH_CACHE:
        return _BATCH_CACHE[key]
    engine.solve_kpoints(kpoints[:1], interval)
    rates: dict[int, float] = {}
    for _ in range(max(1, repeats)):
        for s in sizes:
            sync()
            t0 = perf_counter()
            engine.solve_kpoints(kpoints[:s], interval)
            sync()
            rates[s] = max(rates.get(s, 0.0), s / (perf_counter() - t0))
    best = max(rates, key=rates.get)
    _BATCH_CACHE[key] = (best, rates)
    return best, rates
