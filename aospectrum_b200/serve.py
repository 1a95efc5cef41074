"""Device-resident Band serving loop with continuous batching.

Band requests (bundle, k points, energy window, CISS sizes) arrive at any
time.  The server keeps, per bundle, the Bloch tables with the resident
block values, the CSR pattern and the symbolic plan on the GPU
(``BundleResources``), so a request for a bundle that is already resident
skips the pattern build, the analysis and the upload.

Admission is by HBM footprint.  A request's footprint is the resident bytes
of its bundle (counted once per resident bundle) plus its working set: the
factor storage, pivots, staging and solve buffers of the pencils of one
work unit (``kpoints_per_unit`` k points x the node pairs of the contour)
plus the H(k), S(k) values and moments of that unit.  Waiting requests are
admitted in arrival order while their footprint fits the budget and a slot
is free; a request that does not fit lets later, smaller requests that do
fit go first (backfill).  A request larger than the whole budget is
rejected with ``InputError``.

Continuous batching: every admitted request is cut into work units of
``kpoints_per_unit`` k points.  ``slots`` worker threads, each with its own
CUDA stream, take units round-robin over the admitted requests (one unit of
a request at a time: its engine and working set serve one stream), so units
of different requests run concurrently on the device and a request that
arrives while others are running starts as soon as a slot and memory free
up.  A unit's numerics do not depend on what else runs: each pencil is
factored and solved on its own, so a request's eigenvalues are the same
alone and in the mix.

This loop has no counterpart in the reference, whose CLI runs one band job
per process and shards k points over processes through the filesystem
(``src/aospectrum/cli.py:330-436``).
"""

from __future__ import annotations

import itertools
import math
import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field, replace
from typing import Any, Callable, Sequence

import numpy as np

from .ciss import CissSettings, EngineSettings
from .data import EnergyInterval, LocalizedOperatorBundle
from .errors import InputError, SolverError


@dataclass
class BandRequest:
    """One band job: eigenvalues in ``interval`` at every k point."""

    bundle: LocalizedOperatorBundle
    kpoints: Sequence[Sequence[float]]
    interval: EnergyInterval
    settings: CissSettings = field(default_factory=CissSettings)
    request_id: str = ""


@dataclass
class BandResponse:
    request_id: str
    energies_ev: list[np.ndarray]
    maximum_residual_ev: float
    latency_seconds: float       # arrival -> last k point done
    queue_seconds: float         # arrival -> admission
    kpoints: int
    warnings: tuple[str, ...] = ()


@dataclass(eq=False)
class _Active:
    req: BandRequest
    future: Future
    arrival: float
    admitted: float = 0.0
    footprint: int = 0
    bundle_key: int = 0
    engine: Any = None
    units: deque = field(default_factory=deque)
    in_flight: int = 0
    results: dict = field(default_factory=dict)
    failed: BaseException | None = None


def percentile(values: Sequence[float], q: float) -> float:
    """Nearest-rank percentile (q in [0, 100])."""
    if not values:
        return float("nan")
    v = sorted(values)
    rank = max(1, math.ceil(q / 100.0 * len(v)))
    return float(v[rank - 1])


class BandServer:
    """Continuous-batching Band server on one GPU.

    ``engine_factory(request, resources, engine_settings, device)`` and
    ``resources_factory(bundle, device, tile)`` default to the GPU engine;
    tests pass host stand-ins.  ``footprint_fn(request, resources,
    kpoints_per_unit)`` returns (resident_bytes, working_bytes).
    """

    def __init__(self, *, device: Any = None, memory_budget_bytes: int | None = None,
                 slots: int = 4, kpoints_per_unit: int = 1,
                 engine_settings: EngineSettings | None = None,
                 engine_factory: Callable[..., Any] | None = None,
                 resources_factory: Callable[..., Any] | None = None,
                 footprint_fn: Callable[..., tuple[int, int]] | None = None,
                 stream_factory: Callable[[], Any] | None = None,
                 clock: Callable[[], float] = time.perf_counter) -> None:
        if slots < 1 or kpoints_per_unit < 1:
            raise InputError("slots and kpoints_per_unit must be >= 1")
        self.device = device
        self.engine_settings = engine_settings or EngineSettings()
        self.slots = slots
        self.kpoints_per_unit = kpoints_per_unit
        self.clock = clock
        self._engine_factory = engine_factory or _gpu_engine
        self._resources_factory = resources_factory or _gpu_resources
        self._footprint = footprint_fn or _gpu_footprint
        self._stream_factory = stream_factory or (lambda: _gpu_stream(device))
        if memory_budget_bytes is None:
            memory_budget_bytes = _default_budget(device)
        self.budget = int(memory_budget_bytes)
        self._lock = threading.Condition()
        self._waiting: deque[_Active] = deque()
        self._active: list[_Active] = []
        self._resources: dict[int, Any] = {}   # admitted (device-resident) bundles
        self._pending: dict[int, Any] = {}     # analysed on the host, not yet admitted
        self._resident_bytes: dict[int, int] = {}
        self._bundle_users: dict[int, int] = {}
        self._used = 0
        self._rr = itertools.count()
        self._closed = False
        self._done: list[BandResponse] = []
        self._kpoints_done = 0
        self._first_arrival: float | None = None
        self._last_done: float | None = None
        self.peak_used = 0
        self.max_concurrent_units = 0
        self._running_units = 0
        self._workers = [threading.Thread(target=self._worker, name=f"band-slot-{i}", daemon=True)
                         for i in range(slots)]
        for w in self._workers:
            w.start()

    # ---------------------------------------------------------------- public
    def submit(self, request: BandRequest) -> Future:
        """Queue a request; the future resolves to a ``BandResponse``."""
        kp = np.asarray([[float(v) for v in k] for k in request.kpoints], dtype=np.float64)
        if kp.ndim != 2 or kp.shape[1] != 3 or kp.shape[0] == 0:
            raise InputError("a band request needs one or more k points of three values")
        fut: Future = Future()
        now = self.clock()
        with self._lock:
            if self._closed:
                raise InputError("server is closed")
            if self._first_arrival is None:
                self._first_arrival = now
            act = _Active(req=request, future=fut, arrival=now)
            act.bundle_key = id(request.bundle)
            act.units = deque((i, kp[i:i + self.kpoints_per_unit])
                              for i in range(0, kp.shape[0], self.kpoints_per_unit))
            self._waiting.append(act)
            self._lock.notify_all()
        return fut

    def drain(self, timeout: float | None = None) -> None:
        """Block until every submitted request has finished."""
        deadline = None if timeout is None else time.monotonic() + timeout
        with self._lock:
            while self._waiting or self._active:
                left = None if deadline is None else deadline - time.monotonic()
                if left is not None and left <= 0:
                    raise TimeoutError("band server did not drain in time")
                self._lock.wait(timeout=left if left is not None else 0.5)

    def stats(self) -> dict[str, Any]:
        with self._lock:
            lat = [r.latency_seconds for r in self._done]
            span = ((self._last_done - self._first_arrival)
                    if self._done and self._first_arrival is not None else float("nan"))
            return {"requests": len(self._done), "kpoints": self._kpoints_done,
                    "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
                    "kpoints_per_s": self._kpoints_done / span if span and span > 0 else None,
                    "span_s": span, "peak_admitted_bytes": self.peak_used,
                    "budget_bytes": self.budget,
                    "max_concurrent_units": self.max_concurrent_units}

    def close(self) -> None:
        with self._lock:
            self._closed = True
            self._lock.notify_all()
        for w in self._workers:
            w.join(timeout=60)
        for res in list(self._resources.values()) + list(self._pending.values()):
            close = getattr(res, "close", None)
            if close is not None:
                close()
        self._resources.clear()
        self._pending.clear()

    def __enter__(self) -> "BandServer":
        return self

    def __exit__(self, *exc: Any) -> None:
        self.close()

    # ------------------------------------------------------------- internals
    def _admit_locked(self) -> None:
        """Admit waiting requests that fit (arrival order, with backfill);
        when a request still waits for memory, resident bundles that no
        admitted or waiting request uses are evicted and admission is tried
        once more."""
        self._admit_pass_locked()
        if self._waiting and len(self._active) < self.slots and self._evict_idle_locked():
            self._admit_pass_locked()

    def _admit_pass_locked(self) -> None:
        for act in list(self._waiting):
            if len(self._active) >= self.slots:
                break
            try:
                res = self._resources.get(act.bundle_key) or self._pending.get(act.bundle_key)
                fresh = res is None
                if fresh:
                    res = self._resources_factory(act.req.bundle, self.device,
                                                  self._tile(act.req))
                resident, working = self._footprint(act.req, res, self.kpoints_per_unit)
            except Exception as exc:  # noqa: BLE001 - reported through the future
                self._waiting.remove(act)
                act.future.set_exception(exc)
                continue
            extra = working + (resident if act.bundle_key not in self._resident_bytes else 0)
            if resident + working > self.budget:
                self._waiting.remove(act)
                if act.bundle_key not in self._resident_bytes:
                    self._pending.pop(act.bundle_key, None)
                    if not self._waiting_for(act.bundle_key):
                        getattr(res, "close", lambda: None)()
                act.future.set_exception(InputError(
                    f"band request needs {resident + working} device bytes, more than the "
                    f"server budget of {self.budget}"))
                continue
            if self._used + extra > self.budget:
                # host-side analysis is kept for the next attempt; no device
                # memory is held until admission
                self._pending[act.bundle_key] = res
                continue   # later (smaller) requests may still fit
            self._waiting.remove(act)
            self._pending.pop(act.bundle_key, None)
            self._resources[act.bundle_key] = res
            if act.bundle_key not in self._resident_bytes:
                self._resident_bytes[act.bundle_key] = resident
            self._bundle_users[act.bundle_key] = self._bundle_users.get(act.bundle_key, 0) + 1
            act.footprint = working
            act.admitted = self.clock()
            self._used += extra
            self.peak_used = max(self.peak_used, self._used)
            self._active.append(act)

    def _release_locked(self, act: _Active) -> None:
        self._active.remove(act)
        self._used -= act.footprint
        # the bundle stays resident after its last user while memory allows;
        # _evict_idle_locked drops it when a waiting request needs the room
        self._bundle_users[act.bundle_key] -= 1
        if act.engine is not None and act.engine != "pending":
            getattr(act.engine, "close", lambda: None)()
            act.engine = None

    def _waiting_for(self, key: int) -> bool:
        return any(w.bundle_key == key for w in self._waiting)

    def _evict_idle_locked(self) -> bool:
        """Drop resident bundles that no admitted or waiting request uses;
        True when memory was freed."""
        freed = False
        for key in list(self._resources):
            if self._bundle_users.get(key, 0) > 0 or self._waiting_for(key):
                continue
            res = self._resources.pop(key)
            self._used -= self._resident_bytes.pop(key, 0)
            self._bundle_users.pop(key, None)
            getattr(res, "close", lambda: None)()
            freed = True
        return freed

    def _tile(self, req: BandRequest) -> int:
        from .engine import choose_tile

        es = self.engine_settings
        use_tc = es.precision == "mixed" and es.tensor_cores
        return es.tile or (128 if use_tc else choose_tile(req.bundle.n_orbitals))

    def _next_unit_locked(self):
        if not self._active:
            return None
        start = next(self._rr)
        n = len(self._active)
        for j in range(n):
            act = self._active[(start + j) % n]
            # one unit in flight per request: a request's engine (and its
            # scratch buffers and working set) serves one stream at a time
            if act.units and act.failed is None and act.in_flight == 0:
                return act, act.units.popleft()
        return None

    def _worker(self) -> None:
        stream = None
        while True:
            with self._lock:
                unit = None
                while unit is None:
                    if self._closed and not self._active and not self._waiting:
                        return
                    self._admit_locked()
                    unit = self._next_unit_locked()
                    if unit is None:
                        if self._closed:
                            return
                        self._lock.wait(timeout=0.5)
                act, (first, kpts) = unit
                act.in_flight += 1
                self._running_units += 1
                self.max_concurrent_units = max(self.max_concurrent_units, self._running_units)
                if act.engine is None:
                    act.engine = "pending"
                    build = True
                else:
                    build = False
            try:
                if stream is None:
                    stream = self._stream_factory()
                if build:
                    eng = self._make_engine(act)
                    with self._lock:
                        act.engine = eng
                        self._lock.notify_all()
                else:
                    with self._lock:
                        while act.engine == "pending":
                            self._lock.wait(timeout=0.5)
                        eng = act.engine
                res = _run_on(stream, eng, kpts, act.req.interval)
                err = None
            except BaseException as exc:  # noqa: BLE001 - propagated to the request
                res, err = None, exc
            with self._lock:
                self._running_units -= 1
                act.in_flight -= 1
                if err is not None:
                    act.failed = act.failed or err
                    if act.engine == "pending":
                        act.engine = None
                else:
                    act.results[first] = res
                if act.in_flight == 0 and (not act.units or act.failed is not None):
                    self._finish_locked(act)
                self._lock.notify_all()

    def _make_engine(self, act: _Active):
        res = self._resources[act.bundle_key]
        working = act.footprint
        settings = self.engine_settings
        cap = getattr(res, "pencil_cap", None)
        cap = cap(act.req, working, self.kpoints_per_unit) if callable(cap) else _pencil_cap(
            act.req, res, working, self.kpoints_per_unit)
        es = replace(settings, max_pencils=max(1, int(cap)))
        return self._engine_factory(act.req, res, es, self.device)

    def _finish_locked(self, act: _Active) -> None:
        now = self.clock()
        self._release_locked(act)
        if act.failed is not None:
            act.future.set_exception(act.failed)
            return
        energies, worst, warns = [], 0.0, []
        for first in sorted(act.results):
            for r in act.results[first]:
                energies.append(np.asarray(r.energies_ev))
                worst = max(worst, float(r.maximum_residual_ev))
                warns.extend(r.warnings)
        resp = BandResponse(act.req.request_id, energies, worst, now - act.arrival,
                            act.admitted - act.arrival, len(energies), tuple(dict.fromkeys(warns)))
        self._done.append(resp)
        self._kpoints_done += len(energies)
        self._last_done = now
        act.future.set_result(resp)


# ----------------------------------------------------------------- GPU side
def _gpu_stream(device: Any):
    import torch

    return torch.cuda.Stream(device=device)


def _run_on(stream: Any, engine: Any, kpts: np.ndarray, interval: EnergyInterval):
    if stream is None or not hasattr(stream, "cuda_stream"):
        return engine.solve_kpoints(kpts, interval)[0]
    import torch

    with torch.cuda.device(stream.device), torch.cuda.stream(stream):
        out = engine.solve_kpoints(kpts, interval)[0]
        stream.synchronize()
    return out


def _default_budget(device: Any) -> int:
    try:
        import torch

        if torch.cuda.is_available():
            free, _ = torch.cuda.mem_get_info(device)
            return int(0.8 * free)
    except Exception:  # noqa: BLE001
        pass
    raise SolverError("memory_budget_bytes is required without a CUDA device")


def _gpu_resources(bundle: LocalizedOperatorBundle, device: Any, tile: int):
    from .engine import BundleResources

    return BundleResources(bundle, device if device is not None else "cuda", tile=tile)


def _pairs_per_k(settings: CissSettings) -> int:
    return (settings.integration_points + 1) // 2


def _gpu_footprint(req: BandRequest, res: Any, kpoints_per_unit: int) -> tuple[int, int]:
    from . import native

    st = req.settings
    info = res.plan.info
    lib = native.library()
    L, M = st.block_size, st.moment_size
    per_pencil = (lib.aosb_factor_bytes(res.plan.handle, 1) + 4 * info.n_pad + 4
                  + 8 * info.n_pad * L * 2 + 16 * info.n * L * 3
                  + lib.aosb_factor_workspace_bytes(res.plan.handle, 1, native.PRECISION_BF16X3)
                  + lib.aosb_solve_scratch_bytes(res.plan.handle, 1, L))
    nk = kpoints_per_unit
    pencils = nk * _pairs_per_k(st)
    per_k = 2 * 8 * info.nnz + 16 * info.n * (L * M * 2 + L)   # H, S values, moments, rhs
    working = pencils * per_pencil + nk * per_k + 64 * 2**20   # + small buffers and slack
    return res.resident_bytes(), int(working)


def _pencil_cap(req: BandRequest, res: Any, working: int, kpoints_per_unit: int) -> int:
    return kpoints_per_unit * _pairs_per_k(req.settings)


def _gpu_engine(req: BandRequest, res: Any, es: EngineSettings, device: Any):
    from .engine import BandEngine

    return BandEngine(None, req.settings, es, device=device, resources=res)
