"""Host logic of the continuous-batching Band server (aospectrum_b200.serve):
admission by device footprint, backfill, rejection of oversized requests,
overlap of units from different requests, per-request failure, latency
percentiles, and identical results alone and in the mix.  The engine is the
CPU oracle stand-in; the GPU form of the same checks is in
test_gpu_serve.py."""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

import bundles
from aospectrum_b200.ciss import CissSettings, EngineSettings
from aospectrum_b200.data import EnergyInterval
from aospectrum_b200.errors import InputError
from aospectrum_b200.serve import BandRequest, BandServer, percentile
from fake_engine import OracleEngine


class FakeResources:
    closed = 0

    def __init__(self, bundle):
        self.bundle = bundle

    def close(self):
        FakeResources.closed += 1


class SlowOracle(OracleEngine):
    """Oracle engine that records how many units run at once."""

    running = 0
    peak = 0
    lock = threading.Lock()
    failing: set[int] = set()   # ids of bundles whose units raise

    def solve_kpoints(self, kpoints, interval):
        with SlowOracle.lock:
            SlowOracle.running += 1
            SlowOracle.peak = max(SlowOracle.peak, SlowOracle.running)
            # an engine (one request) must never serve two units at once
            assert not getattr(self, "_busy", False), "engine used by two units at once"
            self._busy = True
        try:
            time.sleep(0.02)
            if id(self.bundle) in SlowOracle.failing:
                raise RuntimeError("injected unit failure")
            return super().solve_kpoints(kpoints, interval)
        finally:
            with SlowOracle.lock:
                SlowOracle.running -= 1
                self._busy = False


def _server(budget, footprints, slots=3, **kw):
    """footprints: bundle id -> (resident, working)."""
    return BandServer(
        memory_budget_bytes=budget, slots=slots, kpoints_per_unit=1,
        engine_settings=EngineSettings(precision="plain"),
        engine_factory=lambda req, res, es, dev: SlowOracle(req.bundle, req.settings, es),
        resources_factory=lambda bundle, dev, tile: FakeResources(bundle),
        footprint_fn=lambda req, res, nk: footprints[id(req.bundle)],
        stream_factory=lambda: None, **kw)


SETTINGS = CissSettings(integration_points=8, block_size=4, moment_size=2)
LO, HI = -3.0, -1.5


def _req(bundle, ks, rid):
    return BandRequest(bundle, [bundles.KPOINTS[i] for i in ks], EnergyInterval(LO, HI),
                       SETTINGS, rid)


def test_percentile_nearest_rank():
    v = [5.0, 1.0, 3.0, 2.0, 4.0]
    assert percentile(v, 50) == 3.0
    assert percentile(v, 99) == 5.0
    assert percentile(v, 0) == 1.0
    assert np.isnan(percentile([], 50))


def test_results_alone_equal_results_in_mix():
    b1, b2 = bundles.tiny2d(), bundles.tiny3d()
    fp = {id(b1): (10, 20), id(b2): (10, 20)}
    alone = {}
    for name, b, ks in (("a", b1, [0, 1, 2]), ("b", b2, [1, 2]), ("c", b1, [2, 0])):
        with _server(1000, fp, slots=1) as srv:
            alone[name] = srv.submit(_req(b, ks, name)).result(timeout=120)
    SlowOracle.peak = 0
    with _server(1000, fp, slots=3) as srv:
        futs = {"a": srv.submit(_req(b1, [0, 1, 2], "a"))}
        time.sleep(0.01)   # later arrivals join while "a" runs
        futs["b"] = srv.submit(_req(b2, [1, 2], "b"))
        futs["c"] = srv.submit(_req(b1, [2, 0], "c"))
        mixed = {k: f.result(timeout=120) for k, f in futs.items()}
        stats = srv.stats()
    assert SlowOracle.peak >= 2          # units of different requests overlapped
    for k in alone:
        assert len(alone[k].energies_ev) == len(mixed[k].energies_ev)
        for ea, em in zip(alone[k].energies_ev, mixed[k].energies_ev):
            np.testing.assert_allclose(np.sort(em), np.sort(ea), rtol=0, atol=1e-4)
    assert stats["requests"] == 3 and stats["kpoints"] == 7
    assert stats["p50_latency_s"] <= stats["p99_latency_s"]
    assert stats["kpoints_per_s"] > 0


def test_admission_by_footprint_and_backfill():
    big, small = bundles.tiny3d(), bundles.tiny2d()
    # the budget holds one big request or two small ones, never big + small
    fp = {id(big): (10, 80), id(small): (5, 30)}
    SlowOracle.peak = 0
    with _server(100, fp, slots=4) as srv:
        f1 = srv.submit(_req(small, [0, 1, 2, 0], "s1"))
        f2 = srv.submit(_req(big, [1], "big"))          # does not fit next to s1
        f3 = srv.submit(_req(small, [1, 2], "s2"))      # fits: backfills past big
        r1, r2, r3 = (f.result(timeout=120) for f in (f1, f2, f3))
        st = srv.stats()
    assert st["peak_admitted_bytes"] <= 100
    assert r3.queue_seconds <= r2.queue_seconds
    assert r2.kpoints == 1 and r1.kpoints == 4 and r3.kpoints == 2


def test_oversized_request_rejected_and_others_served():
    b1, b2 = bundles.tiny2d(), bundles.tiny3d()
    fp = {id(b1): (10, 20), id(b2): (10, 500)}
    with _server(100, fp) as srv:
        bad = srv.submit(_req(b2, [0], "huge"))
        good = srv.submit(_req(b1, [0], "ok"))
        with pytest.raises(InputError, match="server budget"):
            bad.result(timeout=60)
        assert good.result(timeout=120).kpoints == 1


def test_unit_failure_reaches_only_its_request():
    ok, broken = bundles.tiny2d(), bundles.tiny3d()
    SlowOracle.failing.add(id(broken))
    fp = {id(ok): (10, 20), id(broken): (10, 20)}
    with _server(1000, fp) as srv:
        fb = srv.submit(_req(broken, [0, 1], "broken"))
        fo = srv.submit(_req(ok, [0, 1], "ok"))
        with pytest.raises(RuntimeError, match="injected unit failure"):
            fb.result(timeout=120)
        assert fo.result(timeout=120).kpoints == 2
        srv.drain(timeout=60)
    SlowOracle.failing.discard(id(broken))


def test_submit_validates_kpoints():
    with _server(100, {}) as srv:
        with pytest.raises(InputError):
            srv.submit(BandRequest(bundles.tiny2d(), [], EnergyInterval(LO, HI), SETTINGS))
        with pytest.raises(InputError):
            srv.submit(BandRequest(bundles.tiny2d(), [[0.0, 0.0]], EnergyInterval(LO, HI),
                                   SETTINGS))
