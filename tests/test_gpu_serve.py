"""The continuous-batching Band server on the GPU: requests over three
different bundles, each solved alone and then together with staggered
arrivals (their work units overlap on separate CUDA streams).  Each
request's eigenvalues must be the same alone and in the mix within the
eigenvalue tolerance of the parity tests (1e-4 eV), and the admitted
footprint must stay inside the budget."""

from __future__ import annotations

import time

import numpy as np
import pytest

import bundles
from aospectrum_b200.ciss import CissSettings, EngineSettings
from aospectrum_b200.data import EnergyInterval
from aospectrum_b200.serve import BandRequest, BandServer

pytestmark = pytest.mark.gpu

EIG_TOL_EV = 1e-4
SETTINGS = CissSettings(integration_points=16, block_size=8, moment_size=4)


@pytest.fixture(scope="module")
def torch():
    import torch as t

    return t


def _requests():
    b_tiny, b_small, b_c1 = bundles.tiny3d(), bundles.small2d(), bundles.c1()
    return [
        ("tiny3d", b_tiny, [0, 1, 2], (-3.2, -1.6)),
        ("small2d", b_small, [1, 2], (-2.6, -2.2)),
        ("c1", b_c1, [0, 3], (-3.0296 - 0.02, -2.2616 + 0.02)),
    ]


def _submit(srv, name, b, ks, win):
    return srv.submit(BandRequest(b, [bundles.KPOINTS[i] for i in ks], EnergyInterval(*win),
                                  SETTINGS, name))


def test_server_results_same_alone_and_in_mix(torch):
    dev = torch.device("cuda", 0)
    es = EngineSettings(precision="mixed")
    reqs = _requests()
    alone = {}
    with BandServer(device=dev, slots=1, engine_settings=es,
                    memory_budget_bytes=8 * 2**30) as srv:
        for name, b, ks, win in reqs:
            alone[name] = _submit(srv, name, b, ks, win).result(timeout=600)
    with BandServer(device=dev, slots=3, engine_settings=es,
                    memory_budget_bytes=8 * 2**30) as srv:
        futs = {}
        for name, b, ks, win in reqs:
            futs[name] = _submit(srv, name, b, ks, win)
            time.sleep(0.05)
        mixed = {k: f.result(timeout=600) for k, f in futs.items()}
        stats = srv.stats()
    for name in alone:
        a, m = alone[name], mixed[name]
        assert a.kpoints == m.kpoints
        for ea, em in zip(a.energies_ev, m.energies_ev):
            assert ea.size == em.size and ea.size > 0
            np.testing.assert_allclose(np.sort(em), np.sort(ea), rtol=0, atol=EIG_TOL_EV)
    assert stats["requests"] == 3
    assert stats["peak_admitted_bytes"] <= 8 * 2**30
    assert stats["p50_latency_s"] <= stats["p99_latency_s"]
