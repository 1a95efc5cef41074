"""CPU stand-in for BandEngine used by host-logic tests only: H(k), S(k) and
the CISS result come from the oracle (reference algorithm on the host)."""

from __future__ import annotations

import os
from time import perf_counter

import numpy as np
from scipy import sparse

from aospectrum_b200.ciss import CissResult
from aospectrum_b200.sparse import SparsePair
from oracle import bloch_ref, ciss_ref


class OracleEngine:
    calls = 0

    def __init__(self, bundle, settings, engine_settings):
        self.bundle = bundle
        self.settings = settings
        self.pattern = bloch_ref.build_pattern(bundle)
        # fail after this many solved k points (host-side fault injection)
        self.fail_after = int(os.environ.get("AOSB_TEST_FAIL_AFTER", "-1"))
        self.solved = 0

    def host_pair(self, k):
        h, s = bloch_ref.bloch_pair(self.pattern, self.bundle, k)
        n = self.bundle.n_orbitals
        ip = self.pattern.indptr.astype(np.int32)
        ix = self.pattern.indices.astype(np.int32)
        return SparsePair(sparse.csr_matrix((h, ix, ip), shape=(n, n)),
                          sparse.csr_matrix((s, ix, ip), shape=(n, n)), tuple(k))

    def solve_kpoints(self, kpoints, interval):
        out, asm = [], []
        for k in kpoints:
            if 0 <= self.fail_after <= self.solved:
                raise RuntimeError("injected host failure")
            t0 = perf_counter()
            pair = self.host_pair(k)
            asm.append(perf_counter() - t0)
            st = self.settings
            r = ciss_ref.solve_interval(pair.hamiltonian, pair.overlap, interval.lower_ev,
                                        interval.upper_ev, n_points=st.integration_points,
                                        block=st.block_size, moments=st.moment_size)
            self.solved += 1
            OracleEngine.calls += 1
            out.append(CissResult(r.energies, r.max_residual, {"solver_total": 0.0}, None, (),
                                  not r.saturated))
        return out, asm

    def close(self):
        pass


def factory(bundle, settings, engine_settings):
    return OracleEngine(bundle, settings, engine_settings)
