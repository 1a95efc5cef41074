"""Parity at the benched workload (c2: 1000 atoms, n = 13000, nnz 15.7M,
3D periodic; the 32-node contour, 32 probes and 4 moments of the bench)
against golden vectors the reference itself produced
(tests/golden/make_golden.py --c2): at two k points of the Y-G-X-M path,
the reference's BlochWorkspace.update digests (bit-exact), FP64 dense
generalized eigenvalues in the solve interval, and the reference's own
complex64 CISS (src/aospectrum/ciss.py:266-391) run with exact complex128
shifted solves -- its eigenvalues and maximum eigenpair residual.

Both forms of this engine -- mixed (split-BF16 tensor-core factorization,
FP64 refinement, node pairs) and plain (complex64, one factorization per
node, no refinement) -- must give every eigenvalue within 1e-4 eV of the
FP64 oracle and of the reference.  The chosen (mixed) form's maximum
residual must be no worse than the reference's (1 % slack for rounding of
the residual itself).  The plain form factors in complex64 and does not
refine its solves, while the reference here ran with exact solves; its
residual may exceed the reference's by at most 5 % (measured: 1.0 % at k
point 0, below the reference's at k point 37)."""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EIG_TOL_EV = 1e-4


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def c2(golden):
    import torch

    from aospectrum_b200 import synth
    from aospectrum_b200.kpath import kpath_from_dict

    torch.cuda.set_device(0)
    man = json.loads((golden / "manifest_c2.json").read_text())
    ref = np.load(golden / "c2.npz")
    w = synth.WORKLOADS["c2"]
    return {"man": man, "ref": ref, "w": w, "bundle": synth.generate_bundle(w.spec),
            "kpts": kpath_from_dict(w.kpath).fractional_points}


def test_c2_bloch_matches_reference_digests(c2):
    import torch

    from aospectrum_b200.engine import BlochDevice

    dev = BlochDevice(c2["bundle"], torch.device("cuda", 0))
    try:
        man = c2["man"]
        assert dev.nnz == man["nnz"]
        assert _sha(dev.indptr.astype(np.int32)) == man["indptr"]
        assert _sha(dev.indices) == man["indices"]
        for key, rec in man["kpoints"].items():
            h, s = dev.apply(np.asarray([c2["kpts"][int(key)]]))
            assert _sha(h[0].cpu().numpy()) == rec["h"], f"H(k{key}) differs"
            assert _sha(s[0].cpu().numpy()) == rec["s"], f"S(k{key}) differs"
    finally:
        dev.close()


@pytest.mark.parametrize("precision", ["mixed", "plain"])
def test_c2_ciss_matches_reference_and_fp64(c2, precision):
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine

    w = c2["w"]
    lo, hi = c2["man"]["interval"]
    eng = BandEngine(c2["bundle"], CissSettings(integration_points=w.integration_points,
                                                block_size=w.block_size,
                                                moment_size=w.moment_size),
                     EngineSettings(precision=precision))
    try:
        for key, rec in c2["man"]["kpoints"].items():
            res, _ = eng.solve_kpoints([c2["kpts"][int(key)]], EnergyInterval(lo, hi))
            got = np.sort(res[0].energies_ev.astype(np.float64))
            exact = np.sort(c2["ref"][f"k{key}_fp64"])
            ref = np.sort(c2["ref"][f"k{key}_energies"].astype(np.float64))
            assert got.size == exact.size == ref.size, (key, got.size, exact.size, ref.size)
            assert np.max(np.abs(got - exact)) < EIG_TOL_EV, key
            assert np.max(np.abs(got - ref)) < EIG_TOL_EV, key
            slack = 1.01 if precision == "mixed" else 1.05
            assert res[0].maximum_residual_ev <= rec["max_residual_ev"] * slack, (
                key, res[0].maximum_residual_ev, rec["max_residual_ev"])
    finally:
        eng.close()
