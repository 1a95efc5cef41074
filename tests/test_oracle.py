"""The oracle pinned against golden vectors produced by the reference's own
Python package (tests/golden/make_golden.py)."""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

import bundles
from aospectrum_b200.ciss import CissSettings, contour_geometry, probe_block
from aospectrum_b200.data import EnergyInterval
from aospectrum_b200.kpath import kpath_from_dict
from aospectrum_b200 import synth
from oracle import bloch_c, bloch_ref, ciss_ref, dense_ref


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _bundle(name):
    return bundles.complexified(bundles.tiny2d()) if name == "tinycx" else getattr(bundles, name)()


@pytest.mark.parametrize("name", ["tiny2d", "tiny3d", "tinycx"])
def test_numpy_oracle_bloch_is_bit_exact(name, golden):
    ref = np.load(golden / f"bloch_{name}.npz")
    b = _bundle(name)
    pat = bloch_ref.build_pattern(b)
    assert np.array_equal(pat.indptr, ref["indptr"])
    assert np.array_equal(pat.indices, ref["indices"])
    for i, k in enumerate(bundles.KPOINTS):
        h, s = bloch_ref.bloch_pair(pat, b, k)
        assert np.array_equal(h, ref[f"h{i}"]) and np.array_equal(s, ref[f"s{i}"])


@pytest.mark.parametrize("name", ["tiny2d", "tiny3d", "tinycx"])
def test_c_oracle_bloch_matches_reference(name, golden):
    ref = np.load(golden / f"bloch_{name}.npz")
    b = _bundle(name)
    pat = bloch_ref.build_pattern(b)
    for i, k in enumerate(bundles.KPOINTS):
        h = bloch_c.bloch_values(pat, b.operators.h_values, k)
        s = bloch_c.bloch_values(pat, b.operators.s_values, k)
        if name == "tinycx":
            np.testing.assert_allclose(h, ref[f"h{i}"], rtol=0, atol=2e-6)
            np.testing.assert_allclose(s, ref[f"s{i}"], rtol=0, atol=2e-7)
        else:
            assert np.array_equal(h, ref[f"h{i}"]) and np.array_equal(s, ref[f"s{i}"])


def test_oracle_bloch_digests_small2d_and_c1(golden):
    man = json.loads((golden / "manifest.json").read_text())["bloch"]
    for name, b in (("small2d", bundles.small2d()), ("c1", bundles.c1())):
        pat = bloch_ref.build_pattern(b)
        for i, k in enumerate(bundles.KPOINTS):
            h, s = bloch_ref.bloch_pair(pat, b, k)
            assert _sha(h) == man[name][f"h{i}"] and _sha(s) == man[name][f"s{i}"]


def test_contour_geometry_is_bit_exact(golden):
    g = np.load(golden / "contour.npz")
    for i in range(3):
        lo, hi, npts = g[f"interval{i}"]
        mine = contour_geometry(EnergyInterval(lo, hi), CissSettings(integration_points=int(npts)))
        orc = ciss_ref.contour(lo, hi, int(npts))
        for a, b, key in zip(mine, orc, ("shifts", "nodes", "weights")):
            assert np.array_equal(a, g[f"{key}{i}"])
            assert np.array_equal(b, g[f"{key}{i}"])


@pytest.mark.parametrize("key", ["tiny3d_k2", "small2d_k2", "tinycx_k1"])
def test_probe_rhs_matches_reference(key, golden):
    case = json.loads((golden / "manifest.json").read_text())["ciss"][key]
    rhs_ref = np.load(golden / "ciss.npz")[f"{key}_rhs"]
    b = _bundle(case["bundle"])
    pat = bloch_ref.build_pattern(b)
    h, s = bloch_ref.bloch_pair(pat, b, bundles.KPOINTS[case["k_index"]])
    from scipy import sparse

    n = b.n_orbitals
    sm = sparse.csr_matrix((s, pat.indices, pat.indptr), shape=(n, n))
    q = probe_block(n, CissSettings(block_size=case["block_size"]))
    assert np.array_equal(q, ciss_ref.probes(n, case["block_size"]))
    np.testing.assert_allclose(np.asarray(sm @ q, dtype=np.complex64), rhs_ref, rtol=0, atol=1e-6)


@pytest.mark.parametrize("key", ["tiny3d_k2", "small2d_k2", "tinycx_k1", "c1_k0", "c1_k2"])
def test_ciss_oracle_matches_reference(key, golden):
    case = json.loads((golden / "manifest.json").read_text())["ciss"][key]
    ref_e = np.sort(np.load(golden / "ciss.npz")[f"{key}_energies"])
    b = _bundle(case["bundle"])
    pat = bloch_ref.build_pattern(b)
    h, s = bloch_ref.bloch_pair(pat, b, bundles.KPOINTS[case["k_index"]])
    from scipy import sparse

    n = b.n_orbitals
    hm = sparse.csr_matrix((h, pat.indices, pat.indptr), shape=(n, n))
    sm = sparse.csr_matrix((s, pat.indices, pat.indptr), shape=(n, n))
    lo, hi = case["interval"]
    r = ciss_ref.solve_interval(hm, sm, lo, hi, n_points=case["integration_points"],
                                block=case["block_size"], moments=case["moment_size"])
    assert r.energies.size == ref_e.size == case["count"]
    assert np.max(np.abs(np.sort(r.energies) - ref_e)) < 2e-6
    assert abs(r.max_residual - case["max_residual_ev"]) <= 0.05 * case["max_residual_ev"] + 1e-6
    # and the FP64 dense oracle agrees within 1e-4 eV
    hd, sd = dense_ref.dense_pair(pat.indptr, pat.indices, h, s, n)
    exact = dense_ref.window(dense_ref.eigenvalues(hd, sd), lo, hi)
    assert exact.size == ref_e.size
    assert np.max(np.abs(exact - ref_e)) < 1e-4


def test_kpath_matches_reference(golden):
    g = np.load(golden / "kpath_ygxm.npz")
    kp = kpath_from_dict(synth.YGXM)
    assert np.array_equal(kp.fractional_points, g["points"])
    assert np.array_equal(kp.node_indices, g["nodes"])
    assert list(kp.node_labels) == list(g["labels"])
    assert kp.n_points == 121
