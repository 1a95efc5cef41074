"""Host-side Band path: bundle format, data validation, k paths, settings,
checkpoints and output files (no GPU)."""

from __future__ import annotations

import csv
import json
from dataclasses import fields

import numpy as np
import pytest

import bundles
from aospectrum_b200 import synth
from aospectrum_b200.band import (
    BandPoint,
    BandResult,
    assign_track_ids,
    read_point,
    resolve_energy_reference,
    summary_dict,
    write_band_output,
    write_point,
)
from aospectrum_b200.bundle import load_bundle, write_bundle
from aospectrum_b200.ciss import CissSettings, EngineSettings
from aospectrum_b200.data import EnergyInterval, LocalizedOperatorBlocks
from aospectrum_b200.errors import InputError
from aospectrum_b200.kpath import KPath, kpath_from_dict


def test_bundle_round_trip(tmp_path):
    b = bundles.tiny3d()
    write_bundle(b, tmp_path / "b")
    r = load_bundle(tmp_path / "b")
    assert r.n_orbitals == b.n_orbitals
    for name in ("row_atom", "col_atom", "lattice_shift", "block_offsets", "block_shapes",
                 "h_values", "s_values"):
        assert np.array_equal(getattr(r.operators, name), getattr(b.operators, name))
    assert r.structure.periodic == b.structure.periodic
    assert r.basis.basis_identity == b.basis.basis_identity
    with pytest.raises(InputError):
        write_bundle(b, tmp_path / "b")


def test_bundle_rejects_bad_schema(tmp_path):
    b = bundles.tiny2d()
    root = write_bundle(b, tmp_path / "b")
    man = json.loads((root / "manifest.json").read_text())
    man["schema"] = "other/v0"
    (root / "manifest.json").write_text(json.dumps(man))
    with pytest.raises(InputError, match="unsupported operator bundle"):
        load_bundle(root)


def test_block_table_validation():
    ops = bundles.tiny2d().operators
    with pytest.raises(InputError, match="offsets do not match"):
        bad = np.array(ops.block_offsets)
        bad[1] += 1
        LocalizedOperatorBlocks(ops.row_atom, ops.col_atom, ops.lattice_shift, bad,
                                ops.block_shapes, ops.h_values, ops.s_values)
    with pytest.raises(InputError, match="H/S values"):
        LocalizedOperatorBlocks(ops.row_atom, ops.col_atom, ops.lattice_shift,
                                ops.block_offsets, ops.block_shapes, ops.h_values[:-1],
                                ops.s_values[:-1])


def test_synthetic_generator_is_seeded_and_hermitian():
    a, b = bundles.tiny3d(), bundles.tiny3d()
    assert np.array_equal(a.operators.h_values, b.operators.h_values)
    h, s = synth.dense_gamma(a)
    assert np.allclose(h, h.T) and np.allclose(s, s.T)
    assert np.linalg.eigvalsh(s).min() > 0.1


def test_kpath_forms_and_errors():
    kp = kpath_from_dict(synth.YGXM)
    assert kp.n_points == 121 and list(kp.node_indices) == [0, 40, 80, 120]
    d = kp.distances(np.diag([20.0, 20.0, 15.0]))
    assert d[0] == 0 and np.all(np.diff(d) >= 0)
    grid = kpath_from_dict(synth.uniform_grid_kpath(2, 2, 1))
    assert grid.n_points == 4
    with pytest.raises(InputError):
        KPath(np.zeros((2, 3)), [0, 2], ("a", "b"))
    with pytest.raises(InputError):
        kpath_from_dict({"labels": ["a"], "schema": "x"})


def test_cisssettings_matches_reference_fields():
    names = [f.name for f in fields(CissSettings)]
    assert names == ["integration_points", "contour_batch_size", "block_size", "moment_size",
                     "ellipse_vertical_scale", "endpoint_guard_ev", "rank_relative_tolerance",
                     "spurious_relative_threshold", "random_seed"]
    with pytest.raises(InputError):
        CissSettings(integration_points=32, contour_batch_size=5)
    with pytest.raises(InputError):
        EngineSettings(precision="fp16")
    with pytest.raises(InputError):
        EngineSettings(tile=48)


def test_energy_reference_modes():
    b = bundles.tiny2d()
    assert resolve_energy_reference(b, "input_zero") == 0.0
    assert resolve_energy_reference(b, "fixed", 1.5) == 1.5
    with pytest.raises(InputError):
        resolve_energy_reference(b, "bundle_fermi")
    with pytest.raises(InputError):
        resolve_energy_reference(b, "nonsense")


def test_checkpoint_round_trip_and_mismatch(tmp_path):
    p = BandPoint(3, np.array([0.1, 0.2, 0.0]), np.array([-1.0, -0.5]), 1e-5,
                  {"solver_total": 0.3}, 0.01, 1234, ("w",))
    path = tmp_path / "k-000003.npz"
    write_point(path, p)
    q = read_point(path, index=3, k_fractional=np.array([0.1, 0.2, 0.0]))
    assert q.index == 3 and np.array_equal(q.energies_ev, p.energies_ev)
    assert q.stage_seconds == {"solver_total": 0.3} and q.peak_gpu_memory_bytes == 1234
    assert q.warnings == ("w",)
    assert read_point(tmp_path / "none.npz", index=3, k_fractional=p.k_fractional) is None
    with pytest.raises(InputError):
        read_point(path, index=4, k_fractional=p.k_fractional)


def test_track_ids_follow_bands():
    e = [np.array([0.0, 1.0]), np.array([1.05, 0.02]), np.array([0.03, 1.1, 2.0])]
    t = assign_track_ids(e)
    assert list(t[0]) == [0, 1]
    assert list(t[1]) == [1, 0]
    assert list(t[2]) == [0, 1, 2]


def test_band_output_format_matches_reference(tmp_path, golden):
    kp = kpath_from_dict({"schema": "aospectrum.kpath/v1",
                          "nodes_fractional": [[0, 0.5, 0], [0, 0, 0], [0.5, 0, 0]],
                          "labels": ["Y", "G", "X"], "points_per_segment": 3})
    pts = tuple(BandPoint(i, kp.fractional_points[i], np.array([-2.0 + 0.01 * i, -1.5]), 1e-4,
                          {"solver_total": 0.1}, 0.001, None) for i in range(kp.n_points))
    res = BandResult(kp, EnergyInterval(-3.0, -1.0), EnergyInterval(-3.02, -0.98), 0.0,
                     np.diag([7.5, 7.5, 15.0]), pts, 1.0, ("note",))
    out = write_band_output(res, tmp_path / "out")
    mine = list(csv.reader((out / "bands.csv").open()))
    ref = list(csv.reader((golden / "band_tiny2d" / "bands.csv").open()))
    assert mine[0] == ref[0]
    assert len(mine[1][1].split("e")[0].split(".")[1]) == len(ref[1][1].split("e")[0].split(".")[1])
    summary = json.loads((out / "summary.json").read_text())
    ref_summary = json.loads((golden / "band_tiny2d" / "summary.json").read_text())
    assert set(summary) == set(ref_summary)
    assert summary["backend"] == "ciss-b200" and summary["scalar_dtype"] == "complex64"
    assert summary_dict(res)["kpoint_count"] == kp.n_points


def test_parallel_small_eigensolves_match_serial():
    """BandEngine._host_map runs the k points' small FP64 eigenproblems in
    threads under one BLAS thread limit: same results, in order, as the
    serial calls with their own limit; errors propagate."""
    from aospectrum_b200.ciss import projected_eigh, truncate_gram
    from aospectrum_b200.engine import BandEngine
    from aospectrum_b200.errors import SolverError

    eng = BandEngine.__new__(BandEngine)   # host part only: no device state
    eng._lapack_pool = None
    rng = np.random.default_rng(12)
    grams, pencils = [], []
    for _ in range(5):
        m = rng.standard_normal((40, 24)) + 1j * rng.standard_normal((40, 24))
        grams.append(m.conj().T @ m)
        h = rng.standard_normal((24, 24)) + 1j * rng.standard_normal((24, 24))
        pencils.append((h + h.conj().T, grams[-1] + 24 * np.eye(24)))
    par = eng._host_map(lambda g: truncate_gram(g, 1e-5, limit_threads=False), grams)
    for g, (t, s) in zip(grams, par):
        t0, s0 = truncate_gram(g, 1e-5)
        assert np.array_equal(t, t0) and np.array_equal(s, s0)
    par = eng._host_map(lambda p: projected_eigh(p[0], p[1], limit_threads=False), pencils)
    for p, (e, c) in zip(pencils, par):
        e0, c0 = projected_eigh(*p)
        assert np.array_equal(e, e0) and np.array_equal(c, c0)
    with pytest.raises(SolverError):
        eng._host_map(lambda g: truncate_gram(g, 1e-5, limit_threads=False),
                      [grams[0], np.zeros((24, 24), complex)])
    eng._lapack_pool.shutdown()


def test_interval_selection_uses_float32_energies():
    """The reference casts the Ritz energies to float32 before its strict
    interval test (ciss.py:145-150, :355-358): an FP64 energy that lies a
    hair inside a bound but rounds onto it in float32 is dropped, and no
    kept energy equals a bound."""
    from aospectrum_b200.ciss import interval_mask

    iv = EnergyInterval(-2.5, -1.0)
    e = np.array([-2.5 + 1e-9, -2.0, -1.0 - 1e-9, -1.0 - 1e-6])
    got = interval_mask(e, iv)
    e32 = np.asarray(e, dtype=np.float32)
    ref = np.logical_and(e32 > iv.lower_ev, e32 < iv.upper_ev)
    assert np.array_equal(got, ref)
    assert got.tolist() == [False, True, False, True]
    kept = np.asarray(e[got], dtype=np.float32)
    assert not np.any(kept == np.float32(iv.lower_ev)) and not np.any(kept == np.float32(iv.upper_ev))
