"""The drop-in Band application end to end on the GPU: `aospectrum band`
(cli.run_band) with the real engine on the reference's own tiny2d case,
compared with the bands.csv / summary.json that the reference's run_band
wrote for the same inputs (tests/golden/band_tiny2d, made by
tests/golden/make_golden.py).  Eigenvalues within the 1e-4 eV tolerance of
the parity tests, the same k points and track layout, and a maximum
eigenpair residual no worse than the reference's."""

from __future__ import annotations

import csv
import json
import shutil
from pathlib import Path

import pytest

import bundles
from aospectrum_b200 import cli
from aospectrum_b200.bundle import write_bundle

pytestmark = pytest.mark.gpu

EIG_TOL_EV = 1e-4

TOML = """[input]
bundle = "system.aobundle"
[band]
kpath = "path.json"
energy_interval_ev = [-3.0, -1.0]
energy_reference = "input_zero"
[solver]
integration_points = 16
block_size = 8
moment_size = 4
{extra}[output]
directory = "out"
"""


@pytest.mark.parametrize("precision", ["mixed", "plain"])
def test_cli_band_run_matches_reference_outputs(tmp_path, golden, precision):
    write_bundle(bundles.tiny2d(), tmp_path / "system.aobundle")
    shutil.copy(golden / "band_tiny2d" / "path.json", tmp_path / "path.json")
    extra = f'precision = "{precision}"\n' if precision != "mixed" else ""
    (tmp_path / "band.toml").write_text(TOML.format(extra=extra))
    out = cli.run_band(tmp_path / "band.toml")
    mine = list(csv.reader((out / "bands.csv").open()))
    ref = list(csv.reader((golden / "band_tiny2d" / "bands.csv").open()))
    assert mine[0] == ref[0] and len(mine) == len(ref)
    for a, b in zip(mine[1:], ref[1:]):
        assert a[0] == b[0] and a[1] == b[1] and a[2] == b[2]
        assert abs(float(a[3]) - float(b[3])) < EIG_TOL_EV
    summary = json.loads((out / "summary.json").read_text())
    ref_sum = json.loads((golden / "band_tiny2d" / "summary.json").read_text())
    assert summary["kpoint_count"] == ref_sum["kpoint_count"]
    assert summary["energy_interval_ev"] == ref_sum["energy_interval_ev"]
    assert summary["scalar_dtype"] == "complex64"
    assert (summary["maximum_eigenpair_residual_ev"]
            <= ref_sum["maximum_eigenpair_residual_ev"] * 1.01)
    assert not (tmp_path / ".out.work").exists()
