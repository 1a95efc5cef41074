"""The `aospectrum band` application on CPU with an oracle-backed engine:
config parsing, run.json compatibility, outputs, resume after a host-side
failure, and the multi-rank split (gloo, world size 2)."""

from __future__ import annotations

import csv
import json
import os
import shutil
import socket
from pathlib import Path

import numpy as np
import pytest

import bundles
import fake_engine
from aospectrum_b200 import cli
from aospectrum_b200.bundle import write_bundle
from aospectrum_b200.errors import InputError, SolverError

GOLDEN_TOML = """[input]
bundle = "system.aobundle"
[band]
kpath = "path.json"
energy_interval_ev = [-3.0, -1.0]
energy_reference = "input_zero"
[solver]
integration_points = 16
block_size = 8
moment_size = 4
[output]
directory = "out"
"""


def make_case(tmp_path: Path, golden: Path, extra: str = "") -> Path:
    write_bundle(bundles.tiny2d(), tmp_path / "system.aobundle")
    shutil.copy(golden / "band_tiny2d" / "path.json", tmp_path / "path.json")
    (tmp_path / "band.toml").write_text(GOLDEN_TOML + extra)
    return tmp_path / "band.toml"


def test_config_keys_and_defaults(tmp_path, golden):
    cfg = cli.read_band_config(make_case(tmp_path, golden))
    assert cfg.settings.integration_points == 16 and cfg.settings.block_size == 8
    assert cfg.devices == (0,) and cfg.engine.precision == "mixed"
    assert cfg.work.name == ".out.work"
    (tmp_path / "bad.toml").write_text(GOLDEN_TOML.replace("[-3.0, -1.0]", "[1.0]"))
    with pytest.raises(InputError):
        cli.read_band_config(tmp_path / "bad.toml")
    (tmp_path / "bad2.toml").write_text(GOLDEN_TOML + "[compute]\ndevices = [0, 0]\n")
    with pytest.raises(InputError):
        cli.read_band_config(tmp_path / "bad2.toml")


def test_run_spec_keeps_reference_keys(tmp_path, golden):
    cfg = cli.read_band_config(make_case(tmp_path, golden))
    spec = cli.band_specification(cfg, bundles.tiny2d())
    assert set(spec) == {"kind", "bundle", "basis_identity", "n_orbitals", "interval_ev",
                         "reference", "kpoints", "nodes", "labels", "solver"}
    assert len(spec["solver"]) == 9  # default engine knobs are not recorded
    cfg2 = cli.read_band_config(make_case(tmp_path / "x", golden,
                                          '\nprecision = "plain"\n'.replace("\n", "\n", 1)))
    assert cfg2.engine.precision == "mixed"  # key outside [solver] is ignored


def test_band_run_reproduces_reference_outputs(tmp_path, golden):
    out = cli.run_band(make_case(tmp_path, golden), engine_factory=fake_engine.factory)
    mine = list(csv.reader((out / "bands.csv").open()))
    ref = list(csv.reader((golden / "band_tiny2d" / "bands.csv").open()))
    assert mine[0] == ref[0] and len(mine) == len(ref)
    for a, b in zip(mine[1:], ref[1:]):
        assert a[0] == b[0] and a[2] == b[2] and a[1] == b[1]
        assert abs(float(a[3]) - float(b[3])) < 2e-6
    summary = json.loads((out / "summary.json").read_text())
    ref_sum = json.loads((golden / "band_tiny2d" / "summary.json").read_text())
    assert summary["kpoint_count"] == ref_sum["kpoint_count"]
    assert summary["energy_interval_ev"] == ref_sum["energy_interval_ev"]
    assert not (tmp_path / ".out.work").exists()


def test_resume_after_host_failure(tmp_path, golden, monkeypatch):
    cfg_path = make_case(tmp_path, golden)
    monkeypatch.setenv("AOSB_TEST_FAIL_AFTER", "3")
    with pytest.raises(RuntimeError, match="injected"):
        cli.run_band(cfg_path, engine_factory=fake_engine.factory)
    work = tmp_path / ".out.work"
    assert len(list(work.glob("k-*.npz"))) == 3
    with pytest.raises(InputError, match="use --resume"):
        cli.run_band(cfg_path, engine_factory=fake_engine.factory)
    monkeypatch.delenv("AOSB_TEST_FAIL_AFTER")
    before = fake_engine.OracleEngine.calls
    out = cli.run_band(cfg_path, resume=True, engine_factory=fake_engine.factory)
    assert fake_engine.OracleEngine.calls - before == 4  # only the missing points
    assert (out / "bands.csv").exists()


def test_resume_rejects_other_calculation(tmp_path, golden, monkeypatch):
    cfg_path = make_case(tmp_path, golden)
    monkeypatch.setenv("AOSB_TEST_FAIL_AFTER", "1")
    with pytest.raises(RuntimeError):
        cli.run_band(cfg_path, engine_factory=fake_engine.factory)
    cfg_path.write_text(GOLDEN_TOML.replace("block_size = 8", "block_size = 16"))
    with pytest.raises(InputError, match="another calculation"):
        cli.run_band(cfg_path, resume=True, engine_factory=fake_engine.factory)


def test_cli_exit_code_two(tmp_path, capsys):
    (tmp_path / "x.toml").write_text("[band]\n")
    assert cli.main(["band", str(tmp_path / "x.toml")]) == 2
    assert "aospectrum:" in capsys.readouterr().err


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, cfg: str, result: str) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port), "LOCAL_RANK": str(rank)})
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cli.run_band(cfg, engine_factory=fake_engine.factory)
        Path(result + f".{rank}").write_text(str(fake_engine.OracleEngine.calls))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_kpoints_gloo(tmp_path, golden):
    import torch.multiprocessing as mp

    cfg = make_case(tmp_path, golden)
    result = str(tmp_path / "calls")
    mp.start_processes(_rank_main, args=(2, _free_port(), str(cfg), result), nprocs=2,
                       start_method="spawn", join=True)
    calls = [int(Path(result + f".{r}").read_text()) for r in range(2)]
    assert sorted(calls) == [3, 4]          # 7 k points, round-robin over 2 ranks
    rows = list(csv.reader((tmp_path / "out" / "bands.csv").open()))[1:]
    assert sorted({int(r[0]) for r in rows}) == list(range(7))
