"""``aospectrum band <config.toml> [--resume]`` for the B200 engine.

Drop-in for the Band side of the reference CLI (``src/aospectrum/cli.py:
54-177, 270-436, 574-615``): the same TOML sections and keys, the same
``.<output>.work`` directory with ``run.json`` and atomic ``k-NNNNNN.npz``
checkpoints, the same publish step and exit code 2 on ``AOSpectrumError``.

Differences, all opt-in and backward compatible:
  * ``[solver]`` accepts engine keys (``precision``, ``refinement_steps``,
    ``tile``, ``max_pencils``, ``memory_fraction``, ``ordering``,
    ``kpoints_per_batch``); ``run.json`` records them only when they differ
    from the defaults, so work directories of the reference still resume;
  * each device worker solves its k points in batches
    (``kpoints_per_batch``), sharing factorization launches;
  * under ``torchrun`` (``WORLD_SIZE`` > 1) every rank is one worker and the
    ranks meet at a ``torch.distributed`` barrier before rank 0 publishes.
"""

from __future__ import annotations

import argparse
import json
import multiprocessing
import os
import shutil
import sys
from concurrent.futures import ProcessPoolExecutor
from dataclasses import asdict, dataclass, fields
from pathlib import Path
from time import perf_counter
from typing import Any, Callable, Sequence

try:
    import tomllib
except ModuleNotFoundError:  # pragma: no cover
    import tomli as tomllib

from . import __version__
from .band import (
    BandCalculation,
    read_point,
    resolve_energy_reference,
    write_band_output,
    write_point,
)
from .bundle import load_bundle
from .ciss import CissSettings, EngineSettings
from .data import EnergyInterval, LocalizedOperatorBundle
from .errors import AOSpectrumError, InputError, SolverError
from .kpath import KPath, read_kpath


@dataclass(frozen=True, slots=True)
class BandConfig:
    source: Path
    bundle: Path
    kpath: KPath
    interval: EnergyInterval
    reference_mode: str
    reference_value_ev: float | None
    devices: tuple[int, ...]
    settings: CissSettings
    output: Path
    engine: EngineSettings = EngineSettings()
    kpoints_per_batch: int = 1

    @property
    def work(self) -> Path:
        return self.output.with_name(f".{self.output.name}.work")


def _toml(path: str | Path) -> tuple[Path, dict[str, Any]]:
    src = Path(path).expanduser().resolve()
    try:
        with src.open("rb") as handle:
            return src, tomllib.load(handle)
    except (OSError, tomllib.TOMLDecodeError) as exc:
        raise InputError(f"cannot read TOML configuration {src}: {exc}") from exc


def _table(values: dict[str, Any], name: str) -> dict[str, Any]:
    t = values.get(name, {})
    if not isinstance(t, dict):
        raise InputError(f"[{name}] must be a TOML table")
    return t


def _path(base: Path, value: Any, name: str) -> Path:
    if not isinstance(value, str) or not value.strip():
        raise InputError(f"{name} must be a path")
    p = Path(value).expanduser()
    return p.resolve() if p.is_absolute() else (base / p).resolve()


def _two_numbers(value: Any, name: str) -> tuple[float, float]:
    if not isinstance(value, list) or len(value) != 2:
        raise InputError(f"{name} must contain two numbers")
    try:
        return float(value[0]), float(value[1])
    except (TypeError, ValueError) as exc:
        raise InputError(f"{name} must contain two numbers") from exc


_ENGINE_KEYS = ("precision", "refinement_steps", "tile", "max_pencils", "memory_fraction",
                "ordering")


def read_band_config(path: str | Path) -> BandConfig:
    """TOML -> BandConfig with the reference's keys (cli.py:123-177)."""
    src, values = _toml(path)
    base = src.parent
    inp, band, compute = _table(values, "input"), _table(values, "band"), _table(values, "compute")
    solver, resources, output = (_table(values, "solver"), _table(values, "resources"),
                                 _table(values, "output"))
    devices = compute.get("devices", [0])
    valid = (isinstance(devices, list) and devices
             and all(isinstance(d, int) and not isinstance(d, bool) and d >= 0 for d in devices)
             and len(set(devices)) == len(devices))
    if not valid:
        raise InputError("compute.devices must contain unique GPU indices")
    interval = EnergyInterval(*_two_numbers(band.get("energy_interval_ev"),
                                            "band.energy_interval_ev"))
    mode = str(band.get("energy_reference", "input_zero"))
    ref_value = band.get("energy_reference_ev")
    try:
        ref_value = None if ref_value is None else float(ref_value)
        settings = CissSettings(
            integration_points=int(solver.get("integration_points", 32)),
            contour_batch_size=int(solver.get("contour_batch_size",
                                              resources.get("contour_batch_size", 1))),
            block_size=int(solver.get("block_size", 32)),
            moment_size=int(solver.get("moment_size", 4)),
        )
        engine = EngineSettings(**{k: solver[k] for k in _ENGINE_KEYS if k in solver})
        per_batch = int(solver.get("kpoints_per_batch", 1))
    except (TypeError, ValueError) as exc:
        raise InputError("invalid Band solver setting") from exc
    if per_batch < 1:
        raise InputError("solver.kpoints_per_batch must be positive")
    return BandConfig(src, _path(base, inp.get("bundle"), "input.bundle"),
                      read_kpath(_path(base, band.get("kpath"), "band.kpath")), interval, mode,
                      ref_value, tuple(devices), settings,
                      _path(base, output.get("directory"), "output.directory"), engine, per_batch)


def band_specification(config: BandConfig, bundle: LocalizedOperatorBundle) -> dict[str, Any]:
    """``run.json`` contents (reference cli.py:306-327); engine knobs that
    differ from their defaults are appended to ``solver``."""
    solver = asdict(config.settings)
    defaults = EngineSettings()
    for f in fields(EngineSettings):
        v = getattr(config.engine, f.name)
        if v != getattr(defaults, f.name):
            solver[f.name] = v
    if config.kpoints_per_batch != 1:
        solver["kpoints_per_batch"] = config.kpoints_per_batch
    return {
        "kind": "band",
        "bundle": str(config.bundle),
        "basis_identity": bundle.basis.basis_identity,
        "n_orbitals": bundle.n_orbitals,
        "interval_ev": [config.interval.lower_ev, config.interval.upper_ev],
        "reference": [config.reference_mode, config.reference_value_ev],
        "kpoints": config.kpath.fractional_points.tolist(),
        "nodes": config.kpath.node_indices.tolist(),
        "labels": list(config.kpath.node_labels),
        "solver": solver,
    }


def _require_output(path: Path) -> None:
    if path.exists() and (not path.is_dir() or any(path.iterdir())):
        raise InputError(f"output directory is not empty: {path}")


def prepare_work(path: Path, spec: dict[str, Any], *, resume: bool) -> None:
    run = path / "run.json"
    if resume:
        try:
            seen = json.loads(run.read_text(encoding="utf-8"))
        except (OSError, json.JSONDecodeError) as exc:
            raise InputError(f"cannot resume work directory {path}") from exc
        if seen != spec:
            raise InputError("resume work belongs to another calculation")
        return
    if path.exists():
        raise InputError(f"work directory already exists: {path}; use --resume")
    path.mkdir(parents=True)
    run.write_text(json.dumps(spec, indent=2, sort_keys=True) + "\n", encoding="utf-8")


def _cuda_token(index: int, inherited: str | None) -> str:
    if inherited:
        visible = [v.strip() for v in inherited.split(",") if v.strip()]
        if index >= len(visible):
            raise InputError(f"GPU index {index} exceeds CUDA_VISIBLE_DEVICES={inherited}")
        return visible[index]
    return str(index)


EngineFactory = Callable[[LocalizedOperatorBundle, CissSettings, EngineSettings], Any]


def band_worker(config: BandConfig, reference_ev: float, rank: int, world: int,
                cuda_token: str | None, engine_factory: EngineFactory | None = None) -> int:
    """Solve this worker's k points (index rank, rank+world, ...), skipping
    those with a valid checkpoint (reference cli.py:330-365)."""
    if cuda_token is not None:
        os.environ["CUDA_VISIBLE_DEVICES"] = cuda_token
    bundle = load_bundle(config.bundle)
    calc = BandCalculation(bundle, config.kpath, config.interval, reference_ev, config.settings,
                           engine_settings=config.engine, engine_factory=engine_factory)
    done = 0
    try:
        todo = []
        for index in range(rank, config.kpath.n_points, world):
            path = config.work / f"k-{index:06d}.npz"
            if read_point(path, index=index,
                          k_fractional=config.kpath.fractional_points[index]) is None:
                todo.append(index)
            else:
                done += 1
        for b0 in range(0, len(todo), config.kpoints_per_batch):
            batch = todo[b0:b0 + config.kpoints_per_batch]
            print(f"[gpu {rank}] k points {', '.join(str(i + 1) for i in batch)}"
                  f"/{config.kpath.n_points}", flush=True)
            for point in calc.solve_points(batch):
                write_point(config.work / f"k-{point.index:06d}.npz", point)
                done += 1
    finally:
        calc.close()
    return done


def _distributed_env() -> tuple[int, int] | None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None
    return int(os.environ.get("RANK", "0")), world


def run_band(path: str | Path, *, resume: bool = False,
             engine_factory: EngineFactory | None = None) -> Path:
    """The Band application (reference cli.py:368-436)."""
    config = read_band_config(path)
    dist_env = _distributed_env()
    rank = dist_env[0] if dist_env else 0
    bundle = load_bundle(config.bundle)
    reference = resolve_energy_reference(bundle, config.reference_mode,
                                         config.reference_value_ev)
    started = perf_counter()
    if dist_env is not None:
        import torch.distributed as dist

        if not dist.is_initialized():
            backend = "nccl" if engine_factory is None else "gloo"
            dist.init_process_group(backend)
        if rank == 0:
            _require_output(config.output)
            prepare_work(config.work, band_specification(config, bundle), resume=resume)
        dist.barrier()
        local = os.environ.get("LOCAL_RANK")
        if engine_factory is None and local is not None:
            import torch

            torch.cuda.set_device(int(local))
        band_worker(config, reference, rank, dist_env[1], None, engine_factory)
        dist.barrier()
        if rank != 0:
            return config.output
    else:
        _require_output(config.output)
        prepare_work(config.work, band_specification(config, bundle), resume=resume)
        inherited = os.environ.get("CUDA_VISIBLE_DEVICES")
        tokens = tuple(_cuda_token(i, inherited) for i in config.devices)
        if len(tokens) == 1:
            band_worker(config, reference, 0, 1, tokens[0], engine_factory)
        else:
            ctx = multiprocessing.get_context("spawn")
            with ProcessPoolExecutor(max_workers=len(tokens), mp_context=ctx) as pool:
                futures = [pool.submit(band_worker, config, reference, r, len(tokens), t,
                                       engine_factory) for r, t in enumerate(tokens)]
                for f in futures:
                    f.result()
    points = []
    for index, kpt in enumerate(config.kpath.fractional_points):
        point = read_point(config.work / f"k-{index:06d}.npz", index=index, k_fractional=kpt)
        if point is None:
            raise SolverError(f"Band point {index} is missing")
        points.append(point)
    calc = BandCalculation(bundle, config.kpath, config.interval, reference, config.settings,
                           engine_settings=config.engine, engine_factory=engine_factory,
                           lazy_engine=True)
    result = calc.build_result(points, elapsed_seconds=perf_counter() - started)
    publish = config.output.with_name(f".{config.output.name}.publish")
    if publish.exists():
        shutil.rmtree(publish)
    write_band_output(result, publish)
    if config.output.exists():
        config.output.rmdir()
    os.replace(publish, config.output)
    shutil.rmtree(config.work)
    print(config.output)
    return config.output


def _parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="aospectrum",
                                 description="Energy-window band structures on B200 GPUs.")
    ap.add_argument("--version", action="version", version=__version__)
    sub = ap.add_subparsers(dest="command", required=True)
    band = sub.add_parser("band", help="calculate an energy-window band structure")
    band.add_argument("config", type=Path)
    band.add_argument("--resume", action="store_true")
    return ap


def main(argv: Sequence[str] | None = None) -> int:
    args = _parser().parse_args(argv)
    try:
        run_band(args.config, resume=args.resume)
    except AOSpectrumError as exc:
        print(f"aospectrum: {exc}", file=sys.stderr)
        return 2
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
