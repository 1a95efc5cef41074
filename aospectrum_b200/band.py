"""Energy-window Band calculation: per-k solve, checkpoints and outputs.

Drop-in for the reference Band application layer
(``src/aospectrum/band.py:132-499``): the same ``BandCalculation`` seam
(``solver=`` accepts any object with ``solve_interval(SparsePair,
EnergyInterval) -> CissResult``), the same atomic ``k-NNNNNN.npz``
checkpoint fields, and the same ``bands.csv`` / ``summary.json`` outputs.
The default solver is the GPU engine in ``aospectrum_b200.engine``; it also
offers ``solve_points`` to push several k points through one batched
factorization.
"""

from __future__ import annotations

import csv
import json
import os
from dataclasses import dataclass, field
from pathlib import Path
from time import perf_counter
from typing import Any, Sequence

import numpy as np

from .ciss import CissSettings, EngineSettings
from .data import EnergyInterval, LocalizedOperatorBundle
from .errors import InputError, SolverError
from .kpath import KPath, read_kpath  # noqa: F401  (re-exported)

CONTINUITY_GUARD_EV = 0.02
BACKEND_NAME = "ciss-b200"


def resolve_energy_reference(bundle: LocalizedOperatorBundle, mode: str,
                             value_ev: float | None = None) -> float:
    """Reference energy subtracted from the output (reference
    ``band.py:132-147``)."""
    if mode in ("input_zero", "absolute"):
        return 0.0
    if mode == "fixed":
        if value_ev is None:
            raise InputError("fixed energy reference requires a value")
        return float(value_ev)
    if mode == "bundle_fermi":
        fill = bundle.filling
        if fill is None or fill.fermi_energy_ev is None:
            raise InputError("bundle has no Fermi energy")
        return fill.fermi_energy_ev
    raise InputError("energy reference must be input_zero, fixed, or bundle_fermi")


@dataclass(slots=True)
class BandPoint:
    index: int
    k_fractional: np.ndarray
    energies_ev: np.ndarray
    maximum_residual_ev: float
    stage_seconds: dict[str, float]
    assembly_seconds: float
    peak_gpu_memory_bytes: int | None
    warnings: tuple[str, ...] = ()

    def __post_init__(self) -> None:
        self.index = int(self.index)
        self.k_fractional = np.asarray(self.k_fractional, dtype=np.float64)
        self.energies_ev = np.asarray(self.energies_ev, dtype=np.float32)
        if self.index < 0 or self.k_fractional.shape != (3,):
            raise InputError("invalid Band point")


@dataclass(slots=True)
class BandResult:
    kpath: KPath
    display_interval_ev: EnergyInterval
    solve_interval_ev: EnergyInterval
    reference_energy_ev: float
    cell_angstrom: np.ndarray
    points: tuple[BandPoint, ...]
    elapsed_seconds: float
    warnings: tuple[str, ...] = ()

    @property
    def display_energies_ev(self) -> tuple[np.ndarray, ...]:
        return tuple(p.energies_ev - self.reference_energy_ev for p in self.points)


@dataclass(slots=True)
class BandCalculation:
    """Per-k Band driver.  With ``solver=None`` the GPU engine assembles
    H(k), S(k) on the device and runs CISS there; a user ``solver`` receives
    host CSR matrices exactly as in the reference."""

    bundle: LocalizedOperatorBundle
    kpath: KPath
    display_interval_ev: EnergyInterval
    reference_energy_ev: float
    settings: CissSettings = field(default_factory=CissSettings)
    solver: Any | None = None
    engine_settings: EngineSettings = field(default_factory=EngineSettings)
    engine_factory: Any | None = None
    lazy_engine: bool = False
    solve_interval_ev: EnergyInterval = field(init=False)
    absolute_interval_ev: EnergyInterval = field(init=False)
    engine: Any = field(init=False)
    warnings: tuple[str, ...] = field(init=False)

    def __post_init__(self) -> None:
        self.solve_interval_ev = self.display_interval_ev.expanded(CONTINUITY_GUARD_EV)
        ref = self.reference_energy_ev
        self.absolute_interval_ev = EnergyInterval(
            self.solve_interval_ev.lower_ev + ref, self.solve_interval_ev.upper_ev + ref
        )
        self.engine = None
        if not self.lazy_engine:
            self.engine = self._make_engine()
        notes = []
        if self.bundle.basis.spinor_width != 1:
            notes.append("spinor input is outside the current non-SOC Band scope; "
                         "the result may be inaccurate")
        if not all(self.bundle.structure.periodic):
            notes.append("non-periodic axes are outside the current Bloch scope; "
                         "the result may be inaccurate")
        self.warnings = tuple(notes)

    def _make_engine(self):
        if self.engine_factory is not None:
            return self.engine_factory(self.bundle, self.settings, self.engine_settings)
        from .engine import BandEngine

        return BandEngine(self.bundle, self.settings, self.engine_settings)

    def _check_index(self, index: int) -> int:
        if not 0 <= int(index) < self.kpath.n_points:
            raise InputError("k-point index is out of range")
        return int(index)

    def solve_point(self, index: int) -> BandPoint:
        return self.solve_points([index])[0]

    def solve_points(self, indices: Sequence[int]) -> list[BandPoint]:
        """Solve several k points; the GPU engine batches their shifted
        factorizations when memory allows."""
        idx = [self._check_index(i) for i in indices]
        kpts = [self.kpath.fractional_points[i] for i in idx]
        if self.engine is None:
            self.engine = self._make_engine()
        if self.solver is None:
            results, assembly = self.engine.solve_kpoints(kpts, self.absolute_interval_ev)
        else:
            results, assembly = [], []
            for k in kpts:
                started = perf_counter()
                pair = self.engine.host_pair(k)
                assembly.append(perf_counter() - started)
                results.append(self.solver.solve_interval(pair, self.absolute_interval_ev))
        points = []
        for i, k, res, asm in zip(idx, kpts, results, assembly):
            if not res.complete:
                raise SolverError("CISS search subspace is saturated; increase "
                                  "block_size or moment_size")
            points.append(BandPoint(i, k, res.energies_ev, res.maximum_residual_ev,
                                    res.stage_seconds, asm, res.peak_gpu_memory_bytes,
                                    res.warnings))
        return points

    def build_result(self, points: Sequence[BandPoint], *, elapsed_seconds: float) -> BandResult:
        ordered = tuple(sorted(points, key=lambda p: p.index))
        if [p.index for p in ordered] != list(range(self.kpath.n_points)):
            raise SolverError("Band result does not contain every k point")
        return BandResult(self.kpath, self.display_interval_ev, self.solve_interval_ev,
                          self.reference_energy_ev, self.bundle.structure.cell_angstrom,
                          ordered, float(elapsed_seconds), self.warnings)

    def close(self) -> None:
        closer = getattr(self.solver, "close", None)
        if callable(closer):
            closer()
        if self.engine is not None:
            self.engine.close()


def write_point(path: str | Path, point: BandPoint) -> None:
    """Atomic npz checkpoint of one k point (reference ``band.py:281-309``)."""
    dest = Path(path)
    dest.parent.mkdir(parents=True, exist_ok=True)
    tmp = dest.with_name(f".{dest.name}.tmp")
    peak = -1 if point.peak_gpu_memory_bytes is None else int(point.peak_gpu_memory_bytes)
    with tmp.open("wb") as handle:
        np.savez(
            handle,
            index=np.asarray(point.index, dtype=np.int64),
            k_fractional=point.k_fractional,
            energies_ev=point.energies_ev,
            maximum_residual_ev=np.asarray(point.maximum_residual_ev, dtype=np.float64),
            stage_names=np.asarray(tuple(point.stage_seconds), dtype="U64"),
            stage_values=np.asarray(tuple(point.stage_seconds.values()), dtype=np.float64),
            assembly_seconds=np.asarray(point.assembly_seconds, dtype=np.float64),
            peak_gpu_memory_bytes=np.asarray(peak, dtype=np.int64),
            warnings=np.asarray(point.warnings, dtype="U256"),
        )
    os.replace(tmp, dest)


def read_point(path: str | Path, *, index: int, k_fractional: np.ndarray) -> BandPoint | None:
    """Load a checkpoint, or ``None`` when absent; a checkpoint of another
    point is an ``InputError`` (reference ``band.py:312-344``)."""
    src = Path(path)
    if not src.is_file():
        return None
    try:
        with np.load(src, allow_pickle=False) as z:
            kf = np.asarray(z["k_fractional"])
            if int(z["index"]) != index or not np.array_equal(kf, k_fractional):
                raise InputError(f"Band checkpoint does not match point {index}")
            peak = int(z["peak_gpu_memory_bytes"])
            return BandPoint(
                index=index,
                k_fractional=kf,
                energies_ev=z["energies_ev"],
                maximum_residual_ev=float(z["maximum_residual_ev"]),
                stage_seconds=dict(zip(z["stage_names"].tolist(), z["stage_values"].tolist())),
                assembly_seconds=float(z["assembly_seconds"]),
                peak_gpu_memory_bytes=None if peak < 0 else peak,
                warnings=tuple(z["warnings"].tolist()),
            )
    except (OSError, ValueError, KeyError) as exc:
        raise InputError(f"cannot read Band checkpoint {src}: {exc}") from exc


def assign_track_ids(energies: Sequence[np.ndarray]) -> tuple[np.ndarray, ...]:
    """Band tracks by minimum-cost matching of consecutive k points
    (reference ``band.py:347-366``); unmatched states open new tracks."""
    from scipy.optimize import linear_sum_assignment

    tracks = [np.arange(energies[0].size, dtype=np.int64)]
    fresh = int(energies[0].size)
    for prev, cur in zip(energies[:-1], energies[1:]):
        ids = np.full(cur.size, -1, dtype=np.int64)
        if prev.size and cur.size:
            r, c = linear_sum_assignment(np.abs(prev[:, None] - cur[None, :]))
            ids[c] = tracks[-1][r]
        missing = np.flatnonzero(ids < 0)
        ids[missing] = fresh + np.arange(missing.size)
        fresh += int(missing.size)
        tracks.append(ids)
    return tuple(tracks)


def summary_dict(result: BandResult) -> dict[str, Any]:
    stages: dict[str, float] = {}
    notes = list(result.warnings)
    for p in result.points:
        for name, sec in p.stage_seconds.items():
            stages[name] = stages.get(name, 0.0) + float(sec)
        notes.extend(p.warnings)
    peaks = [p.peak_gpu_memory_bytes for p in result.points if p.peak_gpu_memory_bytes is not None]
    return {
        "backend": BACKEND_NAME,
        "scalar_dtype": "complex64",
        "kpoint_count": result.kpath.n_points,
        "energy_interval_ev": [result.display_interval_ev.lower_ev,
                               result.display_interval_ev.upper_ev],
        "reference_energy_ev": result.reference_energy_ev,
        "maximum_eigenpair_residual_ev": max(
            (p.maximum_residual_ev for p in result.points), default=0.0),
        "elapsed_seconds": result.elapsed_seconds,
        "assembly_seconds": sum(p.assembly_seconds for p in result.points),
        "solver_stage_seconds": stages,
        "peak_gpu_memory_bytes": max(peaks) if peaks else None,
        "warnings": list(dict.fromkeys(notes)),
    }


def write_band_output(result: BandResult, root: str | Path) -> Path:
    """``bands.csv`` + ``summary.json`` always, ``band.png`` when matplotlib
    imports (reference ``band.py:396-499``)."""
    out = Path(root)
    out.mkdir(parents=True, exist_ok=True)
    dist = result.kpath.distances(result.cell_angstrom)
    energies = result.display_energies_ev
    tracks = assign_track_ids(energies)
    with (out / "bands.csv").open("w", encoding="utf-8", newline="") as handle:
        w = csv.writer(handle)
        w.writerow(("k_index", "k_distance_inv_angstrom", "track_id", "energy_ev"))
        for p, x, ids, vals in zip(result.points, dist, tracks, energies):
            for t, e in zip(ids, vals):
                w.writerow((p.index, f"{x:.12e}", int(t), f"{float(e):.12e}"))
    (out / "summary.json").write_text(
        json.dumps(summary_dict(result), indent=2, sort_keys=True) + "\n", encoding="utf-8")
    try:
        import matplotlib

        matplotlib.use("Agg")
        import matplotlib.pyplot as plt
        from matplotlib.collections import LineCollection
    except ImportError:
        return out
    segs = []
    for i in range(dist.size - 1):
        nxt = {int(t): j for j, t in enumerate(tracks[i + 1])}
        for j, t in enumerate(tracks[i]):
            m = nxt.get(int(t))
            if m is not None:
                segs.append([[dist[i], energies[i][j]], [dist[i + 1], energies[i + 1][m]]])
    fig, ax = plt.subplots(figsize=(7.2, 5.2), constrained_layout=True)
    if segs:
        ax.add_collection(LineCollection(np.asarray(segs), colors="#17213a", linewidths=1.05))
    ax.set_xlim(float(dist[0]), float(dist[-1]))
    ax.set_ylim(result.display_interval_ev.lower_ev, result.display_interval_ev.upper_ev)
    node_x = dist[result.kpath.node_indices]
    for x in node_x[1:-1]:
        ax.axvline(x, color="#9aa1ad", linewidth=0.7, zorder=0)
    ax.axhline(0.0, color="#b73b3b", linewidth=0.8, linestyle="--")
    ax.set_xticks(node_x, result.kpath.node_labels)
    ax.set_xlabel("K path")
    ax.set_ylabel("Energy relative to reference (eV)")
    fig.savefig(out / "band.png", dpi=240)
    plt.close(fig)
    return out
