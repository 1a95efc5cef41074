"""k paths in the ``aospectrum.kpath/v1`` JSON format.

Two JSON forms are accepted, as in the reference (``src/aospectrum/band.py:
26-129``): ``nodes_fractional`` + ``points_per_segment`` (linear
interpolation, shared endpoints counted once) or explicit
``fractional_points`` + ``node_indices``.  ``labels`` name the nodes.
"""

from __future__ import annotations

import json
from dataclasses import dataclass
from pathlib import Path
from typing import Any, Sequence

import numpy as np

from .errors import InputError

KPATH_SCHEMA = "aospectrum.kpath/v1"


@dataclass(frozen=True, slots=True)
class KPath:
    fractional_points: np.ndarray
    node_indices: np.ndarray
    node_labels: tuple[str, ...]

    def __post_init__(self) -> None:
        pts = np.array(self.fractional_points, dtype=np.float64)
        nodes = np.array(self.node_indices, dtype=np.int64)
        labels = tuple(str(v) for v in self.node_labels)
        if pts.ndim != 2 or pts.shape[1:] != (3,) or pts.shape[0] < 2:
            raise InputError("k path must contain at least two 3D points")
        bad_nodes = (
            nodes.ndim != 1
            or nodes.size < 2
            or nodes[0] != 0
            or nodes[-1] != pts.shape[0] - 1
            or bool(np.any(nodes[1:] <= nodes[:-1]))
            or len(labels) != nodes.size
        )
        if bad_nodes:
            raise InputError("invalid k-path nodes or labels")
        pts.setflags(write=False)
        nodes.setflags(write=False)
        object.__setattr__(self, "fractional_points", pts)
        object.__setattr__(self, "node_indices", nodes)
        object.__setattr__(self, "node_labels", labels)

    @classmethod
    def interpolate(cls, nodes: Sequence[Sequence[float]], labels: Sequence[str], *,
                    points_per_segment: int) -> "KPath":
        corners = np.asarray(nodes, dtype=np.float64)
        per = int(points_per_segment)
        if corners.ndim != 2 or corners.shape[1:] != (3,) or corners.shape[0] < 2 or per < 1:
            raise InputError("invalid interpolated k path")
        pieces = []
        for a, b in zip(corners[:-1], corners[1:]):
            seg = np.linspace(a, b, per + 1, dtype=np.float64)
            pieces.append(seg if not pieces else seg[1:])
        node_idx = np.arange(corners.shape[0], dtype=np.int64) * per
        return cls(np.concatenate(pieces), node_idx, tuple(labels))

    @property
    def n_points(self) -> int:
        return int(self.fractional_points.shape[0])

    def distances(self, cell_angstrom: np.ndarray) -> np.ndarray:
        """Cumulative Cartesian path length in 1/Angstrom."""
        recip = 2.0 * np.pi * np.linalg.inv(np.asarray(cell_angstrom, np.float64)).T
        cart = self.fractional_points @ recip
        steps = np.linalg.norm(np.diff(cart, axis=0), axis=1)
        return np.concatenate(([0.0], np.cumsum(steps)))


def kpath_from_dict(obj: Any) -> KPath:
    if not isinstance(obj, dict):
        raise InputError("k path must contain a JSON object")
    if obj.get("schema", KPATH_SCHEMA) != KPATH_SCHEMA:
        raise InputError(f"k path schema must be {KPATH_SCHEMA}")
    labels = obj.get("labels")
    if not isinstance(labels, list):
        raise InputError("k path labels must be a list")
    if "nodes_fractional" in obj:
        return KPath.interpolate(obj["nodes_fractional"], labels,
                                 points_per_segment=obj.get("points_per_segment", 0))
    if "fractional_points" not in obj or "node_indices" not in obj:
        raise InputError("k path needs nodes_fractional or fractional_points")
    return KPath(obj["fractional_points"], obj["node_indices"], tuple(labels))


def read_kpath(path: str | Path) -> KPath:
    src = Path(path)
    try:
        obj = json.loads(src.read_text(encoding="utf-8"))
    except (OSError, UnicodeError, json.JSONDecodeError) as exc:
        raise InputError(f"cannot read k path {src}: {exc}") from exc
    return kpath_from_dict(obj)
