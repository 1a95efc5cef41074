"""Seeded synthetic operator bundles for the Band-path workloads.

No public dataset is involved: every workload is a deterministic function of
its spec and seed.  A spec places atoms on a jittered grid, connects every
pair of atoms (including periodic images with ``|R_a| <= max_shift``) whose
distance is within ``cutoff``, and draws one block pair per connection::

    H_{i0,jR}  = exp(-d / decay) * G              G  ~ N(0, 1) eV
    S_{i0,jR}  = overlap_scale * exp(-d / decay) * G'
    H_{j0,i(-R)} = H_{i0,jR}^T,   S_{j0,i(-R)} = S_{i0,jR}^T

Onsite blocks are symmetric with diagonal ``U(onsite_low, onsite_high)``
eV; onsite overlap blocks have unit diagonal.  Each atom carries
``orbitals_per_atom`` AOs (13 = an s2p2d1 layout, 5 = s1p1 "C-like").

``WORKLOADS`` holds the five named workloads with their energy windows.
The windows were set from the FP64 dense generalized eigenvalues at Gamma
(``suggest_window``) so that they hold the stated number of states there.
"""

from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import Any

import numpy as np

from .data import (
    AtomicStructure,
    LocalizedOperatorBlocks,
    LocalizedOperatorBundle,
    OrbitalBasisLayout,
)
from .errors import InputError


_LAYOUTS = {
    13: ("s", "s", "px", "py", "pz", "px", "py", "pz", "dxy", "dyz", "dz2", "dxz", "dx2-y2"),
    5: ("s", "px", "py", "pz", "s*"),
}


@dataclass(frozen=True)
class SyntheticSpec:
    """Geometry and block statistics of one synthetic bundle."""

    name: str
    grid: tuple[int, int, int]
    spacing: tuple[float, float, float]
    cell: tuple[float, float, float]
    periodic: tuple[bool, bool, bool]
    cutoff: float
    orbitals_per_atom: int = 13
    jitter: float = 0.05
    max_shift: int = 1
    decay: float = 1.5
    overlap_scale: float = 0.08
    onsite_low: float = -10.0
    onsite_high: float = 5.0
    origin: tuple[float, float, float] = (0.0, 0.0, 0.0)
    seed: int = 20260727

    @property
    def n_atoms(self) -> int:
        return int(np.prod(self.grid))

    @property
    def n_orbitals(self) -> int:
        return self.n_atoms * self.orbitals_per_atom


@dataclass(frozen=True)
class Workload:
    """A named Band workload: bundle spec + k-points + CISS sizes + window."""

    name: str
    spec: SyntheticSpec
    kpath: dict[str, Any]
    window_ev: tuple[float, float]
    states_at_gamma: int
    integration_points: int = 32
    block_size: int = 32
    moment_size: int = 4
    notes: str = ""
    extra: dict[str, Any] = field(default_factory=dict)


def _positions(spec: SyntheticSpec, rng: np.random.Generator) -> np.ndarray:
    axes = [np.arange(g, dtype=np.float64) * s for g, s in zip(spec.grid, spec.spacing)]
    mesh = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
    mesh = mesh + np.asarray(spec.origin)
    return mesh + rng.normal(0.0, spec.jitter, size=mesh.shape)


def _lattice_shifts(spec: SyntheticSpec) -> np.ndarray:
    ranges = [
        range(-spec.max_shift, spec.max_shift + 1) if p else range(0, 1)
        for p in spec.periodic
    ]
    return np.array([(a, b, c) for a in ranges[0] for b in ranges[1] for c in ranges[2]],
                    dtype=np.int32)


def _connections(spec: SyntheticSpec, pos: np.ndarray):
    """Canonical connections (i, j, R, d): i < j, or i == j with R > 0 in
    lexicographic order, or the onsite (i, i, 0)."""
    from scipy.spatial import cKDTree

    cell = np.diag(spec.cell)
    tree = cKDTree(pos)
    out_i, out_j, out_r, out_d = [], [], [], []
    for shift in _lattice_shifts(spec):
        image = cKDTree(pos + shift.astype(np.float64) @ cell)
        pairs = tree.sparse_distance_matrix(image, spec.cutoff, output_type="ndarray")
        i = pairs["i"].astype(np.int64)
        j = pairs["j"].astype(np.int64)
        d = pairs["v"].astype(np.float64)
        positive = tuple(shift) > (0, 0, 0)
        zero = not np.any(shift)
        if zero:
            keep = i < j
        elif positive:
            keep = i <= j
        else:
            keep = i < j
        i, j, d = i[keep], j[keep], d[keep]
        out_i.append(i)
        out_j.append(j)
        out_d.append(d)
        out_r.append(np.broadcast_to(shift, (i.size, 3)))
    i = np.concatenate(out_i)
    j = np.concatenate(out_j)
    r = np.concatenate(out_r).astype(np.int32)
    d = np.concatenate(out_d)
    order = np.lexsort((r[:, 2], r[:, 1], r[:, 0], j, i))
    return i[order], j[order], r[order], d[order]


def generate_bundle(spec: SyntheticSpec) -> LocalizedOperatorBundle:
    """Build the bundle for ``spec`` (deterministic in ``spec.seed``)."""
    if spec.orbitals_per_atom not in _LAYOUTS:
        raise InputError("orbitals_per_atom must be 13 or 5")
    rng = np.random.default_rng(spec.seed)
    no = spec.orbitals_per_atom
    pos = _positions(spec, rng)
    n_atoms = pos.shape[0]
    ci, cj, cr, cd = _connections(spec, pos)
    npair = ci.size
    scale = np.exp(-cd / spec.decay).astype(np.float32)
    g_h = rng.standard_normal((npair, no, no), dtype=np.float32) * scale[:, None, None]
    g_s = rng.standard_normal((npair, no, no), dtype=np.float32) * (
        np.float32(spec.overlap_scale) * scale[:, None, None]
    )
    onsite_h = rng.standard_normal((n_atoms, no, no), dtype=np.float32)
    onsite_h = np.float32(0.5) * (onsite_h + onsite_h.transpose(0, 2, 1))
    diag = rng.uniform(spec.onsite_low, spec.onsite_high, size=(n_atoms, no)).astype(np.float32)
    idx = np.arange(no)
    onsite_h[:, idx, idx] = diag
    onsite_s = rng.standard_normal((n_atoms, no, no), dtype=np.float32)
    onsite_s = np.float32(0.5 * spec.overlap_scale) * (onsite_s + onsite_s.transpose(0, 2, 1))
    onsite_s[:, idx, idx] = 1.0

    # Blocks: onsite, each canonical connection, and its mirror.
    rows = np.concatenate((np.arange(n_atoms), ci, cj))
    cols = np.concatenate((np.arange(n_atoms), cj, ci))
    shifts = np.concatenate((np.zeros((n_atoms, 3), np.int32), cr, -cr))
    hb = np.concatenate((onsite_h, g_h, g_h.transpose(0, 2, 1)))
    sb = np.concatenate((onsite_s, g_s, g_s.transpose(0, 2, 1)))
    order = np.lexsort((shifts[:, 2], shifts[:, 1], shifts[:, 0], cols, rows))
    rows, cols, shifts = rows[order], cols[order], shifts[order]
    hb = np.ascontiguousarray(hb[order]).reshape(-1)
    sb = np.ascontiguousarray(sb[order]).reshape(-1)
    nblk = rows.size
    offsets = np.arange(nblk + 1, dtype=np.int64) * (no * no)
    shapes = np.full((nblk, 2), no, dtype=np.int32)

    owner = np.repeat(np.arange(n_atoms, dtype=np.int32), no)
    local = np.tile(np.arange(no, dtype=np.int32), n_atoms)
    structure = AtomicStructure(
        cell_angstrom=np.diag(spec.cell),
        positions_angstrom=pos,
        atomic_numbers=np.full(n_atoms, 22 if no == 13 else 6, dtype=np.int32),
        periodic=spec.periodic,
        label=spec.name,
    )
    basis = OrbitalBasisLayout(
        n_atoms=n_atoms,
        orbital_atom=owner,
        local_index=local,
        basis_family="synthetic",
        basis_identity=f"synthetic-{no}orb",
        orbital_labels=tuple(_LAYOUTS[no]) * n_atoms,
    )
    operators = LocalizedOperatorBlocks(
        row_atom=rows.astype(np.int32),
        col_atom=cols.astype(np.int32),
        lattice_shift=shifts.astype(np.int32),
        block_offsets=offsets,
        block_shapes=shapes,
        h_values=hb,
        s_values=sb,
    )
    provenance = {
        "generator": "aospectrum_b200.synth",
        "spec": {k: (list(v) if isinstance(v, tuple) else v)
                 for k, v in spec.__dict__.items()},
    }
    return LocalizedOperatorBundle(structure, basis, operators, None, provenance)


def dense_gamma(bundle: LocalizedOperatorBundle) -> tuple[np.ndarray, np.ndarray]:
    """Dense real H(Gamma), S(Gamma) in float64 (small bundles only)."""
    n = bundle.n_orbitals
    off = bundle.basis.atom_offsets
    ops = bundle.operators
    h = np.zeros((n, n))
    s = np.zeros((n, n))
    for b in range(ops.n_blocks):
        r0, c0 = int(off[ops.row_atom[b]]), int(off[ops.col_atom[b]])
        nr, nc = (int(v) for v in ops.block_shapes[b])
        lo, hi = int(ops.block_offsets[b]), int(ops.block_offsets[b + 1])
        h[r0:r0 + nr, c0:c0 + nc] += np.asarray(ops.h_values[lo:hi], np.float64).reshape(nr, nc)
        s[r0:r0 + nr, c0:c0 + nc] += np.asarray(ops.s_values[lo:hi], np.float64).reshape(nr, nc)
    return h, s


def suggest_window(bundle: LocalizedOperatorBundle, states: int,
                   center: float | None = None) -> tuple[float, float, int]:
    """Window (lo, hi) centred on ``center`` (default: the median Gamma
    eigenvalue) that holds ``states`` FP64 Gamma eigenvalues."""
    from scipy import linalg

    h, s = dense_gamma(bundle)
    e = linalg.eigh(h, s, eigvals_only=True)
    c = float(np.median(e)) if center is None else float(center)
    dist = np.sort(np.abs(e - c))
    half = 0.5 * (dist[states - 1] + dist[states])
    lo, hi = c - half, c + half
    return lo, hi, int(np.count_nonzero((e > lo) & (e < hi)))


def _cubic(name: str, side: int, spacing: float, cutoff: float, **kw: Any) -> SyntheticSpec:
    length = side * spacing
    return SyntheticSpec(name=name, grid=(side, side, side),
                         spacing=(spacing,) * 3, cell=(length,) * 3,
                         periodic=(True, True, True), cutoff=cutoff, **kw)


SPEC_C1 = SyntheticSpec(
    name="c1-square-8x8", grid=(8, 8, 1), spacing=(2.5, 2.5, 1.0),
    cell=(20.0, 20.0, 15.0), periodic=(True, True, False), cutoff=6.0,
    origin=(0.0, 0.0, 7.5),
)
SPEC_C2 = _cubic("c2-cubic-10", 10, 2.4, 7.0)
SPEC_C3 = _cubic("c3-cubic-16", 16, 2.4, 7.0)
SPEC_C5 = SyntheticSpec(
    name="c5-slab-2x100x100", grid=(100, 100, 2), spacing=(1.0, 2.0, 2.4),
    cell=(100.0, 200.0, 30.0), periodic=(True, True, False), cutoff=6.0,
    origin=(0.0, 0.0, 13.8),
)

YGXM = {"schema": "aospectrum.kpath/v1",
        "nodes_fractional": [[0.0, 0.5, 0.0], [0.0, 0.0, 0.0],
                             [0.5, 0.0, 0.0], [0.5, 0.5, 0.0]],
        "labels": ["Y", "G", "X", "M"], "points_per_segment": 40}


def uniform_grid_kpath(nx: int, ny: int, nz: int) -> dict[str, Any]:
    """An ``nx*ny*nz`` Monkhorst-style grid written as a k path (the k-path
    format needs node indices; the first and last points are the nodes)."""
    pts = [[i / nx, j / ny, k / nz] for i in range(nx) for j in range(ny) for k in range(nz)]
    return {"schema": "aospectrum.kpath/v1", "fractional_points": pts,
            "node_indices": [0, len(pts) - 1], "labels": ["first", "last"]}


# Energy windows (display intervals).  The solve interval the contour
# encloses is the display interval widened by 0.02 eV on each side (the
# Band continuity guard); the windows are set so that the SOLVE interval
# holds the stated number of FP64 dense generalized eigenvalues at Gamma
# (suggest_window-style search around the median Gamma eigenvalue).  c3 and
# c5 are too large for a dense Gamma solve here: their windows are scaled
# from the c2 density of states (about 560 states/eV per 13000 orbitals).
WORKLOADS: dict[str, Workload] = {
    "c1": Workload("c1", SPEC_C1, YGXM, (-3.0296, -2.2616), 40,
                   notes="64 atoms, n=832, 2D periodic, 121-point Y-G-X-M"),
    "c2": Workload("c2", SPEC_C2, YGXM, (-2.6188, -2.5204), 100,
                   notes="1000 atoms, n=13000, 3D periodic, 121 k"),
    # the window holds 87 states at Gamma (the engine's count, FP64 residuals
    # <= 1.6e-4 eV); with the 0.02 eV guards the solve interval holds about
    # 200, more than L x M = 192 resolve
    "c3": Workload("c3", SPEC_C3, uniform_grid_kpath(8, 8, 4), (-2.5845, -2.5548), 87,
                   block_size=48, notes="4096 atoms, n=53248, 256 k x 32 nodes"),
    # 48 probes; the window is 5 meV wide: 0.03 eV held more than the 192
    # search columns of L = 48, M = 4 at every k point, 0.01 eV held 118
    # states at Gamma
    "c5": Workload("c5", SPEC_C5, YGXM, (-2.5075, -2.5025), 64, block_size=48,
                   notes="20000 atoms, n=260000, two-layer slab"),
}


def small_spec(name: str = "tiny", side: int = 3, orbitals: int = 5, seed: int = 7,
               dims: int = 2) -> SyntheticSpec:
    """A tiny bundle for unit tests (dims=2: periodic square sheet)."""
    if dims == 2:
        return SyntheticSpec(name=name, grid=(side, side, 1), spacing=(2.5, 2.5, 1.0),
                             cell=(2.5 * side, 2.5 * side, 15.0),
                             periodic=(True, True, False), cutoff=4.0,
                             orbitals_per_atom=orbitals, seed=seed, origin=(0, 0, 7.5))
    return replace(_cubic(name, side, 2.4, 4.0), orbitals_per_atom=orbitals, seed=seed)


@dataclass(frozen=True)
class ServingRequestSpec:
    """One request of a seeded serving stream."""

    spec: SyntheticSpec
    kpoint_indices: tuple[int, ...]   # indices into the Y-G-X-M path
    states: int                        # states the window holds at Gamma
    arrival_s: float                   # offset from the start of the stream


def ygxm_path(points: int) -> dict[str, Any]:
    """The Y-G-X-M path with ``points`` points (3 segments)."""
    per = (points - 1) // 3
    return dict(YGXM, points_per_segment=per)


# The serving workload at the sizes it is specified with: 216-8000 atoms
# (cubic sides 6-20), 16-256 k points per request (drawn from a 301-point
# Y-G-X-M path), windows of 20-200 Gamma states.
STREAM_FULL = {"sides": tuple(range(6, 21)), "kpoints": (16, 256), "states": (20, 200),
               "path_points": 301}


def serving_stream(n_requests: int = 12, *, seed: int = 20261203, rate_per_s: float = 2.0,
                   sides: tuple[int, ...] = (6, 7, 8, 9, 10),
                   kpoints: tuple[int, int] = (4, 16), states: tuple[int, int] = (20, 60),
                   path_points: int = 121) -> list[ServingRequestSpec]:
    """A seeded stream of band requests for the serving benchmark: cubic
    bundles of side**3 atoms (216-1000 with the default sides) with 13
    (Ti-like) or 5 (C-like) orbitals per atom, k points drawn from the
    ``path_points``-point Y-G-X-M path (``ygxm_path``), windows holding
    ``states`` Gamma states, and Poisson arrivals at ``rate_per_s``.
    Bundles repeat across requests (same side, orbitals and seed), as a
    service sees repeated systems."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for _ in range(n_requests):
        side = int(rng.choice(sides))
        orbitals = int(rng.choice([13, 5]))
        spec = replace(_cubic(f"serve-{side}-{orbitals}", side, 2.4, 7.0),
                       orbitals_per_atom=orbitals, seed=1000 + side * 17 + orbitals)
        nk = int(rng.integers(kpoints[0], kpoints[1] + 1))
        ks = tuple(int(v) for v in np.sort(rng.choice(path_points, size=nk, replace=False)))
        st = int(rng.integers(states[0], states[1] + 1))
        out.append(ServingRequestSpec(spec, ks, st, t))
        t += float(rng.exponential(1.0 / rate_per_s))
    return out
