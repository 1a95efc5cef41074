"""Validated, immutable data model of an operator bundle.

The field names and the validation rules follow the reference data model
(``src/aospectrum/data.py:27-334``) because they define the
``aospectrum.operator-bundle/v1`` contract: a bundle accepted there must be
accepted here and vice versa.  Arrays are stored read-only; large value
arrays may be memory maps.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np

from .errors import InputError


def _frozen(value: Any, dtype: Any, ndim: int | None, name: str) -> np.ndarray:
    out = np.asarray(value, dtype=dtype)
    if ndim is not None and out.ndim != ndim:
        raise InputError(f"{name} must be {ndim}-dimensional")
    out.setflags(write=False)
    return out


def _set(obj: Any, **values: Any) -> None:
    for key, value in values.items():
        object.__setattr__(obj, key, value)


@dataclass(frozen=True, slots=True)
class AtomicStructure:
    """Cell vectors (rows, Angstrom), Cartesian positions and atomic numbers
    (reference ``data.py:27-68``)."""

    cell_angstrom: np.ndarray
    positions_angstrom: np.ndarray
    atomic_numbers: np.ndarray
    periodic: tuple[bool, bool, bool] = (True, True, True)
    label: str | None = None

    def __post_init__(self) -> None:
        cell = _frozen(self.cell_angstrom, np.float64, 2, "cell_angstrom")
        pos = _frozen(self.positions_angstrom, np.float64, 2, "positions_angstrom")
        num = _frozen(self.atomic_numbers, np.int32, 1, "atomic_numbers")
        if cell.shape != (3, 3) or pos.shape != (num.size, 3):
            raise InputError("structure arrays have incompatible shapes")
        if num.size == 0:
            raise InputError("structure has no atoms")
        flags = tuple(bool(v) for v in self.periodic)
        if len(flags) != 3:
            raise InputError("periodic must contain three values")
        _set(self, cell_angstrom=cell, positions_angstrom=pos,
             atomic_numbers=num, periodic=flags)

    @property
    def n_atoms(self) -> int:
        return int(self.atomic_numbers.size)


@dataclass(frozen=True, slots=True)
class OrbitalBasisLayout:
    """AO-to-atom map; each atom owns a contiguous AO range
    (reference ``data.py:71-180``)."""

    n_atoms: int
    orbital_atom: np.ndarray
    local_index: np.ndarray
    basis_family: str
    basis_identity: str
    orbital_labels: tuple[str, ...] = ()
    angular_momentum: np.ndarray | None = None
    radial_index: np.ndarray | None = None
    real_harmonic_index: np.ndarray | None = None
    spinor_width: int = 1
    metadata: dict[str, Any] = field(default_factory=dict)
    _atom_offsets: np.ndarray = field(init=False, repr=False)

    def __post_init__(self) -> None:
        owner = _frozen(self.orbital_atom, np.int32, 1, "orbital_atom")
        local = _frozen(self.local_index, np.int32, 1, "local_index")
        count = int(self.n_atoms)
        ok = (
            count > 0
            and owner.size > 0
            and owner.shape == local.shape
            and int(owner.min()) >= 0
            and int(owner.max()) < count
            and bool(np.all(owner[1:] >= owner[:-1]))
        )
        if not ok:
            raise InputError("invalid AO-to-atom layout")
        per_atom = np.bincount(owner, minlength=count)
        if np.any(per_atom == 0):
            raise InputError("each atom must own at least one AO")
        offsets = np.concatenate(([0], np.cumsum(per_atom, dtype=np.int64)))
        if not np.array_equal(local, np.arange(owner.size) - offsets[owner]):
            raise InputError("local AO indices must be contiguous within each atom")
        extra = (self.angular_momentum, self.radial_index, self.real_harmonic_index)
        present = [v is not None for v in extra]
        if any(present) and not all(present):
            raise InputError("orbital descriptors must be supplied together")
        if all(present):
            ang, rad, harm = (
                _frozen(v, np.int32, 1, n)
                for v, n in zip(extra, ("angular_momentum", "radial_index",
                                        "real_harmonic_index"))
            )
            if not (ang.shape == rad.shape == harm.shape == owner.shape):
                raise InputError("orbital descriptor lengths do not match AO layout")
        else:
            ang = rad = harm = None
        labels = tuple(str(v) for v in self.orbital_labels)
        if labels and len(labels) != owner.size:
            raise InputError("orbital_labels must contain one value per AO")
        if int(self.spinor_width) < 1:
            raise InputError("spinor_width must be positive")
        offsets.setflags(write=False)
        _set(self, n_atoms=count, orbital_atom=owner, local_index=local,
             orbital_labels=labels, angular_momentum=ang, radial_index=rad,
             real_harmonic_index=harm, spinor_width=int(self.spinor_width),
             metadata=dict(self.metadata), _atom_offsets=offsets)

    @property
    def n_orbitals(self) -> int:
        return int(self.orbital_atom.size)

    @property
    def atom_offsets(self) -> np.ndarray:
        return self._atom_offsets

    @property
    def has_real_space_descriptors(self) -> bool:
        return self.angular_momentum is not None

    def orbital_count(self, atom: int) -> int:
        return int(self._atom_offsets[atom + 1] - self._atom_offsets[atom])


@dataclass(frozen=True, slots=True)
class ElectronicFilling:
    """Closed-shell filling (reference ``data.py:183-209``)."""

    electron_count: int
    spin_degeneracy: int = 2
    fermi_energy_ev: float | None = None

    def __post_init__(self) -> None:
        electrons, degeneracy = int(self.electron_count), int(self.spin_degeneracy)
        if electrons <= 0 or degeneracy <= 0 or electrons % degeneracy:
            raise InputError("invalid closed-shell filling")
        fermi = None if self.fermi_energy_ev is None else float(self.fermi_energy_ev)
        _set(self, electron_count=electrons, spin_degeneracy=degeneracy,
             fermi_energy_ev=fermi)

    @property
    def vbm_state_number(self) -> int:
        return self.electron_count // self.spin_degeneracy

    @property
    def cbm_state_number(self) -> int:
        return self.vbm_state_number + 1


@dataclass(frozen=True, slots=True)
class LocalizedOperatorBlocks:
    """Atom-pair blocks H(R), S(R) stored as flat row-major value arrays.

    Block ``b`` couples reference-cell atom ``row_atom[b]`` to atom
    ``col_atom[b]`` translated by ``lattice_shift[b]``; its values occupy
    ``h_values[block_offsets[b]:block_offsets[b+1]]`` in row-major order
    (reference ``data.py:212-285``).
    """

    row_atom: np.ndarray
    col_atom: np.ndarray
    lattice_shift: np.ndarray
    block_offsets: np.ndarray
    block_shapes: np.ndarray
    h_values: np.ndarray
    s_values: np.ndarray

    def __post_init__(self) -> None:
        rows = _frozen(self.row_atom, np.int32, 1, "row_atom")
        cols = _frozen(self.col_atom, np.int32, 1, "col_atom")
        shifts = _frozen(self.lattice_shift, np.int32, 2, "lattice_shift")
        offsets = _frozen(self.block_offsets, np.int64, 1, "block_offsets")
        shapes = _frozen(self.block_shapes, np.int32, 2, "block_shapes")
        hv = _frozen(self.h_values, None, 1, "h_values")
        sv = _frozen(self.s_values, None, 1, "s_values")
        nb = rows.size
        if (
            nb == 0
            or cols.shape != rows.shape
            or int(rows.min()) < 0
            or int(cols.min()) < 0
            or shifts.shape != (nb, 3)
            or shapes.shape != (nb, 2)
            or offsets.shape != (nb + 1,)
            or offsets[0] != 0
        ):
            raise InputError("invalid operator block table")
        if not np.array_equal(np.diff(offsets), shapes[:, 0].astype(np.int64) * shapes[:, 1]):
            raise InputError("operator block offsets do not match block shapes")
        if hv.shape != sv.shape or hv.size != offsets[-1]:
            raise InputError("H/S values do not match the operator blocks")

        def storage(v: np.ndarray, name: str) -> np.ndarray:
            if v.dtype in (np.float32, np.complex64):
                return v
            kind = np.complex64 if np.iscomplexobj(v) else np.float32
            return _frozen(v, kind, 1, name)

        _set(self, row_atom=rows, col_atom=cols, lattice_shift=shifts,
             block_offsets=offsets, block_shapes=shapes,
             h_values=storage(hv, "h_values"), s_values=storage(sv, "s_values"))

    @property
    def n_blocks(self) -> int:
        return int(self.row_atom.size)


@dataclass(frozen=True, slots=True)
class LocalizedOperatorBundle:
    """Structure + AO layout + operator blocks (reference ``data.py:288-314``)."""

    structure: AtomicStructure
    basis: OrbitalBasisLayout
    operators: LocalizedOperatorBlocks
    filling: ElectronicFilling | None = None
    provenance: dict[str, Any] = field(default_factory=dict)

    def __post_init__(self) -> None:
        if self.structure.n_atoms != self.basis.n_atoms:
            raise InputError("structure and basis atom counts differ")
        ops = self.operators
        if int(ops.row_atom.max()) >= self.structure.n_atoms or int(
            ops.col_atom.max()
        ) >= self.structure.n_atoms:
            raise InputError("operator block references an unknown atom")
        sizes = np.diff(self.basis.atom_offsets)
        expect = np.stack((sizes[ops.row_atom], sizes[ops.col_atom]), axis=1)
        if not np.array_equal(ops.block_shapes, expect):
            raise InputError("operator block shapes do not match the AO layout")
        _set(self, provenance=dict(self.provenance))

    @property
    def n_orbitals(self) -> int:
        return self.basis.n_orbitals


@dataclass(frozen=True, slots=True)
class EnergyInterval:
    """Open interval (lower_ev, upper_ev) (reference ``data.py:317-334``)."""

    lower_ev: float
    upper_ev: float

    def __post_init__(self) -> None:
        lo, hi = float(self.lower_ev), float(self.upper_ev)
        if not (np.isfinite(lo) and np.isfinite(hi) and lo < hi):
            raise InputError("energy interval requires lower < upper")
        _set(self, lower_ev=lo, upper_ev=hi)

    def expanded(self, guard_ev: float) -> "EnergyInterval":
        g = float(guard_ev)
        return EnergyInterval(self.lower_ev - g, self.upper_ev + g)
