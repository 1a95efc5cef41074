"""Reader and writer of the ``aospectrum.operator-bundle/v1`` directory.

The directory layout is an external contract shared with the reference
(``src/aospectrum/bundle.py:21-191``), so file names, JSON keys and array
dtypes are kept identical:

    manifest.json            schema, periodic, structure_label, units
    basis/layout.json        n_atoms, basis_family, basis_identity, ...
    filling.json             optional closed-shell filling
    provenance.json          optional free-form JSON
    structure/{cell,positions,atomic_numbers}.npy
    basis/{orbital_atom,local_index}.npy (+ optional descriptors)
    operators/{row_atom,col_atom,lattice_shift,block_offsets,block_shapes,
               h_values,s_values}.npy

Large arrays are memory-mapped on load (``mmap_mode='r'``) exactly as the
reference does, so opening a bundle costs no copy until the values are used.
"""

from __future__ import annotations

import json
from pathlib import Path
from typing import Any

import numpy as np

from .data import (
    AtomicStructure,
    ElectronicFilling,
    LocalizedOperatorBlocks,
    LocalizedOperatorBundle,
    OrbitalBasisLayout,
)
from .errors import InputError

SCHEMA = "aospectrum.operator-bundle/v1"

_STRUCTURE = ("cell", "positions", "atomic_numbers")
_OPERATORS = ("row_atom", "col_atom", "lattice_shift", "block_offsets",
              "block_shapes", "h_values", "s_values")
_DESCRIPTORS = ("angular_momentum", "radial_index", "real_harmonic_index")


def _read_json(path: Path) -> dict[str, Any]:
    try:
        obj = json.loads(path.read_text(encoding="utf-8"))
    except (OSError, UnicodeError, json.JSONDecodeError) as exc:
        raise InputError(f"cannot read {path}: {exc}") from exc
    if not isinstance(obj, dict):
        raise InputError(f"{path} must contain a JSON object")
    return obj


def _dump_json(path: Path, obj: dict[str, Any]) -> None:
    path.write_text(json.dumps(obj, indent=2, sort_keys=True) + "\n", encoding="utf-8")


def load_bundle(root: str | Path, *, mmap_mode: str | None = "r") -> LocalizedOperatorBundle:
    """Open a bundle directory; arrays stay memory-mapped when ``mmap_mode``
    is set (reference ``bundle.py:41-114``)."""
    base = Path(root).expanduser().resolve()
    manifest = _read_json(base / "manifest.json")
    if manifest.get("schema") != SCHEMA:
        raise InputError(f"unsupported operator bundle: {manifest.get('schema')}")
    layout = _read_json(base / "basis" / "layout.json")

    def npy(rel: str) -> np.ndarray:
        try:
            return np.load(base / rel, allow_pickle=False, mmap_mode=mmap_mode)
        except (OSError, ValueError) as exc:
            raise InputError(f"cannot read bundle array {rel}: {exc}") from exc

    filling = None
    if (base / "filling.json").is_file():
        raw = _read_json(base / "filling.json")
        filling = ElectronicFilling(
            electron_count=raw["electron_count"],
            spin_degeneracy=raw.get("spin_degeneracy", 2),
            fermi_energy_ev=raw.get("fermi_energy_ev"),
        )
    provenance = (
        _read_json(base / "provenance.json")
        if (base / "provenance.json").is_file()
        else {}
    )
    described = bool(layout.get("has_real_space_descriptors", False))
    desc = {k: (npy(f"basis/{k}.npy") if described else None) for k in _DESCRIPTORS}
    structure = AtomicStructure(
        *(npy(f"structure/{k}.npy") for k in _STRUCTURE),
        periodic=tuple(manifest.get("periodic", (True, True, True))),
        label=manifest.get("structure_label"),
    )
    basis = OrbitalBasisLayout(
        n_atoms=layout["n_atoms"],
        orbital_atom=npy("basis/orbital_atom.npy"),
        local_index=npy("basis/local_index.npy"),
        basis_family=str(layout["basis_family"]),
        basis_identity=str(layout["basis_identity"]),
        orbital_labels=tuple(layout.get("orbital_labels", ())),
        spinor_width=layout.get("spinor_width", 1),
        metadata=dict(layout.get("metadata", {})),
        **desc,
    )
    operators = LocalizedOperatorBlocks(*(npy(f"operators/{k}.npy") for k in _OPERATORS))
    return LocalizedOperatorBundle(structure, basis, operators, filling, provenance)


def write_bundle(bundle: LocalizedOperatorBundle, root: str | Path) -> Path:
    """Write ``bundle`` into an empty (or absent) directory
    (reference ``bundle.py:117-191``)."""
    base = Path(root).expanduser().resolve()
    if base.exists() and (not base.is_dir() or any(base.iterdir())):
        raise InputError(f"bundle destination is not empty: {base}")
    for sub in ("structure", "basis", "operators"):
        (base / sub).mkdir(parents=True, exist_ok=True)
    st, bs, op = bundle.structure, bundle.basis, bundle.operators
    arrays: dict[str, np.ndarray] = {
        "structure/cell.npy": st.cell_angstrom,
        "structure/positions.npy": st.positions_angstrom,
        "structure/atomic_numbers.npy": st.atomic_numbers,
        "basis/orbital_atom.npy": bs.orbital_atom,
        "basis/local_index.npy": bs.local_index,
    }
    for key in _OPERATORS:
        arrays[f"operators/{key}.npy"] = getattr(op, key)
    if bs.has_real_space_descriptors:
        for key in _DESCRIPTORS:
            arrays[f"basis/{key}.npy"] = getattr(bs, key)
    for rel, values in arrays.items():
        np.save(base / rel, values, allow_pickle=False)
    _dump_json(base / "manifest.json", {
        "schema": SCHEMA,
        "periodic": list(st.periodic),
        "structure_label": st.label,
        "hamiltonian_unit": "eV",
        "length_unit": "angstrom",
    })
    _dump_json(base / "basis" / "layout.json", {
        "n_atoms": bs.n_atoms,
        "basis_family": bs.basis_family,
        "basis_identity": bs.basis_identity,
        "orbital_labels": list(bs.orbital_labels),
        "has_real_space_descriptors": bs.has_real_space_descriptors,
        "spinor_width": bs.spinor_width,
        "metadata": bs.metadata,
    })
    if bundle.filling is not None:
        _dump_json(base / "filling.json", {
            "mode": "closed_shell",
            "electron_count": bundle.filling.electron_count,
            "spin_degeneracy": bundle.filling.spin_degeneracy,
            "fermi_energy_ev": bundle.filling.fermi_energy_ev,
        })
    _dump_json(base / "provenance.json", bundle.provenance)
    return base
