"""Generates the golden vectors under tests/golden/ from the REFERENCE itself.

Run in a container where the reference sources are available, passing
their root (the directory holding src/aospectrum and examples/):
    python tests/golden/make_golden.py REFERENCE_ROOT
    python tests/golden/make_golden.py REFERENCE_ROOT --c2 0,37

It imports the reference's Python package (yumiaoyi-o/AOSpectrum,
src/aospectrum) and records, for seeded bundles written by
aospectrum_b200.write_bundle and read back by the reference's load_bundle:
  * BlochPattern.from_bundle + BlochWorkspace.update outputs
    (CSR pattern and H(k), S(k) values; SHA-256 digests for c1);
  * _contour_geometry outputs;
  * CudssCissSolver.solve_interval results with a scipy SuperLU shifted
    solver injected through its shifted_solver seam (ciss.py:253-264),
    together with the rhs block the reference passes to that solver;
  * read_kpath on the reference's example k path;
  * the bands.csv / summary.json of the reference's run_band on a tiny
    bundle (same injected solver).
With ``--c2 K1,K2,...`` only the 1000-atom c2 workload is recorded
(tests/golden/c2.npz and manifest_c2.json): the reference's Bloch digests at
those k-path indices, FP64 dense generalized eigenvalues of the same H(k),
S(k) in the solve interval, and the reference's complex64 CISS
(solve_interval) with exact complex128 dense-LU shifted solves injected
through its shifted_solver seam: its eigenvalues and maximum residual.  One
LU of H - z S serves the node z and its conjugate partner, since
(H - z S)^H = H - conj(z) S for Hermitian H, S.  This takes tens of minutes
of host time (16 dense LUs of n = 13000 per k point).
The reference's cuDSS extension is not importable here and is not needed.
"""

from __future__ import annotations

import hashlib
import json
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "tests"))

import bundles  # noqa: E402
from aospectrum_b200 import bundle as my_bundle  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(reference_root: str) -> None:
    sys.path.insert(0, str(Path(reference_root) / "src"))
    import aospectrum.band as rband
    from aospectrum.bundle import load_bundle
    from aospectrum.ciss import CissSettings, CudssCissSolver, ShiftedResult, _contour_geometry
    from aospectrum.data import EnergyInterval
    from aospectrum.sparse import BlochPattern
    from scipy.sparse import linalg as splinalg

    class SpluShifted:
        """Exact (complex128 SuperLU) shifted solves for the reference CISS."""

        def __init__(self):
            self.rhs = None
            self.shifts = []

        def solve_shifted(self, matrices, shifts, rhs):
            self.rhs = np.array(rhs)
            out = np.empty((shifts.size,) + rhs.shape, dtype=np.complex64)
            h = matrices.hamiltonian.astype(np.complex128)
            s = matrices.overlap.astype(np.complex128)
            for i, z in enumerate(shifts):
                self.shifts.append(complex(z))
                lu = splinalg.splu((h - complex(z) * s).tocsc())
                out[i] = lu.solve(rhs.astype(np.complex128))
            return ShiftedResult(out, {}, None)

        def close(self):
            pass

    tmp = Path(tempfile.mkdtemp())
    cases = {"tiny2d": bundles.tiny2d(), "tiny3d": bundles.tiny3d(),
             "tinycx": bundles.complexified(bundles.tiny2d()), "small2d": bundles.small2d()}
    manifest: dict = {"generator": "tests/golden/make_golden.py", "bloch": {}, "ciss": {}}
    for name, b in cases.items():
        path = tmp / name
        my_bundle.write_bundle(b, path)
        rb = load_bundle(path)
        pat = BlochPattern.from_bundle(rb)
        ws = pat.workspace(complex_values=True)
        arrays = {"indptr": np.asarray(pat.csr_indptr), "indices": np.asarray(pat.csr_indices)}
        for i, k in enumerate(bundles.KPOINTS):
            pair = ws.update(rb, k)
            arrays[f"h{i}"] = pair.hamiltonian.data.copy()
            arrays[f"s{i}"] = pair.overlap.data.copy()
        if name == "small2d":
            manifest["bloch"][name] = {key: sha(v) for key, v in arrays.items()}
        else:
            np.savez_compressed(HERE / f"bloch_{name}.npz", **arrays)
    # c1: digests only (bit-exact comparison)
    c1 = bundles.c1()
    my_bundle.write_bundle(c1, tmp / "c1")
    rb = load_bundle(tmp / "c1")
    pat = BlochPattern.from_bundle(rb)
    ws = pat.workspace(complex_values=True)
    dig = {"indptr": sha(np.asarray(pat.csr_indptr)), "indices": sha(np.asarray(pat.csr_indices)),
           "nnz": int(pat.nnz)}
    for i, k in enumerate(bundles.KPOINTS):
        pair = ws.update(rb, k)
        dig[f"h{i}"] = sha(pair.hamiltonian.data)
        dig[f"s{i}"] = sha(pair.overlap.data)
    manifest["bloch"]["c1"] = dig
    # contour geometry
    geo = {}
    for i, (lo, hi, npts) in enumerate([(-2.0, -1.0, 32), (-3.0496, -2.2416, 32), (0.5, 0.9, 16)]):
        s, z, w = _contour_geometry(EnergyInterval(lo, hi), CissSettings(integration_points=npts))
        geo[f"shifts{i}"], geo[f"nodes{i}"], geo[f"weights{i}"] = s, z, w
        geo[f"interval{i}"] = np.array([lo, hi, npts])
    np.savez_compressed(HERE / "contour.npz", **geo)
    # CISS on small cases
    ciss_arrays = {}
    ciss_cases = [("tiny3d", (-3.2, -1.6), 2, 16, 8, 4), ("small2d", (-2.6, -1.9), 2, 32, 16, 4),
                  ("tinycx", (-3.0, -1.0), 1, 16, 8, 4)]
    for name, (lo, hi), kidx, npts, block, mom in ciss_cases:
        rb = load_bundle(tmp / name)
        pat = BlochPattern.from_bundle(rb)
        ws = pat.workspace(complex_values=True)
        pair = ws.update(rb, bundles.KPOINTS[kidx])
        shim = SpluShifted()
        settings = CissSettings(integration_points=npts, block_size=block, moment_size=mom)
        res = CudssCissSolver(settings, shifted_solver=shim).solve_interval(
            pair, EnergyInterval(lo, hi))
        key = f"{name}_k{kidx}"
        manifest["ciss"][key] = {"bundle": name, "interval": [lo, hi], "k_index": kidx,
                                 "integration_points": npts, "block_size": block,
                                 "moment_size": mom, "max_residual_ev": res.maximum_residual_ev,
                                 "complete": res.complete, "count": int(res.energies_ev.size)}
        ciss_arrays[f"{key}_energies"] = np.asarray(res.energies_ev)
        ciss_arrays[f"{key}_rhs"] = shim.rhs
    # c1 at two k points (40-state window)
    rb = load_bundle(tmp / "c1")
    pat = BlochPattern.from_bundle(rb)
    ws = pat.workspace(complex_values=True)
    for kidx in (0, 2):
        pair = ws.update(rb, bundles.KPOINTS[kidx])
        shim = SpluShifted()
        res = CudssCissSolver(CissSettings(), shifted_solver=shim).solve_interval(
            pair, EnergyInterval(-3.0496 - 0.02, -2.2416 + 0.02))
        key = f"c1_k{kidx}"
        manifest["ciss"][key] = {"bundle": "c1", "interval": [-3.0696, -2.2216], "k_index": kidx,
                                 "integration_points": 32, "block_size": 32, "moment_size": 4,
                                 "max_residual_ev": res.maximum_residual_ev,
                                 "complete": res.complete, "count": int(res.energies_ev.size)}
        ciss_arrays[f"{key}_energies"] = np.asarray(res.energies_ev)
    np.savez_compressed(HERE / "ciss.npz", **ciss_arrays)
    # k path
    kp = rband.read_kpath(Path(reference_root) / "examples" / "band" / "YGXM-121.json")
    np.savez_compressed(HERE / "kpath_ygxm.npz", points=kp.fractional_points,
                        nodes=kp.node_indices, labels=np.asarray(kp.node_labels))
    # reference run_band on tiny2d with the injected solver
    orig = rband.CudssCissSolver
    rband.CudssCissSolver = lambda settings: CudssCissSolver(settings, shifted_solver=SpluShifted())
    import aospectrum.cli as rcli

    work = tmp / "band"
    work.mkdir()
    shutil.copytree(tmp / "tiny2d", work / "system.aobundle")
    kpath = {"schema": "aospectrum.kpath/v1", "nodes_fractional": [[0, 0.5, 0], [0, 0, 0],
                                                                    [0.5, 0, 0]],
             "labels": ["Y", "G", "X"], "points_per_segment": 3}
    (work / "path.json").write_text(json.dumps(kpath))
    (work / "band.toml").write_text(
        '[input]\nbundle = "system.aobundle"\n[band]\nkpath = "path.json"\n'
        'energy_interval_ev = [-3.0, -1.0]\nenergy_reference = "input_zero"\n'
        '[solver]\nintegration_points = 16\nblock_size = 8\nmoment_size = 4\n'
        '[output]\ndirectory = "out"\n')
    try:
        rcli.run_band(work / "band.toml")
    except Exception as exc:  # matplotlib may be missing after the CSV/JSON
        print("run_band ended with", type(exc).__name__, exc)
    finally:
        rband.CudssCissSolver = orig
    out = work / "out"
    if not (out / "bands.csv").exists():
        out = work / ".out.publish"
    golden_band = HERE / "band_tiny2d"
    if golden_band.exists():
        shutil.rmtree(golden_band)
    golden_band.mkdir()
    shutil.copy(out / "bands.csv", golden_band / "bands.csv")
    shutil.copy(out / "summary.json", golden_band / "summary.json")
    (golden_band / "band.toml").write_text((work / "band.toml").read_text())
    (golden_band / "path.json").write_text((work / "path.json").read_text())
    (HERE / "manifest.json").write_text(json.dumps(manifest, indent=2, sort_keys=True) + "\n")
    shutil.rmtree(tmp)
    print("golden vectors written to", HERE)


def main_c2(reference_root: str, kidx: list[int], name: str = "c2") -> None:
    import time

    sys.path.insert(0, str(Path(reference_root) / "src"))
    from aospectrum.bundle import load_bundle
    from aospectrum.ciss import CissSettings, CudssCissSolver, ShiftedResult
    from aospectrum.data import EnergyInterval
    from aospectrum.sparse import BlochPattern
    from scipy import linalg

    from aospectrum_b200 import synth
    from aospectrum_b200.kpath import kpath_from_dict

    class DenseShifted:
        """Exact complex128 dense-LU shifted solves; the LU of node z also
        solves its conjugate partner with the conjugate transpose."""

        def __init__(self):
            self.cache: dict[complex, np.ndarray] = {}
            self.factorizations = 0

        def solve_shifted(self, matrices, shifts, rhs):
            out = np.empty((shifts.size,) + rhs.shape, dtype=np.complex64)
            b = rhs.astype(np.complex128)
            for i, z in enumerate(shifts):
                z = complex(z)
                if z in self.cache:
                    out[i] = self.cache.pop(z)
                    continue
                a = matrices.hamiltonian.toarray().astype(np.complex128)
                a -= z * matrices.overlap.toarray().astype(np.complex128)
                lu = linalg.lu_factor(a, overwrite_a=True, check_finite=False)
                del a
                self.factorizations += 1
                out[i] = linalg.lu_solve(lu, b, check_finite=False)
                self.cache[z.conjugate()] = linalg.lu_solve(lu, b, trans=2, check_finite=False)
            return ShiftedResult(out, {}, None)

        def close(self):
            pass

    w = synth.WORKLOADS["c2"]
    kp = kpath_from_dict(w.kpath)
    guard = 0.02
    lo, hi = w.window_ev[0] - guard, w.window_ev[1] + guard
    tmp = Path(tempfile.mkdtemp())
    my_bundle.write_bundle(synth.generate_bundle(w.spec), tmp / "c2")
    rb = load_bundle(tmp / "c2")
    pat = BlochPattern.from_bundle(rb)
    ws = pat.workspace(complex_values=True)
    manifest = {"generator": "tests/golden/make_golden.py --c2", "workload": "c2",
                "interval": [lo, hi], "nnz": int(pat.nnz),
                "indptr": sha(np.asarray(pat.csr_indptr)),
                "indices": sha(np.asarray(pat.csr_indices)), "kpoints": {}}
    arrays = {}
    for i in kidx:
        t0 = time.perf_counter()
        pair = ws.update(rb, kp.fractional_points[i])
        rec = {"k": [float(v) for v in kp.fractional_points[i]],
               "h": sha(pair.hamiltonian.data), "s": sha(pair.overlap.data)}
        h = pair.hamiltonian.toarray().astype(np.complex128)
        s_ = pair.overlap.toarray().astype(np.complex128)
        exact = linalg.eigh(0.5 * (h + h.conj().T), 0.5 * (s_ + s_.conj().T),
                            eigvals_only=True, subset_by_value=(lo, hi), check_finite=False)
        del h, s_
        arrays[f"k{i}_fp64"] = np.sort(exact)
        shim = DenseShifted()
        res = CudssCissSolver(CissSettings(), shifted_solver=shim).solve_interval(
            pair, EnergyInterval(lo, hi))
        arrays[f"k{i}_energies"] = np.asarray(res.energies_ev)
        rec.update({"max_residual_ev": res.maximum_residual_ev, "complete": res.complete,
                    "count": int(res.energies_ev.size), "fp64_count": int(exact.size),
                    "factorizations": shim.factorizations,
                    "seconds": round(time.perf_counter() - t0, 1)})
        manifest["kpoints"][str(i)] = rec
        print("c2 k", i, rec, flush=True)
    np.savez_compressed(HERE / f"{name}.npz", **arrays)
    (HERE / f"manifest_{name}.json").write_text(json.dumps(manifest, indent=2, sort_keys=True) +
                                                "\n")
    shutil.rmtree(tmp)
    print("c2 golden vectors written to", HERE)


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("reference_root", help="root of the reference sources")
    ap.add_argument("--c2", default="", help="record only c2 at these k-path indices")
    ap.add_argument("--c2-name", default="c2",
                    help="file stem of the c2 record (c2 -> c2.npz, manifest_c2.json)")
    a = ap.parse_args()
    if a.c2:
        main_c2(a.reference_root, [int(v) for v in a.c2.split(",")], a.c2_name)
    else:
        main(a.reference_root)
