"""GPU parity: every CUDA entry point against the oracle / golden vectors.

Tolerances: the Bloch sum is bit-exact (real block values; complex values
within 2 ulp); shifted solves match complex128 SuperLU to 2e-4 relative
(plain complex64 factor, no refinement) or 1e-9 (FP64 refinement); CISS
eigenvalues match the reference's own CISS and the FP64 dense oracle to
1e-4 eV.
"""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

import bundles
from oracle import bloch_ref, dense_ref
from oracle import ciss_ref

pytestmark = pytest.mark.gpu

EIG_TOL_EV = 1e-4


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def torch():
    import torch as t

    return t


def _bloch(bundle, torch):
    from aospectrum_b200.engine import BlochDevice

    return BlochDevice(bundle, torch.device("cuda", 0))


@pytest.mark.parametrize("name", ["tiny2d", "tiny3d", "tinycx"])
def test_bloch_matches_reference_golden(name, golden, torch):
    b = bundles.complexified(bundles.tiny2d()) if name == "tinycx" else getattr(bundles, name)()
    ref = np.load(golden / f"bloch_{name}.npz")
    dev = _bloch(b, torch)
    try:
        assert np.array_equal(dev.indptr, ref["indptr"])
        assert np.array_equal(dev.indices, ref["indices"])
        h, s = dev.apply(np.asarray(bundles.KPOINTS))
        h, s = h.cpu().numpy(), s.cpu().numpy()
        for i in range(len(bundles.KPOINTS)):
            if name == "tinycx":
                # complex block values: products may round differently from numpy's loop
                np.testing.assert_allclose(h[i], ref[f"h{i}"], rtol=0, atol=2e-6)
                np.testing.assert_allclose(s[i], ref[f"s{i}"], rtol=0, atol=2e-7)
            else:
                assert np.array_equal(h[i], ref[f"h{i}"]), f"H(k{i}) differs"
                assert np.array_equal(s[i], ref[f"s{i}"]), f"S(k{i}) differs"
    finally:
        dev.close()


def test_bloch_c1_digest(golden, torch):
    man = json.loads((golden / "manifest.json").read_text())["bloch"]["c1"]
    dev = _bloch(bundles.c1(), torch)
    try:
        assert dev.nnz == man["nnz"]
        h, s = dev.apply(np.asarray(bundles.KPOINTS))
        h, s = h.cpu().numpy(), s.cpu().numpy()
        for i in range(len(bundles.KPOINTS)):
            assert _sha(h[i]) == man[f"h{i}"]
            assert _sha(s[i]) == man[f"s{i}"]
    finally:
        dev.close()


def _pencil_case(bundle, k, torch, tile, ordering="nested_dissection"):
    from aospectrum_b200.engine import BlochDevice, SymbolicPlan

    dev = BlochDevice(bundle, torch.device("cuda", 0))
    plan = SymbolicPlan(dev.n, dev.indptr, dev.indices, tile=tile,
                        supervariables=np.asarray(bundle.basis.atom_offsets),
                        ordering=ordering, device=torch.device("cuda", 0))
    h, s = dev.apply(np.asarray([k]))
    return dev, plan, h, s


def _factor_solve(dev, plan, h, s, shifts, rhs, torch, precision=0, adjoint=0, steps=0,
                  flags=0):
    """Factor len(shifts) pencils of one k and solve with rhs (n x L)."""
    from aospectrum_b200 import native

    n, L = rhs.shape
    P = len(shifts)
    info = plan.info
    lib = native.library()
    dv = torch.device("cuda", 0)
    factor = torch.empty(lib.aosb_factor_bytes(plan.handle, P) // 4, dtype=torch.float32,
                         device=dv)
    piv = torch.empty((P, info.n_pad), dtype=torch.int32, device=dv)
    status = torch.zeros(P, dtype=torch.int32, device=dv)
    ws = torch.empty(max(16, lib.aosb_factor_workspace_bytes(plan.handle, P, precision)),
                     dtype=torch.uint8, device=dv)
    pk = torch.zeros(P, dtype=torch.int32, device=dv)
    z = torch.tensor(np.asarray(shifts, dtype=np.complex128), device=dv)
    st = torch.cuda.current_stream().cuda_stream
    fa = native.FactorArgs(native.ABI_VERSION, native.C.sizeof(native.FactorArgs), P, precision,
                           h.data_ptr(), s.data_ptr(), pk.data_ptr(), z.data_ptr(),
                           factor.data_ptr(), piv.data_ptr(), status.data_ptr(), ws.data_ptr(), st)
    native.call("aosb_factor", plan.handle, native.C.byref(fa))
    torch.cuda.synchronize()
    assert status.cpu().numpy().tolist() == [0] * P
    b = torch.tensor(np.broadcast_to(rhs, (P, n, L)).astype(np.complex128).copy(), device=dv)
    x = torch.zeros((P, n, L), dtype=torch.complex128, device=dv)
    r = torch.zeros_like(x)
    w = torch.empty((P, info.n_pad, L), dtype=torch.complex64, device=dv)
    scratch = torch.empty(max(16, lib.aosb_solve_scratch_bytes(plan.handle, P, L)),
                          dtype=torch.uint8, device=dv)
    sa = native.SolveArgs(native.ABI_VERSION, native.C.sizeof(native.SolveArgs), P, L, adjoint,
                          flags, factor.data_ptr(), piv.data_ptr(), w.data_ptr(),
                          scratch.data_ptr(), st)
    zz = torch.conj_physical(z) if adjoint else z
    for it in range(steps + 1):
        src = b if it == 0 else r
        native.call("aosb_gather_rhs", plan.handle, P, L, src.data_ptr(), n * L, w.data_ptr(), st)
        native.call("aosb_solve", plan.handle, native.C.byref(sa))
        native.call("aosb_scatter_solution", plan.handle, P, L, w.data_ptr(), x.data_ptr(),
                    1 if it else 0, st)
        if it < steps:
            native.call("aosb_shifted_residual", n, L, P, dev.d_indptr, dev.d_indices,
                        h.data_ptr(), s.data_ptr(), dev.nnz, pk.data_ptr(), zz.data_ptr(),
                        b.data_ptr(), n * L, x.data_ptr(), r.data_ptr(), st)
    native.call("aosb_solve_check", plan.handle, native.C.byref(sa))
    torch.cuda.synchronize()
    return x.cpu().numpy()


def _splu_reference(dev, h, s, z, rhs, adjoint=False):
    from scipy import sparse
    from scipy.sparse import linalg as spl

    n = dev.n
    hm = sparse.csr_matrix((h[0].cpu().numpy().astype(np.complex128), dev.indices, dev.indptr),
                           shape=(n, n))
    sm = sparse.csr_matrix((s[0].cpu().numpy().astype(np.complex128), dev.indices, dev.indptr),
                           shape=(n, n))
    zz = np.conj(z) if adjoint else z
    return spl.splu((hm - zz * sm).tocsc()).solve(rhs.astype(np.complex128))


@pytest.mark.parametrize("case,tile,ordering", [("tiny3d", 32, "nested_dissection"),
                                                ("tiny3d", 32, "natural"),
                                                ("small2d", 64, "nested_dissection"),
                                                ("small2d", 128, "nested_dissection")])
def test_plain_factor_solve_matches_superlu(case, tile, ordering, torch):
    b = getattr(bundles, case)()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[1], torch, tile, ordering)
    try:
        rng = np.random.default_rng(1)
        rhs = (rng.standard_normal((dev.n, 8)) + 1j * rng.standard_normal((dev.n, 8)))
        shifts = [-2.3 + 0.01j, -2.0 + 0.2j, 0.5 + 0.001j]
        x = _factor_solve(dev, plan, h, s, shifts, rhs, torch)
        for p, z in enumerate(shifts):
            ref = _splu_reference(dev, h, s, z, rhs)
            err = np.linalg.norm(x[p] - ref) / np.linalg.norm(ref)
            assert err < 2e-4, (p, err)
    finally:
        dev.close()
        plan.close()


@pytest.mark.parametrize("precision,flags", [(1, 0), (2, 0), (3, 0), (1, 1)])
@pytest.mark.parametrize("case", ["small2d", "c1"])
def test_tensor_core_factor_matches_superlu(case, precision, flags, torch):
    """Split-BF16 tcgen05 Schur updates (precision 1: tensor-core panels and
    two-step updates; 2: FP32 SIMT panels; 3: one-step updates; flags 1:
    tensor-core solve updates): unrefined solves within 1e-3, FP64
    refinement to 1e-9, both directions."""
    b = getattr(bundles, case)()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[1], torch, 128)
    try:
        rng = np.random.default_rng(3)
        rhs = (rng.standard_normal((dev.n, 8)) + 1j * rng.standard_normal((dev.n, 8)))
        shifts = [-2.6 + 0.004j, -2.4 + 0.04j, -1.0 + 0.5j]
        x0 = _factor_solve(dev, plan, h, s, shifts, rhs, torch, precision=precision,
                           flags=flags)
        for adjoint in (0, 1):
            x = _factor_solve(dev, plan, h, s, shifts, rhs, torch, precision=precision,
                              adjoint=adjoint, steps=3, flags=flags)
            for p, z in enumerate(shifts):
                ref = _splu_reference(dev, h, s, z, rhs, adjoint=bool(adjoint))
                if adjoint == 0:
                    e0 = np.linalg.norm(x0[p] - ref) / np.linalg.norm(ref)
                    assert e0 < 1e-3, (p, e0)
                err = np.linalg.norm(x[p] - ref) / np.linalg.norm(ref)
                assert err < 1e-9, (adjoint, p, err)
    finally:
        dev.close()
        plan.close()


@pytest.mark.parametrize("adjoint", [0, 1])
def test_refined_solve_reaches_fp64(adjoint, torch):
    b = bundles.small2d()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[2], torch, 64)
    try:
        rng = np.random.default_rng(2)
        rhs = (rng.standard_normal((dev.n, 16)) + 1j * rng.standard_normal((dev.n, 16)))
        shifts = [-2.25 + 0.003j, -1.95 + 0.03j]
        x = _factor_solve(dev, plan, h, s, shifts, rhs, torch, adjoint=adjoint, steps=3)
        for p, z in enumerate(shifts):
            ref = _splu_reference(dev, h, s, z, rhs, adjoint=bool(adjoint))
            err = np.linalg.norm(x[p] - ref) / np.linalg.norm(ref)
            assert err < 1e-9, (p, err)
    finally:
        dev.close()
        plan.close()


def test_ubatch_dropin_host_buffers(torch):
    """aospectrum_b200_solve_complex64_ubatch_v1 with the reference's packing
    (values = H - z S per batch entry, column-major rhs)."""
    from aospectrum_b200 import native

    b = bundles.tiny3d()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[3], torch, 32)
    try:
        n, nnz, B, L = dev.n, dev.nnz, 3, 5
        hv, sv = h[0].cpu().numpy(), s[0].cpu().numpy()
        shifts = np.asarray([-2.0 + 0.05j, -1.0 + 0.01j, 0.3 + 0.4j], dtype=np.complex64)
        values = np.stack([hv - z * sv for z in shifts]).astype(np.complex64)
        rng = np.random.default_rng(4)
        rhs = (rng.standard_normal((B, L, n)) + 1j * rng.standard_normal((B, L, n))).astype(
            np.complex64)
        sol = np.zeros_like(rhs)
        ip = dev.indptr.astype(np.int32)
        req = native.UbatchRequest(native.ABI_VERSION, native.C.sizeof(native.UbatchRequest), n,
                                   nnz, B, L, ip.ctypes.data, dev.indices.ctypes.data,
                                   values.ctypes.data, rhs.ctypes.data, sol.ctypes.data)
        res = native.UbatchResult()
        rc = native.library().aospectrum_b200_solve_complex64_ubatch_v1(native.C.byref(req),
                                                                       native.C.byref(res))
        assert rc == 0 and res.status == 0, res.error_message
        assert res.iterative_refinement_steps == 2
        from scipy import sparse
        from scipy.sparse import linalg as spl

        for bi in range(B):
            a = sparse.csr_matrix((values[bi].astype(np.complex128), dev.indices, dev.indptr),
                                  shape=(n, n))
            ref = spl.splu(a.tocsc()).solve(rhs[bi].T.astype(np.complex128))
            err = np.linalg.norm(sol[bi].T - ref) / np.linalg.norm(ref)
            assert err < 1e-6, err
        # error path: a non-finite value is rejected with status 35
        values[1, 3] = np.nan
        res2 = native.UbatchResult()
        rc = native.library().aospectrum_b200_solve_complex64_ubatch_v1(native.C.byref(req),
                                                                       native.C.byref(res2))
        assert rc != 0 and res2.status == 35
    finally:
        dev.close()
        plan.close()


def _engine(bundle, precision, tensor_cores=True, **kw):
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.engine import BandEngine

    return BandEngine(bundle, CissSettings(**kw),
                      EngineSettings(precision=precision, tensor_cores=tensor_cores))


@pytest.mark.parametrize("precision,tc", [("plain", False), ("mixed", False), ("mixed", True)])
@pytest.mark.parametrize("key", ["tiny3d_k2", "small2d_k2", "tinycx_k1", "c1_k0"])
def test_engine_ciss_matches_reference(key, precision, tc, golden, torch):
    from aospectrum_b200.data import EnergyInterval

    case = json.loads((golden / "manifest.json").read_text())["ciss"][key]
    ref_e = np.load(golden / "ciss.npz")[f"{key}_energies"]
    name = case["bundle"]
    b = bundles.complexified(bundles.tiny2d()) if name == "tinycx" else getattr(bundles, name)()
    eng = _engine(b, precision, tc, integration_points=case["integration_points"],
                  block_size=case["block_size"], moment_size=case["moment_size"])
    try:
        lo, hi = case["interval"]
        res, _ = eng.solve_kpoints([bundles.KPOINTS[case["k_index"]]], EnergyInterval(lo, hi))
        got = np.sort(res[0].energies_ev.astype(np.float64))
        assert got.size == ref_e.size, (got, ref_e)
        assert np.max(np.abs(got - np.sort(ref_e))) < EIG_TOL_EV
        # FP64 dense oracle
        pair = eng.host_pair(bundles.KPOINTS[case["k_index"]])
        hd, sd = dense_ref.dense_pair(pair.hamiltonian.indptr, pair.hamiltonian.indices,
                                      pair.hamiltonian.data, pair.overlap.data, eng.n)
        exact = dense_ref.window(dense_ref.eigenvalues(hd, sd), lo, hi)
        assert exact.size == got.size
        assert np.max(np.abs(got - exact)) < EIG_TOL_EV
        # residual no worse than the reference's complex64 CISS
        assert res[0].maximum_residual_ev <= max(case["max_residual_ev"], 1e-6) * 1.01
    finally:
        eng.close()


def test_dropin_solver_classes(golden, torch):
    """B200CissSolver / NativeB200ShiftSolver behave like the reference's
    CudssCissSolver / NativeCudssShiftSolver on host CSR matrices."""
    from aospectrum_b200.ciss import CissSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.solvers import B200CissSolver, NativeB200ShiftSolver
    from fake_engine import OracleEngine

    case = json.loads((golden / "manifest.json").read_text())["ciss"]["small2d_k2"]
    ref_e = np.sort(np.load(golden / "ciss.npz")["small2d_k2_energies"])
    b = bundles.small2d()
    settings = CissSettings(integration_points=case["integration_points"],
                            block_size=case["block_size"], moment_size=case["moment_size"])
    pair = OracleEngine(b, settings, None).host_pair(bundles.KPOINTS[case["k_index"]])
    solver = B200CissSolver(settings)
    try:
        res = solver.solve_interval(pair, EnergyInterval(*case["interval"]))
        got = np.sort(res.energies_ev.astype(np.float64))
        assert got.size == ref_e.size and np.max(np.abs(got - ref_e)) < EIG_TOL_EV
        assert res.complete
    finally:
        solver.close()
    shifted = NativeB200ShiftSolver()
    try:
        rng = np.random.default_rng(5)
        rhs = (rng.standard_normal((b.n_orbitals, 6)) + 1j * rng.standard_normal(
            (b.n_orbitals, 6))).astype(np.complex64)
        shifts = np.asarray([-2.3 + 0.01j, -2.0 + 0.1j], dtype=np.complex64)
        out = shifted.solve_shifted(pair, shifts, rhs)
        assert out.solutions.shape == (2, b.n_orbitals, 6)
        from scipy.sparse import linalg as spl

        for i, z in enumerate(shifts):
            a = (pair.hamiltonian.astype(np.complex128)
                 - complex(z) * pair.overlap.astype(np.complex128)).tocsc()
            ref = spl.splu(a).solve(rhs.astype(np.complex128))
            assert np.linalg.norm(out.solutions[i] - ref) / np.linalg.norm(ref) < 1e-6
        assert "numeric_factorization" in out.stage_seconds
    finally:
        shifted.close()


def test_row_block_residual_matches_per_row(torch):
    """aosb_shifted_residual_blocks == aosb_shifted_residual (FP64)."""
    from aospectrum_b200 import native
    from aospectrum_b200.engine import row_blocks

    b = bundles.small2d()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[1], torch, 64)
    try:
        n, L, P = dev.n, 40, 3
        dv = torch.device("cuda", 0)
        rng = np.random.default_rng(9)
        x = torch.tensor(rng.standard_normal((P, n, L)) + 1j * rng.standard_normal((P, n, L)),
                         device=dv)
        bb = torch.tensor(rng.standard_normal((P, n, L)) + 1j * rng.standard_normal((P, n, L)),
                          device=dv)
        z = torch.tensor(np.asarray([-2.0 + 0.1j, 0.5 + 0.01j, -1.0 + 1.0j]), device=dv)
        pk = torch.zeros(P, dtype=torch.int32, device=dv)
        rb = torch.from_numpy(row_blocks(dev.indptr, dev.indices,
                                         starts=np.asarray(b.basis.atom_offsets)[:-1])).to(dv)
        r1 = torch.empty_like(x)
        r2 = torch.empty_like(x)
        st = torch.cuda.current_stream().cuda_stream
        native.call("aosb_shifted_residual", n, L, P, dev.d_indptr, dev.d_indices, h.data_ptr(),
                    s.data_ptr(), dev.nnz, pk.data_ptr(), z.data_ptr(), bb.data_ptr(), n * L,
                    x.data_ptr(), r1.data_ptr(), st)
        max_rows = int(torch.diff(rb).max().item())
        native.call("aosb_shifted_residual_blocks", n, L, P, rb.numel() - 1, rb.data_ptr(),
                    max_rows, dev.d_indptr, dev.d_indices, h.data_ptr(), s.data_ptr(), dev.nnz,
                    pk.data_ptr(), z.data_ptr(), bb.data_ptr(), n * L, x.data_ptr(),
                    r2.data_ptr(), st)
        torch.cuda.synchronize()
        a, c = r1.cpu().numpy(), r2.cpu().numpy()
        assert np.max(np.abs(a - c)) <= 1e-11 * np.max(np.abs(a))
    finally:
        dev.close()
        plan.close()


@pytest.mark.parametrize("bundle_name,max_rows,ncols",
                         [("small2d", None, 40), ("small2d", 16, 7), ("c1", None, 128),
                          ("c1", 4, 33)])
def test_row_block_spmm_matches_per_row(bundle_name, max_rows, ncols, torch):
    """aosb_spmm_blocks == aosb_spmm (FP64 sums in another order) and the
    complex128 product A x in scipy; blocks split to at most max_rows rows."""
    import scipy.sparse as sp

    from aospectrum_b200 import native
    from aospectrum_b200.engine import BlochDevice, row_blocks

    b = getattr(bundles, bundle_name)()
    dv = torch.device("cuda", 0)
    dev = BlochDevice(b, dv)
    try:
        h, _ = dev.apply(np.asarray([bundles.KPOINTS[1]]))
        n = dev.n
        rb_h = row_blocks(dev.indptr, dev.indices, max_rows=max_rows or 16,
                          starts=np.asarray(b.basis.atom_offsets)[:-1])
        rb = torch.from_numpy(rb_h).to(dv)
        rows = int(np.diff(rb_h).max())
        rng = np.random.default_rng(11)
        ld = ncols + 3   # strided x and y
        x = torch.tensor(rng.standard_normal((n, ld)) + 1j * rng.standard_normal((n, ld)),
                         device=dv)
        y1 = torch.zeros((n, ld), dtype=torch.complex128, device=dv)
        y2 = torch.zeros_like(y1)
        st = torch.cuda.current_stream().cuda_stream
        native.call("aosb_spmm", n, ncols, dev.d_indptr, dev.d_indices, h.data_ptr(),
                    x.data_ptr(), ld, y1.data_ptr(), ld, st)
        native.call("aosb_spmm_blocks", n, ncols, rb.numel() - 1, rb.data_ptr(), rows,
                    dev.d_indptr, dev.d_indices, h.data_ptr(), dev.nnz, x.data_ptr(), ld,
                    y2.data_ptr(), ld, st)
        torch.cuda.synchronize()
        a, c = y1.cpu().numpy(), y2.cpu().numpy()
        assert np.max(np.abs(a - c)) <= 1e-12 * np.max(np.abs(a))
        assert np.all(c[:, ncols:] == 0)
        m = sp.csr_matrix((h[0].cpu().numpy().astype(np.complex128), dev.indices, dev.indptr),
                          shape=(n, n))
        ref = m @ x.cpu().numpy()[:, :ncols]
        assert np.max(np.abs(c[:, :ncols] - ref)) <= 1e-12 * np.max(np.abs(ref))
    finally:
        dev.close()


@pytest.mark.parametrize("adjoint", [0, 1])
def test_graph_replayed_solve_equals_direct(adjoint, torch):
    """AOSB_SOLVE_GRAPH: the first call captures, later calls replay; every
    result equals the directly launched solve bit for bit."""
    from aospectrum_b200 import native

    b = bundles.small2d()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[1], torch, 64)
    try:
        rng = np.random.default_rng(4)
        rhs = (rng.standard_normal((dev.n, 8)) + 1j * rng.standard_normal((dev.n, 8)))
        shifts = [-2.3 + 0.01j, -2.0 + 0.2j]
        ref = _factor_solve(dev, plan, h, s, shifts, rhs, torch, adjoint=adjoint, steps=1)
        for _ in range(3):
            got = _factor_solve(dev, plan, h, s, shifts, rhs, torch, adjoint=adjoint, steps=1,
                                flags=native.SOLVE_GRAPH)
            assert np.array_equal(got, ref)
    finally:
        dev.close()
        plan.close()


@pytest.mark.parametrize("adjoint,L", [(0, 32), (1, 32), (0, 40), (1, 40)])
def test_tc_solve_two_ctas_per_sm_equals_one(adjoint, L, torch):
    """The tensor-core solve update with two CTAs per SM (shallow rings, one
    epilogue box per warp) gives the one-CTA result bit for bit (each X tile
    gets one reduce-add per step in both forms); L = 40 adds an 8-column
    strip."""
    from aospectrum_b200 import native

    b = bundles.c1()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[1], torch, 128, "natural")
    lib = native.library()
    try:
        rng = np.random.default_rng(8)
        rhs = (rng.standard_normal((dev.n, L)) + 1j * rng.standard_normal((dev.n, L)))
        shifts = [-2.6 + 0.02j, -1.0 + 0.3j, -2.2 + 0.1j]
        kw = dict(precision=native.PRECISION_BF16X3, adjoint=adjoint, steps=1,
                  flags=native.SOLVE_TENSOR_CORES)
        lib.aosb_solve_set_ctas_per_sm(1)
        one = _factor_solve(dev, plan, h, s, shifts, rhs, torch, **kw)
        lib.aosb_solve_set_ctas_per_sm(2)
        two = _factor_solve(dev, plan, h, s, shifts, rhs, torch, **kw)
        assert np.array_equal(one, two)
    finally:
        lib.aosb_solve_set_ctas_per_sm(0)
        dev.close()
        plan.close()


def test_two_step_factor_matches_one_step(torch):
    """Two-step (K = 256) Schur updates give the factor of the one-step
    updates up to split-BF16 rounding (same pivots on this pencil)."""
    from aospectrum_b200 import native

    b = bundles.c1()
    dev, plan, h, s = _pencil_case(b, bundles.KPOINTS[1], torch, 128, "natural")
    try:
        rng = np.random.default_rng(5)
        rhs = (rng.standard_normal((dev.n, 4)) + 1j * rng.standard_normal((dev.n, 4)))
        shifts = [-2.6 + 0.02j, -1.0 + 0.3j]
        one = _factor_solve(dev, plan, h, s, shifts, rhs, torch,
                            precision=native.PRECISION_BF16X3_ONE_STEP)
        two = _factor_solve(dev, plan, h, s, shifts, rhs, torch,
                            precision=native.PRECISION_BF16X3)
        for p in range(len(shifts)):
            rel = np.linalg.norm(two[p] - one[p]) / np.linalg.norm(one[p])
            assert rel < 1e-3, (p, rel)
    finally:
        dev.close()
        plan.close()
