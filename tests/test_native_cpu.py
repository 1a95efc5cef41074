"""The C-ABI library without a GPU: it loads, exports every symbol the
header declares, and its host-only entry points (pattern build, symbolic
analysis, request validation) behave."""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import bundles
from aospectrum_b200 import native
from oracle import bloch_ref

HEADER = Path(__file__).resolve().parent.parent / "include" / "aospectrum_b200.h"


def header_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(aos\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = native.library()
    names = header_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
        assert name in native.exported_symbols(), name
    assert lib.aosb_abi_version() == native.ABI_VERSION
    assert b"sm_100a" in lib.aosb_build_info()


def _bloch_create(b, drop_block=None):
    ops = b.operators
    keep = np.ones(ops.n_blocks, bool)
    if drop_block is not None:
        keep[drop_block] = False
    rows = np.ascontiguousarray(ops.row_atom[keep], np.int32)
    cols = np.ascontiguousarray(ops.col_atom[keep], np.int32)
    sh = np.ascontiguousarray(ops.lattice_shift[keep], np.int32)
    sizes = np.diff(ops.block_offsets)[keep]
    bo = np.concatenate(([0], np.cumsum(sizes))).astype(np.int64)
    off = np.ascontiguousarray(b.basis.atom_offsets, np.int64)
    h = C.c_void_p()
    buf = C.create_string_buffer(512)
    rc = native.library().aosb_bloch_create(b.n_orbitals, b.basis.n_atoms, off.ctypes.data,
                                            int(keep.sum()), rows.ctypes.data, cols.ctypes.data,
                                            sh.ctypes.data, bo.ctypes.data, C.byref(h), buf, 512)
    return rc, h, buf.value


@pytest.mark.parametrize("name", ["tiny2d", "tiny3d", "small2d"])
def test_host_pattern_builder_matches_reference(name, golden):
    b = getattr(bundles, name)()
    rc, h, _ = _bloch_create(b)
    assert rc == 0
    lib = native.library()
    nnz, nsh = C.c_int64(), C.c_int64()
    lib.aosb_bloch_info(h, C.byref(nnz), C.byref(nsh))
    ip = np.empty(b.n_orbitals + 1, np.int64)
    ix = np.empty(nnz.value, np.int32)
    shifts = np.empty((nsh.value, 3), np.int32)
    bsh = np.empty(b.operators.n_blocks, np.int32)
    lib.aosb_bloch_export(h, ip.ctypes.data, ix.ctypes.data, shifts.ctypes.data, bsh.ctypes.data)
    pat = bloch_ref.build_pattern(b)
    assert np.array_equal(ip, pat.indptr) and np.array_equal(ix, pat.indices)
    assert np.array_equal(shifts, pat.shifts)
    lib.aosb_bloch_destroy(h)


def test_host_pattern_builder_rejects_non_hermitian_topology():
    b = bundles.tiny2d()
    # drop one off-diagonal block: its mirror loses its partner
    off_diag = int(np.flatnonzero(b.operators.row_atom != b.operators.col_atom)[0])
    rc, h, msg = _bloch_create(b, drop_block=off_diag)
    assert rc == 41 and b"not Hermitian" in msg


def _plan(ip, ix, n, tile=32, ordering=1, sv=None):
    opts = native.PlanOptions(native.ABI_VERSION, C.sizeof(native.PlanOptions), tile, ordering,
                              4 * tile, 1)
    h = C.c_void_p()
    buf = C.create_string_buffer(512)
    ip = np.ascontiguousarray(ip, np.int64)
    ix = np.ascontiguousarray(ix, np.int32)
    rc = native.library().aosb_plan_create(n, ip.ctypes.data, ix.ctypes.data,
                                           None if sv is None else sv.ctypes.data,
                                           0 if sv is None else sv.size - 1, C.byref(opts),
                                           C.byref(h), buf, 512)
    return rc, h, buf.value


@pytest.mark.parametrize("name,tile,ordering", [("tiny3d", 32, 1), ("tiny3d", 32, 0),
                                                ("small2d", 64, 1), ("c1", 128, 1),
                                                ("c1", 64, 0)])
def test_symbolic_plan_is_a_closed_fill_pattern(name, tile, ordering):
    b = getattr(bundles, name)()
    pat = bloch_ref.build_pattern(b)
    n = b.n_orbitals
    rc, h, msg = _plan(pat.indptr, pat.indices, n, tile, ordering,
                       np.ascontiguousarray(b.basis.atom_offsets, np.int64))
    assert rc == 0, msg
    lib = native.library()
    info = native.PlanInfo()
    lib.aosb_plan_info(h, C.byref(info))
    perm = np.empty(info.n_pad, np.int32)
    lib.aosb_plan_export_perm(h, perm.ctypes.data)
    assert sorted(perm[perm >= 0].tolist()) == list(range(n))
    assert info.n_pad % tile == 0 and info.n_tiles * tile == info.n_pad
    nb = info.n_tiles
    slot = np.empty(nb * nb, np.int32)
    lib.aosb_plan_export_slots(h, slot.ctypes.data)
    nz = slot.reshape(nb, nb) >= 0
    assert int(nz.sum()) == info.n_slots
    # A's tile pattern is covered
    pinv = np.empty(n, np.int64)
    pinv[perm[perm >= 0]] = np.flatnonzero(perm >= 0)
    rows = np.repeat(np.arange(n), np.diff(pat.indptr))
    assert nz[pinv[rows] // tile, pinv[pat.indices] // tile].all()
    # closed under elimination: L(i,k) and U(k,j) nonzero => (i,j) nonzero
    for k in range(nb):
        below = np.flatnonzero(nz[k + 1:, k]) + k + 1
        right = np.flatnonzero(nz[k, k + 1:]) + k + 1
        assert nz[np.ix_(below, right)].all()
    assert info.factor_flops >= info.factor_flops_alg > 0
    lib.aosb_plan_destroy(h)


@pytest.mark.parametrize("name,tile,ordering", [("c1", 32, 1), ("c1", 64, 0), ("small2d", 32, 0)])
def test_two_step_schur_lists_cover_both_steps(name, tile, ordering):
    """Super-step s = tile steps (k0, k1) = (2s, 2s + 1): the K = 256 items
    hold exactly step k0's Schur targets outside tile row/column k1 (those go
    to the K = 128 "inner" update) and all of step k1's targets, with the
    staged operand indices of the step lists; "cross" items are exactly the
    ones in tile rows/columns k0 + 2, k0 + 3."""
    b = getattr(bundles, name)()
    pat = bloch_ref.build_pattern(b)
    rc, h, msg = _plan(pat.indptr, pat.indices, b.n_orbitals, tile, ordering,
                       np.ascontiguousarray(b.basis.atom_offsets, np.int64))
    assert rc == 0, msg
    lib = native.library()
    info = native.PlanInfo()
    lib.aosb_plan_info(h, C.byref(info))
    nb = info.n_tiles
    slot = np.empty(nb * nb, np.int32)
    lib.aosb_plan_export_slots(h, slot.ctypes.data)
    slot = slot.reshape(nb, nb)
    ns, nc, nr = C.c_int64(), C.c_int64(), C.c_int64()
    lib.aosb_plan_export_super_steps(h, C.byref(ns), C.byref(nc), C.byref(nr), None, None, None,
                                     None)
    assert ns.value == nb // 2
    coff = np.empty(ns.value + 1, np.int64)
    roff = np.empty(ns.value + 1, np.int64)
    cross = np.empty(5 * max(nc.value, 1), np.int32)
    rest = np.empty(5 * max(nr.value, 1), np.int32)
    lib.aosb_plan_export_super_steps(h, None, None, None, coff.ctypes.data, roff.ctypes.data,
                                     cross.ctypes.data, rest.ctypes.data)
    cross, rest = cross[:5 * nc.value].reshape(-1, 5), rest[:5 * nr.value].reshape(-1, 5)
    where = {int(slot[i, j]): (i, j) for i in range(nb) for j in range(nb) if slot[i, j] >= 0}
    nonempty = 0
    for s in range(ns.value):
        k0, k1 = 2 * s, 2 * s + 1
        L0 = [i for i in range(k0 + 1, nb) if slot[i, k0] >= 0]
        U0 = [j for j in range(k0 + 1, nb) if slot[k0, j] >= 0]
        L1 = [i for i in range(k1 + 1, nb) if slot[i, k1] >= 0]
        U1 = [j for j in range(k1 + 1, nb) if slot[k1, j] >= 0]
        want = {}
        for a, i in enumerate(L0):
            for bb, j in enumerate(U0):
                if i != k1 and j != k1:
                    want.setdefault((i, j), [-1, -1, -1, -1])[0:2] = [a, len(L0) + bb]
        for a, i in enumerate(L1):
            for bb, j in enumerate(U1):
                want.setdefault((i, j), [-1, -1, -1, -1])[2:4] = [a, len(L1) + bb]
        got = {}
        for part, items in (("cross", cross[coff[s]:coff[s + 1]]), ("rest", rest[roff[s]:roff[s + 1]])):
            for it in items:
                i, j = where[int(it[0])]
                assert (i, j) not in got
                in_cross = i in (k0 + 2, k0 + 3) or j in (k0 + 2, k0 + 3)
                assert in_cross == (part == "cross"), (s, i, j, part)
                got[(i, j)] = [int(v) for v in it[1:]]
        assert got == want, s
        nonempty += len(got) > 0
    assert nonempty > 0
    lib.aosb_plan_destroy(h)


@pytest.mark.parametrize("name,tile,ordering", [("c1", 32, 1), ("c1", 64, 0), ("small2d", 32, 0),
                                                ("c1", 128, 0)])
def test_pair_lists_hold_the_two_step_items_in_column_pairs(name, tile, ordering):
    """The two-CTA pair lists: every two-step item appears exactly once, as
    the even or odd member of a pair; the two members of a pair share their
    tile column, the B index and which halves are present; a single has odd
    slot -1 and repeats the even member's A indices; pairs are ordered by
    (first row, column)."""
    b = getattr(bundles, name)()
    pat = bloch_ref.build_pattern(b)
    rc, h, msg = _plan(pat.indptr, pat.indices, b.n_orbitals, tile, ordering,
                       np.ascontiguousarray(b.basis.atom_offsets, np.int64))
    assert rc == 0, msg
    lib = native.library()
    info = native.PlanInfo()
    lib.aosb_plan_info(h, C.byref(info))
    nb = info.n_tiles
    slot = np.empty(nb * nb, np.int32)
    lib.aosb_plan_export_slots(h, slot.ctypes.data)
    where = {int(v): divmod(q, nb) for q, v in enumerate(slot) if v >= 0}
    ns, nc, nr = C.c_int64(), C.c_int64(), C.c_int64()
    lib.aosb_plan_export_super_steps(h, C.byref(ns), C.byref(nc), C.byref(nr), None, None, None,
                                     None)
    coff = np.empty(ns.value + 1, np.int64)
    roff = np.empty(ns.value + 1, np.int64)
    cross = np.empty(5 * max(nc.value, 1), np.int32)
    rest = np.empty(5 * max(nr.value, 1), np.int32)
    lib.aosb_plan_export_super_steps(h, None, None, None, coff.ctypes.data, roff.ctypes.data,
                                     cross.ctypes.data, rest.ctypes.data)
    pc, pr = C.c_int64(), C.c_int64()
    lib.aosb_plan_export_pair_steps(h, C.byref(pc), C.byref(pr), None, None, None, None)
    pcoff = np.empty(ns.value + 1, np.int64)
    proff = np.empty(ns.value + 1, np.int64)
    pcross = np.empty(8 * max(pc.value, 1), np.int32)
    prest = np.empty(8 * max(pr.value, 1), np.int32)
    lib.aosb_plan_export_pair_steps(h, None, None, pcoff.ctypes.data, proff.ctypes.data,
                                    pcross.ctypes.data, prest.ctypes.data)
    pairs_total = singles = 0
    for items, off, pitems, poff in ((cross, coff, pcross, pcoff), (rest, roff, prest, proff)):
        for s in range(ns.value):
            want = {int(it[0]): tuple(int(v) for v in it[1:])
                    for it in items[5 * off[s]:5 * off[s + 1]].reshape(-1, 5)}
            got = {}
            prev = None
            for p in pitems[8 * poff[s]:8 * poff[s + 1]].reshape(-1, 8):
                e, o, a0e, a0o, b0, a1e, a1o, b1 = (int(v) for v in p)
                got[e] = (a0e, b0, a1e, b1)
                ie, je = where[e]
                if o >= 0:
                    io, jo = where[o]
                    assert jo == je and io > ie
                    got[o] = (a0o, b0, a1o, b1)
                    assert (a0o >= 0) == (a0e >= 0) and (a1o >= 0) == (a1e >= 0)
                else:
                    singles += 1
                    assert (a0o, a1o) == (a0e, a1e)
                key = (ie, je)
                assert prev is None or key > prev
                prev = key
                pairs_total += 1
            assert got == want, s
    assert pairs_total > 0
    # most items pair up
    assert singles < 0.5 * pairs_total
    lib.aosb_plan_destroy(h)


def test_symbolic_plan_rejects_bad_patterns():
    ip = np.array([0, 2, 3], np.int64)
    assert _plan(ip, np.array([0, 1, 0], np.int32), 2)[0] == 33      # row 1 misses its diagonal
    assert _plan(ip, np.array([1, 0, 1], np.int32), 2)[0] == 32      # unsorted columns
    assert _plan(ip, np.array([0, 5, 1], np.int32), 2)[0] == 31      # column out of range
    assert _plan(np.array([0, 1, 2], np.int64), np.array([0, 1], np.int32), 2, tile=48)[0] == 53
    bad = native.PlanOptions(99, C.sizeof(native.PlanOptions), 32, 1, 128, 1)
    h = C.c_void_p()
    rc = native.library().aosb_plan_create(2, np.array([0, 1, 2], np.int64).ctypes.data,
                                           np.array([0, 1], np.int32).ctypes.data, None, 0,
                                           C.byref(bad), C.byref(h), None, 0)
    assert rc == 10


def _ubatch(n=3, batch=1, rhs=1, values=None, indptr=None, indices=None, abi=None):
    indptr = np.array([0, 1, 2, 3], np.int32) if indptr is None else indptr
    indices = np.array([0, 1, 2], np.int32) if indices is None else indices
    nnz = int(indices.size)
    values = np.ones(batch * nnz, np.complex64) if values is None else values
    r = np.ones(batch * n * rhs, np.complex64)
    sol = np.zeros_like(r)
    req = native.UbatchRequest(abi or native.ABI_VERSION, C.sizeof(native.UbatchRequest), n, nnz,
                               batch, rhs, indptr.ctypes.data, indices.ctypes.data,
                               values.ctypes.data, r.ctypes.data, sol.ctypes.data)
    res = native.UbatchResult()
    rc = native.library().aospectrum_b200_solve_complex64_ubatch_v1(C.byref(req), C.byref(res))
    return rc, res


def test_ubatch_request_validation_codes():
    """The reference's validation codes (native/src/aospectrum_cudss_complex64_
    ubatch.c:136-241), all raised before any device call."""
    assert _ubatch(abi=7)[1].status == 10
    assert _ubatch(batch=65)[1].status == 12
    assert _ubatch(rhs=257)[1].status == 12
    assert _ubatch(indptr=np.array([0, 1, 2, 2], np.int32))[1].status == 14
    assert _ubatch(indices=np.array([0, 1, 1], np.int32),
                   indptr=np.array([0, 1, 2, 3], np.int32))[1].status == 33
    vals = np.ones(3, np.complex64)
    vals[1] = np.inf
    rc, res = _ubatch(values=vals)
    assert rc != 0 and res.status == 35 and b"non-finite" in res.error_message


def test_gram_rejects_row_counts_beyond_the_launch_grid():
    """Both Gram entry points split n into 512-row chunks on the grid's z
    axis (at most 65535): a larger n is rejected with status 34 before any
    launch, so no pointer is touched (these are never dereferenced)."""
    lib = native.library()
    fake = 1 << 20
    n = 65536 * 512   # one chunk too many; p = q = 1 fits the no-alloc scratch
    buf = C.create_string_buffer(512)
    rc = lib.aosb_gram(n, 1, 1, fake, 1, fake, 1, fake, fake, None, buf, 512)
    assert rc == 34 and b"65535" in buf.value
    buf = C.create_string_buffer(512)
    rc = lib.aosb_gram_noalloc(n, 1, 1, fake, 1, fake, 1, fake, None, buf, 512)
    assert rc == 34 and b"65535" in buf.value


def test_shift_session_argument_checks():
    from aospectrum_b200.solvers import B200ShiftSession

    with pytest.raises(ValueError):
        B200ShiftSession([0, 1], [0], 2)
    with pytest.raises(ValueError):
        B200ShiftSession([0, 1, 2], [0, 1], 2, "float32")
    s = B200ShiftSession([0, 1, 2], [0, 1], 2)
    with pytest.raises(ValueError, match="1 through 64"):
        s.solve(np.ones(2), np.ones(2), np.zeros(65), np.ones((2, 1)))
    with pytest.raises(ValueError, match="RHS"):
        s.solve(np.ones(2), np.ones(2), np.zeros(1), np.ones((3, 1)))
    s.close()
    with pytest.raises(RuntimeError, match="closed"):
        s.solve(np.ones(2), np.ones(2), np.zeros(1), np.ones((2, 1)))


def test_process_wide_tuning_setters_round_trip():
    """The lookahead-SM and solve-CTA setters only swap a process-wide value
    (no device work): each returns the previous value and rejects bad ones."""
    from aospectrum_b200 import native

    lib = native.library()
    prev = lib.aosb_factor_set_lookahead_sms(24)
    assert lib.aosb_factor_set_lookahead_sms(0) == 24
    assert lib.aosb_factor_set_lookahead_sms(-1) == -1
    lib.aosb_factor_set_lookahead_sms(prev)
    prev = lib.aosb_solve_set_ctas_per_sm(1)
    assert lib.aosb_solve_set_ctas_per_sm(0) == 1
    assert lib.aosb_solve_set_ctas_per_sm(3) == -1
    assert lib.aosb_solve_set_ctas_per_sm(prev) == 2   # 0 restored the default, 2
    prev = lib.aosb_solve_set_lookahead(1)
    assert lib.aosb_solve_set_lookahead(prev) == 1
    assert lib.aosb_solve_set_lookahead(-1) == -1
    prev = lib.aosb_factor_set_schur_pairs(1)
    assert lib.aosb_factor_set_schur_pairs(prev) == 1
    assert lib.aosb_factor_set_schur_pairs(2) == -1
    prev = lib.aosb_tc_set_wait_limit(7)
    assert prev == 1 << 22
    assert lib.aosb_tc_set_wait_limit(0) == 7
    assert lib.aosb_tc_set_wait_limit(-3) == -1
    assert lib.aosb_tc_set_wait_limit(prev) == 1 << 22


@pytest.mark.parametrize("max_rows", [4, 13, 16])
def test_row_blocks_share_columns_and_respect_the_cap(max_rows):
    """engine.row_blocks: every block holds consecutive rows with one column
    set, at most max_rows of them, and the blocks tile 0..n."""
    from aospectrum_b200.engine import row_blocks

    b = bundles.small2d()
    pat = bloch_ref.build_pattern(b)
    indptr, indices = pat.indptr, pat.indices
    starts = np.asarray(b.basis.atom_offsets)[:-1]
    for st in (starts, None):
        rb = row_blocks(indptr, indices, max_rows=max_rows, starts=st)
        assert rb[0] == 0 and rb[-1] == indptr.size - 1
        assert np.all(np.diff(rb) >= 1) and np.all(np.diff(rb) <= max_rows)
        for a, z in zip(rb[:-1], rb[1:]):
            first = indices[indptr[a]:indptr[a + 1]]
            for r in range(a + 1, z):
                assert np.array_equal(indices[indptr[r]:indptr[r + 1]], first)


def _emulate_bloch_windows(tables, values, ph, nnz):
    """numpy restatement of bloch_windows_kernel's index mapping and float32
    arithmetic (products without contraction, members added in block order,
    the upper window's mean, its conjugate in the lower window)."""
    info, dst, mem, moff, msh = tables
    f32 = np.float32
    zero, half = f32(0.0), f32(0.5)
    out_r = np.zeros(nnz, f32)
    out_i = np.zeros(nnz, f32)

    def sums(rng, elem):
        sr = si = None
        for m in range(rng[0], rng[1]):
            v = values[moff[m] + elem].astype(f32)
            pr, pi = f32(ph[msh[m]].real), f32(ph[msh[m]].imag)
            re, im = v * pr - zero * pi, v * pi + zero * pr
            sr, si = (re, im) if sr is None else (sr + re, si + im)
        return sr, si

    for g in range(info.shape[0]):
        nr, nc, rl, gm = (int(x) for x in info[g])
        a = np.repeat(np.arange(nr), nc)
        c = np.tile(np.arange(nc), nr)
        pos = dst[g] + a * rl + c
        if gm == g:
            lo, hi = np.minimum(a, c), np.maximum(a, c)
            xr, xi = sums(mem[g], lo * nc + hi)
            yr, yi = sums(mem[g], hi * nc + lo)
            mr_, mi_ = (xr + yr) * half, (xi - yi) * half
            vr = np.where(a == c, xr, mr_)
            vi = np.where(a == c, zero, np.where(a < c, mi_, -mi_))
        else:
            eg, em = a * nc + c, c * nr + a
            lower = gm < g
            xr, xi = sums(mem[gm] if lower else mem[g], em if lower else eg)
            yr, yi = sums(mem[g] if lower else mem[gm], eg if lower else em)
            vr, vi = (xr + yr) * half, (xi - yi) * half
            if lower:
                vi = -vi
        out_r[pos] = vr
        out_i[pos] = vi
    out = np.empty(nnz, np.complex64)
    out.real, out.imag = out_r, out_i
    return out


@pytest.mark.parametrize("name", ["small2d", "c1"])
def test_bloch_window_kernel_emulation_matches_reference(name, golden):
    """The device Bloch kernel's algorithm, replayed on the host from the
    tables the library builds (aosb_bloch_export_groups), reproduces the
    reference's H(k), S(k) bit for bit."""
    b = getattr(bundles, name)()
    rc, h, _ = _bloch_create(b)
    assert rc == 0
    lib = native.library()
    try:
        ng, nm = C.c_int64(), C.c_int64()
        lib.aosb_bloch_export_groups(h, C.byref(ng), C.byref(nm), None, None, None, None, None)
        info = np.empty((ng.value, 4), np.int32)
        dst = np.empty(ng.value, np.int64)
        mem = np.empty((ng.value, 2), np.int32)
        moff = np.empty(nm.value, np.int64)
        msh = np.empty(nm.value, np.int32)
        lib.aosb_bloch_export_groups(h, C.byref(ng), C.byref(nm), info.ctypes.data,
                                     dst.ctypes.data, mem.ctypes.data, moff.ctypes.data,
                                     msh.ctypes.data)
        pat = bloch_ref.build_pattern(b)
        for k in bundles.KPOINTS[:2]:
            ph = bloch_ref.phases(pat.shifts, k)
            ref_h, ref_s = bloch_ref.bloch_pair(pat, b, k)
            for vals, ref in ((b.operators.h_values, ref_h), (b.operators.s_values, ref_s)):
                got = _emulate_bloch_windows((info, dst, mem, moff, msh), np.asarray(vals), ph,
                                             ref.size)
                assert np.array_equal(got, ref)
    finally:
        lib.aosb_bloch_destroy(h)


def _emulate_row_block_residual(rb, indptr, indices, h, s, pk, z, b, x, ncols, np_,
                                warps=4):
    """numpy restatement of row_block_kernel<R, residual>'s work split: CTA
    index = (block, 32-column strip) * np + pencil; per CTA the block's
    nonzeros are split between `warps` warps and their partial sums added."""
    n = indptr.size - 1
    r = np.full((np_, n, ncols), np.nan, np.complex128)
    ncs = (ncols + 31) // 32
    for cta in range((rb.size - 1) * ncs * np_):
        p = cta % np_
        bs = cta // np_
        blk, strip = bs // ncs, bs % ncs
        cols = np.arange(strip * 32, min(ncols, strip * 32 + 32))
        r0, nr = rb[blk], rb[blk + 1] - rb[blk]
        base0 = indptr[r0]
        ln = indptr[r0 + 1] - base0
        per = (ln + warps - 1) // warps
        a = (h[pk[p]].astype(np.complex128) - z[p] * s[pk[p]].astype(np.complex128))
        acc = np.zeros((nr, cols.size), np.complex128)
        for w in range(warps):
            w0, w1 = w * per, min(w * per + per, ln)
            for q in range(nr):
                seg = slice(base0 + q * ln + w0, base0 + q * ln + w1)
                acc[q] += a[seg] @ x[p][indices[base0 + w0:base0 + w1]][:, cols]
        r[p, r0:r0 + nr][:, cols] = b[p, r0:r0 + nr][:, cols] - acc
    return r


def test_row_block_residual_work_split_emulation():
    """The row-block residual's CTA decode (pencil fastest), column strips and
    warp split cover every (pencil, row, column) once and give b - (H - zS) x."""
    from aospectrum_b200.engine import row_blocks
    import scipy.sparse as sp

    b_ = bundles.small2d()
    pat = bloch_ref.build_pattern(b_)
    k = bundles.KPOINTS[1]
    hv, sv = bloch_ref.bloch_pair(pat, b_, k)
    n = pat.indptr.size - 1
    rb = row_blocks(pat.indptr, pat.indices, max_rows=13,
                    starts=np.asarray(b_.basis.atom_offsets)[:-1])
    rng = np.random.default_rng(3)
    np_, ncols = 3, 40
    x = rng.standard_normal((np_, n, ncols)) + 1j * rng.standard_normal((np_, n, ncols))
    bb = rng.standard_normal((np_, n, ncols)) + 1j * rng.standard_normal((np_, n, ncols))
    z = np.asarray([-2.0 + 0.1j, 0.5 + 0.01j, -1.0 + 1.0j])
    pk = np.zeros(np_, np.int64)
    got = _emulate_row_block_residual(rb, pat.indptr, pat.indices, hv[None], sv[None], pk, z,
                                      bb, x, ncols, np_)
    assert not np.isnan(got).any()
    for p in range(np_):
        a = sp.csr_matrix((hv.astype(np.complex128) - z[p] * sv.astype(np.complex128),
                           pat.indices, pat.indptr), shape=(n, n))
        ref = bb[p] - a @ x[p]
        assert np.max(np.abs(got[p] - ref)) <= 1e-12 * np.max(np.abs(ref))
