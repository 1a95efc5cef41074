"""Bundle ingest to the device (the reference's load_bundle + pattern
build, src/aospectrum/bundle.py:41-114, src/aospectrum/sparse.py:64-140):
a bundle written to disk and opened memory-mapped gives, through the C++
pattern build and the device upload, the same CSR pattern and the same
H(k), S(k) as the in-memory bundle; BandEngine.load_values replaces the
resident block values from pinned host memory."""

from __future__ import annotations

import numpy as np
import pytest

import bundles
from oracle import bloch_ref

pytestmark = pytest.mark.gpu


def test_memmapped_bundle_to_device_matches_in_memory(tmp_path):
    import torch

    from aospectrum_b200.bundle import load_bundle, write_bundle
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.engine import BandEngine, BlochDevice

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    b = bundles.small2d()
    write_bundle(b, tmp_path / "b")
    loaded = load_bundle(tmp_path / "b")
    assert isinstance(np.asarray(loaded.operators.h_values), np.memmap) or \
        getattr(loaded.operators.h_values, "base", None) is not None
    mem, disk = BlochDevice(b, dev), BlochDevice(loaded, dev)
    try:
        pat = bloch_ref.build_pattern(b)
        assert np.array_equal(disk.indptr, pat.indptr) and np.array_equal(disk.indices, pat.indices)
        k = np.asarray([bundles.KPOINTS[1]])
        hm, sm = mem.apply(k)
        hd, sd = disk.apply(k)
        assert torch.equal(hm, hd) and torch.equal(sm, sd)
    finally:
        mem.close()
        disk.close()
    # values replaced from pinned host memory: H scaled by 2 doubles H(k)
    eng = BandEngine(loaded, CissSettings(block_size=8), EngineSettings(precision="plain"))
    try:
        h0 = eng.bloch.apply(k)[0].clone()
        hv = torch.from_numpy(2.0 * np.asarray(loaded.operators.h_values, np.float32)).pin_memory()
        sv = torch.from_numpy(np.asarray(loaded.operators.s_values, np.float32).copy()).pin_memory()
        eng.load_values(hv, sv)
        torch.cuda.synchronize()
        h1 = eng.bloch.apply(k)[0]
        assert torch.allclose(h1, 2 * h0, rtol=0, atol=0)
    finally:
        eng.close()
