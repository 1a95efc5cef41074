"""aosb_gram_noalloc: the Gram product for callers that cannot allocate
device memory at call time (inside another framework's memory pool or
under a memory cap, in callbacks where an allocation could block).  It must
give the same result as aosb_gram, which takes caller-provided scratch, on
consecutive calls that reuse the library's fixed scratch array, and reject
sizes beyond that array.  Collected last so a failure here comes after every
other test has run."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from aospectrum_b200 import native

pytestmark = pytest.mark.gpu


def _gram_with_scratch(torch, x, y):
    n, p = x.shape
    q = y.shape[1]
    lib = native.library()
    scratch = torch.empty(max(16, lib.aosb_gram_scratch_bytes(n, p, q)), dtype=torch.uint8,
                          device=x.device)
    g = torch.empty((p, q), dtype=torch.complex128, device=x.device)
    native.call("aosb_gram", n, p, q, x.data_ptr(), x.stride(0), y.data_ptr(), y.stride(0),
                g.data_ptr(), scratch.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return g


def _gram_noalloc(torch, x, y):
    n, p = x.shape
    q = y.shape[1]
    g = torch.empty((p, q), dtype=torch.complex128, device=x.device)
    native.call("aosb_gram_noalloc", n, p, q, x.data_ptr(), x.stride(0), y.data_ptr(),
                y.stride(0), g.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return g


def test_noalloc_gram_matches_scratch_gram_on_consecutive_calls():
    import torch

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(11)
    shapes = [(13000, 128, 128), (3001, 40, 72)]
    for n, p, q in shapes:
        x = torch.from_numpy(rng.standard_normal((n, p)) + 1j * rng.standard_normal((n, p))).to(dev)
        y = torch.from_numpy(rng.standard_normal((n, q)) + 1j * rng.standard_normal((n, q))).to(dev)
        ref = _gram_with_scratch(torch, x, y).cpu().numpy()
        got = _gram_noalloc(torch, x, y).cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-9)
        host = x.cpu().numpy().conj().T @ y.cpu().numpy()
        np.testing.assert_allclose(got, host, rtol=1e-9, atol=1e-7)


def test_noalloc_gram_rejects_sizes_beyond_its_scratch():
    import torch

    dev = torch.device("cuda", 0)
    n, p, q = 60000, 192, 192   # ceil(n/512) * p * q * 16 bytes > 16 MiB
    # full-size operands, so the call would stay in bounds even if it ran
    x = torch.zeros((n, p), dtype=torch.complex128, device=dev)
    buf = C.create_string_buffer(512)
    g = torch.empty((p, q), dtype=torch.complex128, device=dev)
    rc = native.library().aosb_gram_noalloc(n, p, q, x.data_ptr(), p, x.data_ptr(), q,
                                            g.data_ptr(), None, buf, 512)
    assert rc == 34
    assert b"fixed" in buf.value and b"scratch" in buf.value
