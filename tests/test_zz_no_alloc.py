"""The allocation-free Gram entry point, lgh_gram_noalloc, on the GPU.

Some callers cannot let this library allocate device memory: applications
that hand the library a fixed slice of the device up front (a memory pool,
or one partition per tenant) and forbid it to take more, where a cudaMalloc
inside the library would fail or break the budget.  For them
lgh_gram_noalloc computes X^T X with its split-K partial sums in a fixed
file-scope device array instead of an allocation.  It is not for code
inside a CUDA stream capture: the call synchronises the legacy default
stream, which no capture allows.  It must give the same result as the
library's regular Gram path (lgh_test_gram) within the tolerance of the
other Gram tests, on two calls in a row that reuse that array, make no
allocation through the library's allocator, and reject a width beyond the
array's limit with a clear error.  This file is named to run after every
other test file.
"""

import ctypes

import numpy as np
import pytest

import lgh_b200 as L

pytestmark = pytest.mark.gpu


def _fn():
    f = L.load().lgh_gram_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64]
    return f


def _noalloc_gram(X):
    n, w = X.shape
    dx = L.Vec(data=np.ascontiguousarray(X).reshape(-1))
    dg = L.Vec(w * w)
    rc = _fn()(n, w, dx.ptr(), w, dg.ptr(), w)
    assert rc == 0, L.load().lgh_last_error()
    return dg.get().reshape(w, w).T


def test_noalloc_gram_matches_regular_path(cuda_device):
    rng = np.random.default_rng(21)
    X1 = rng.standard_normal((70000, 220))
    X2 = rng.standard_normal((3001, 7))
    # two calls in a row on the shared scratch, different shapes
    G1 = _noalloc_gram(X1)
    dx = L.Vec(data=np.ascontiguousarray(X2).reshape(-1))
    dg = L.Vec(7 * 7)
    before = L.runtime_counters()["allocs"]
    assert _fn()(3001, 7, dx.ptr(), 7, dg.ptr(), 7) == 0
    assert L.runtime_counters()["allocs"] == before   # a warm call allocates nothing
    G2 = dg.get().reshape(7, 7).T
    for X, G in ((X1, G1), (X2, G2)):
        ref = L.test_gram(X)
        assert np.max(np.abs(G - ref)) <= 1e-12 * np.max(np.abs(ref))
    # the array keeps the previous call's partials; a repeat is identical
    G1b = _noalloc_gram(X1)
    assert np.array_equal(G1, G1b)


def test_noalloc_gram_rejects_oversize(cuda_device):
    dx = L.Vec(16)
    dg = L.Vec(16)
    rc = _fn()(4, 1100, dx.ptr(), 1100, dg.ptr(), 1100)
    assert rc == 63
    assert b"1024" in L.load().lgh_last_error()
