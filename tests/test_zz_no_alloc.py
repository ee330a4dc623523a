"""The allocation-free Gram entry point, lgh_gram_noalloc, on the GPU.

Some callers cannot allocate device memory: code that runs inside a CUDA
stream capture (where cudaMalloc is not allowed) and applications that hand
the library a fixed slice of the device and forbid it to take more.  For
them lgh_gram_noalloc computes X^T X with its split-K partial sums in a
fixed file-scope device array instead of an allocation.  It must give the
same result as the library's regular Gram path (lgh_test_gram) within the
tolerance of the other Gram tests, on two calls in a row that reuse that
array, and reject a width beyond the array's limit with a clear error.
This file is named to run after every other test file.
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
    G2 = _noalloc_gram(X2)
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
