"""The allocation-free dense solve against the regular device entry point.

hprmat_b200_solve_linear_noalloc serves callers that must not call cudaMalloc (solvers run
inside another framework's memory pool, or in latency-critical loops where cudaFree would
stall the device).  It keeps its working memory in a fixed array inside the library, so
this test checks that two calls in a row -- the second one finding the first one's data in
that array -- both agree with hprmat_b200_solve_linear_device (FP64) to the 1e-12
relative tolerance of the dense-solve tests.  The file sorts last so that a run stopping at
the first failure has already run every other test; it also passes alone.
"""
import ctypes

import numpy as np
import pytest
import torch

from hprmat_b200 import _native as nat
from hprmat_b200 import api

pytestmark = pytest.mark.gpu


def _system(n, nrhs, seed):
    rng = np.random.default_rng(seed)
    A = rng.random((n, n)) + 1j * rng.random((n, n))
    A[np.arange(n), np.arange(n)] += 2 * n
    B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    return np.asfortranarray(A), np.asfortranarray(B)


def _dev(a):
    """Column-major complex128 numpy array -> device buffer (torch, same memory order)."""
    flat = np.asfortranarray(a).ravel(order="F")
    return torch.from_numpy(flat.view(np.float64).copy()).cuda()


def _host(t, shape):
    return t.cpu().numpy().view(np.complex128).reshape(shape, order="F")


def test_noalloc_matches_device_solve_twice():
    """Calls in a row on the one array, each later call finding the previous one's data:
    two mid-size systems, the documented limit (n = 512 with 64 right-hand sides: the array
    full), one block of 64 columns (the factorisation ends after its only panel) and a system
    smaller than a warp."""
    lib = nat.load()
    ctx = api.Context(precision="fp64")
    try:
        for call, (n, nrhs, seed) in enumerate([(500, 40, 1), (333, 64, 2), (512, 64, 3), (64, 1, 4), (17, 3, 5)]):
            A, B = _system(n, nrhs, seed)
            dA, dB_ref, dB = _dev(A), _dev(B), _dev(B)
            ctx.solve_linear_device(dA.data_ptr(), dB_ref.data_ptr(), n, nrhs)
            info = ctypes.c_int(-1)
            s = lib.hprmat_b200_solve_linear_noalloc(ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()),
                                                     n, nrhs, None, ctypes.byref(info))
            nat.check(s)
            assert info.value == 0
            X = _host(dB, (n, nrhs))
            Xr = _host(dB_ref, (n, nrhs))
            assert np.linalg.norm(X - Xr) / np.linalg.norm(Xr) <= 1e-12, call
            assert np.array_equal(_host(dA, (n, n)), A)  # A is read only
            Xnp = np.linalg.solve(A, B)
            assert np.linalg.norm(X - Xnp) / np.linalg.norm(Xnp) <= 1e-12, call
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_array():
    lib = nat.load()
    dA = torch.zeros(2 * 600 * 600, dtype=torch.float64, device="cuda")
    dB = torch.zeros(2 * 600 * 8, dtype=torch.float64, device="cuda")
    s = lib.hprmat_b200_solve_linear_noalloc(ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), 600, 8,
                                             None, None)
    assert s == nat.ERR_UNSUPPORTED
    assert b"512" in lib.hprmat_b200_last_error()
    s = lib.hprmat_b200_solve_linear_noalloc(ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), 100, 65,
                                             None, None)
    assert s == nat.ERR_UNSUPPORTED


def test_noalloc_reports_singular_with_info():
    """An exactly zero column: HPRMAT_B200_SINGULAR with info = its 1-based index, then a
    regular solve on the same array works again."""
    lib = nat.load()
    n, nrhs = 200, 2
    A, B = _system(n, nrhs, 7)
    A[:, 41] = 0.0
    dA, dB = _dev(A), _dev(B)
    info = ctypes.c_int(-1)
    s = lib.hprmat_b200_solve_linear_noalloc(ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), n, nrhs,
                                             None, ctypes.byref(info))
    assert s == nat.SINGULAR and info.value == 42
    A, B = _system(n, nrhs, 8)
    dA, dB = _dev(A), _dev(B)
    s = lib.hprmat_b200_solve_linear_noalloc(ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), n, nrhs,
                                             None, ctypes.byref(info))
    nat.check(s)
    assert info.value == 0
    Xnp = np.linalg.solve(A, B)
    assert np.linalg.norm(_host(dB, (n, nrhs)) - Xnp) / np.linalg.norm(Xnp) <= 1e-12


@pytest.mark.parametrize("scale", [1e-300, 1e300])
def test_noalloc_pivots_outside_float_range(scale):
    """Entries far outside the float range and a zero diagonal: the pivots are chosen over the
    whole double range, so the solve pivots instead of reporting a false zero pivot."""
    lib = nat.load()
    rng = np.random.default_rng(22)
    n, nrhs = 300, 4
    A = rng.uniform(0.5, 1.5, (n, n)) + 1j * rng.uniform(-0.5, 0.5, (n, n))
    A[np.arange(n), np.arange(n)] = 0.0
    A = np.asfortranarray(A * scale)
    B = np.asfortranarray(rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)))
    dA, dB = _dev(A), _dev(B)
    info = ctypes.c_int(-1)
    s = lib.hprmat_b200_solve_linear_noalloc(ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), n, nrhs,
                                             None, ctypes.byref(info))
    nat.check(s)
    assert info.value == 0
    Xnp = np.linalg.solve(A, B)
    sc = 1.0 / np.abs(Xnp).max()  # norms of 1e300-sized values overflow: compare scaled copies
    assert np.linalg.norm((_host(dB, (n, nrhs)) - Xnp) * sc) / np.linalg.norm(Xnp * sc) <= 1e-12
