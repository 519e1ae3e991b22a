"""The allocation-free solve (mh_solve_mixed_noalloc) through the C ABI (GPU).

Callers that cannot allocate device memory (an application whose pool owns
the device, a fixed-footprint real-time loop) hand the library device buffers
they already own; the entry point keeps its scratch in one static device
array.  This file is collected last so that, if it fails, a run that stops at
the first failure has already run every other test; it also passes when run
alone in a fresh process.

Checked against the existing FP64 entry point mh_solve (cuSOLVER LU) with
S = I, i.e. X = D^-1 B, within 1e-9 (the tolerance of the other mixed-path
tests), on two calls in a row with different matrices and right-hand sides,
so the second call cannot reuse anything the first left in the shared array.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device(a, torch):
    """Column-major complex128 numpy array -> device tensor with the same
    memory layout (the transpose of a C-contiguous tensor)."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.complex128).T)).cuda()


def _noalloc(mh, torch, D, B, tol=1e-12, max_iter=30):
    n, nrhs = B.shape
    dA, dB = _device(D, torch), _device(B, torch)
    dX = torch.empty((nrhs, n), dtype=torch.complex128, device="cuda")
    iters = ctypes.c_int32(0)
    res = ctypes.c_double(0.0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = mh.native.lib().mh_solve_mixed_noalloc(
        n, ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), nrhs,
        ctypes.c_void_p(dX.data_ptr()), tol, max_iter, ctypes.c_void_p(stream),
        ctypes.byref(iters), ctypes.byref(res))
    return rc, dX.cpu().numpy().T, iters.value, res.value


def test_noalloc_matches_fp64_solve_twice(mh, gpu):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(11)
    cases = [(mh.mesh_hemisphere(1.0, (0, 0, 0), (16, 32)), 0.6, 3),
             (mh.mesh_hemisphere(1.0, (0, 0, 0), (24, 36)) + mh.mesh_hemisphere(1.0, (4, 0, 0), (8, 12)),
              1.4, 2)]
    for mesh, k, nrhs in cases:
        _, D = mh.assemble_matrices(mh.DEFAULT_GREEN_FUNCTIONS, mesh, k, ctx=gpu)
        n = mesh.nfaces
        B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
        ref = mh.solve(D, np.eye(n, dtype=np.complex128), B, ctx=gpu)
        rc, X, iters, res = _noalloc(mh, torch, D, B)
        assert rc == 0, mh.native.lib().mh_last_error(None)
        assert 1 <= iters <= 10 and res <= 1e-12
        err = np.max(np.abs(X - ref)) / np.max(np.abs(ref))
        assert err < 1e-9, err


def test_noalloc_rejects_sizes_beyond_its_maximum(mh, gpu):
    torch = pytest.importorskip("torch")
    L = mh.native.lib()
    n = 1025  # MH_NOALLOC_MAX_N + 1
    dA = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    dB = torch.zeros((1, n), dtype=torch.complex128, device="cuda")
    dX = torch.zeros((1, n), dtype=torch.complex128, device="cuda")
    rc = L.mh_solve_mixed_noalloc(n, ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()),
                                  1, ctypes.c_void_p(dX.data_ptr()), 1e-10, 10, None, None, None)
    assert rc == mh.native.MH_ERR_ARG
    assert b"1024" in L.mh_last_error(None)


def test_noalloc_at_its_maximum_allocates_nothing(mh, gpu):
    """n = 1024 and nrhs = 16 (every scratch region full), against mh_solve;
    the device's free memory is the same before and after a second call (the
    first call loads the module and looks up the scratch address)."""
    torch = pytest.importorskip("torch")
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (32, 64))
    assert mesh.nfaces == 1024
    _, D = mh.assemble_matrices(mh.DEFAULT_GREEN_FUNCTIONS, mesh, 0.9, ctx=gpu)
    rng = np.random.default_rng(5)
    B = rng.standard_normal((1024, 16)) + 1j * rng.standard_normal((1024, 16))
    ref = mh.solve(D, np.eye(1024, dtype=np.complex128), B, ctx=gpu)
    dA, dB = _device(D, torch), _device(B, torch)
    dX = torch.empty((16, 1024), dtype=torch.complex128, device="cuda")
    L = mh.native.lib()
    stream = torch.cuda.current_stream().cuda_stream
    iters = ctypes.c_int32(0)
    res = ctypes.c_double(0.0)

    def call():
        return L.mh_solve_mixed_noalloc(1024, ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), 16,
                                        ctypes.c_void_p(dX.data_ptr()), 1e-12, 30, ctypes.c_void_p(stream),
                                        ctypes.byref(iters), ctypes.byref(res))

    assert call() == 0, L.mh_last_error(None)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert call() == 0, L.mh_last_error(None)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    X = dX.cpu().numpy().T
    assert np.max(np.abs(X - ref)) / np.max(np.abs(ref)) < 1e-9
    assert res.value <= 1e-12


def test_noalloc_reports_no_convergence(mh, gpu):
    """One sweep cannot reach tol = 1e-30: MH_ERR_NOT_CONVERGED after exactly
    one sweep, with the residual of that sweep reported."""
    torch = pytest.importorskip("torch")
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (12, 16))
    _, D = mh.assemble_matrices(mh.DEFAULT_GREEN_FUNCTIONS, mesh, 0.9, ctx=gpu)
    B = np.ones((mesh.nfaces, 1), dtype=np.complex128)
    rc, _, iters, res = _noalloc(mh, torch, D, B, tol=1e-30, max_iter=1)
    assert rc == mh.native.MH_ERR_NOT_CONVERGED
    assert iters == 1
    assert 0.0 < res < 1e-3


def test_noalloc_rejects_host_memory(mh, gpu):
    """Host buffers are refused before anything is launched on them."""
    torch = pytest.importorskip("torch")
    n = 8
    A = np.eye(n, dtype=np.complex128)
    B = np.ones((n, 1), dtype=np.complex128)
    X = np.zeros((n, 1), dtype=np.complex128)
    L = mh.native.lib()
    rc = L.mh_solve_mixed_noalloc(n, ctypes.c_void_p(A.ctypes.data), ctypes.c_void_p(B.ctypes.data), 1,
                                  ctypes.c_void_p(X.ctypes.data), 1e-10, 10, None, None, None)
    assert rc == mh.native.MH_ERR_ARG
    assert b"current device" in L.mh_last_error(None)
