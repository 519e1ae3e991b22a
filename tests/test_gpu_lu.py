"""The low-precision LU of the mixed path (GPU).

Backends: FP32 on the CUDA cores (block 32) and the block-64 LU whose
trailing update runs on tcgen05 with FP16 operands and FP32 accumulation.
Checked by reconstruction, ||L U - A||_max / ||A||_max: <= 2e-6 for FP32,
<= 4e-3 for the FP16 tensor-core update (operands rounded to 11 significant
bits), on sizes that are not multiples of the tiles (640: several 256-column
outer steps whose interior tiles take the bulk-copy epilogue; 641: odd, so
every tile takes the per-thread one); and end to end through the batch
driver, whose FP64 refinement must still reach the FP64 result.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bem_like(rng, nb, n):
    """Matrices shaped like the BEM D: 1/2 on the diagonal plus a smooth,
    decaying complex kernel (well conditioned, no pivoting needed)."""
    x = rng.uniform(-1, 1, (nb, n, 3))
    d = np.linalg.norm(x[:, :, None, :] - x[:, None, :, :], axis=-1) + 0.3
    A = (0.8 / n) * (np.exp(-d) * (np.cos(2 * d) + 1j * np.sin(3 * d))) / d
    A += 0.5 * np.eye(n)[None]
    return A


def _reconstruct(LU):
    n = LU.shape[-1]
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    return L @ U


@pytest.mark.parametrize("backend,tol", [("simt", 2e-6), ("tcgen05", 4e-3)])
@pytest.mark.parametrize("n", [64, 200, 320, 640, 641])
def test_lowp_lu_reconstructs(mh, gpu, backend, tol, n):
    rng = np.random.default_rng(n)
    A = _bem_like(rng, 3, n)
    LU, bad = gpu.lu_factor_lowp(A, backend)
    assert not bad.any()
    for b in range(A.shape[0]):
        R = _reconstruct(LU[b].astype(np.complex128))
        err = np.max(np.abs(R - A[b])) / np.max(np.abs(A[b]))
        assert err <= tol, (backend, n, b, err)


@pytest.mark.parametrize("n", [40, 64])
def test_tcgen05_single_block_is_fp32(mh, gpu, n):
    """One diagonal block (n <= 64, padded with the identity when smaller):
    no trailing update, so the tensor-core backend's factors are the FP32
    elimination of the diagonal-block kernel."""
    rng = np.random.default_rng(n + 1)
    A = _bem_like(rng, 3, n)
    LU, bad = gpu.lu_factor_lowp(A, "tcgen05")
    assert not bad.any()
    for b in range(A.shape[0]):
        R = _reconstruct(LU[b].astype(np.complex128))
        assert np.max(np.abs(R - A[b])) / np.max(np.abs(A[b])) <= 2e-6


def test_tcgen05_factors_track_fp32(mh, gpu):
    rng = np.random.default_rng(5)
    A = _bem_like(rng, 2, 300)
    LU32, _ = gpu.lu_factor_lowp(A, "simt")
    LU16, _ = gpu.lu_factor_lowp(A, "tcgen05")
    err = np.max(np.abs(LU16 - LU32)) / np.max(np.abs(LU32))
    assert err < 4e-3


def test_singular_block_flagged(mh, gpu):
    n = 96
    A = np.eye(n, dtype=np.complex128)[None].repeat(2, axis=0)
    A[1, 70, 70] = 0.0
    for backend in ("simt", "tcgen05"):
        _, bad = gpu.lu_factor_lowp(A, backend)
        assert bad[0] == 0 and bad[1] != 0


@pytest.mark.parametrize("direct", [True, False])
def test_batch_with_tensor_core_lu(mh, oracle, gpu, direct):
    """tcgen05 is the default backend; set explicitly to be independent of order."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (14, 20))
    body = mh.FloatingBody.rigid(mesh, ["Heave", "Surge"])
    dofs = list(body.dofs.values())
    om = [0.5, 1.2, 2.5]
    gpu.set_lu_backend("tcgen05")
    A, B, Fd, _, info = mh.hydro_batch(mesh, om, dofs, [0.0], direct=direct, precision="mixed",
                                       tol=1e-12, ctx=gpu)
    Ao, Bo, Fdo, _ = oracle.hydro_coefficients(mesh, om, dofs, [0.0], direct=direct)
    for got, ref in ((A, Ao), (B, Bo), (Fd, Fdo)):
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-9
    assert info.n_fallback == 0
    assert info.refine_iterations <= 12


def test_batch_with_fp32_lu(mh, oracle, gpu):
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (12, 16))
    dofs = [mh.translational_dofs(mesh, "Heave")]
    gpu.set_lu_backend("simt")
    try:
        A, B, _, _, info = mh.hydro_batch(mesh, [0.7, 1.9], dofs, precision="mixed", tol=1e-12,
                                          ctx=gpu)
    finally:
        gpu.set_lu_backend("tcgen05")
    Ao, Bo, _, _ = oracle.hydro_coefficients(mesh, [0.7, 1.9], dofs)
    assert np.max(np.abs(A - Ao)) / np.max(np.abs(Ao)) < 1e-9
    assert info.refine_iterations <= 4


@pytest.mark.parametrize("backend", ["tcgen05", "simt"])
@pytest.mark.parametrize("conj", [False, True])
@pytest.mark.parametrize("n,nrhs", [(40, 2), (64, 1), (130, 3), (200, 3), (256, 4), (320, 5), (517, 16),
                                    (1024, 16), (1100, 4), (1101, 3)])
def test_lowp_solve_matches_its_factors(mh, gpu, backend, conj, n, nrhs):
    """The FP32 block substitution of a refinement step (L U X = B, or
    (L U)^H X = B for the adjoint) against the same factors solved in FP64:
    sizes with a partial last block, one block, whole blocks only; one to
    four right-hand sides (each count its own compile-time variant) and more.
    Even sizes with one to four right-hand sides take the streamed
    left-looking solve of the tensor-core backend (its partial last block:
    130 and 1100); odd sizes and more right-hand sides the flag-synchronised
    right-looking one, where at 1024 x 16 the next block is not staged in
    shared memory (two CTAs would no longer fit on an SM)."""
    rng = np.random.default_rng(10 * n + nrhs)
    A = _bem_like(rng, 2, n)
    B = rng.normal(size=(2, n, nrhs)) + 1j * rng.normal(size=(2, n, nrhs))
    LU, bad = gpu.lu_factor_lowp(A, backend)
    assert not bad.any()
    X = gpu.lu_solve_lowp(A, B, backend, conj)
    for b in range(A.shape[0]):
        M = _reconstruct(LU[b].astype(np.complex128))
        if conj:
            M = M.conj().T
        ref = np.linalg.solve(M, B[b])
        err = np.max(np.abs(X[b] - ref)) / np.max(np.abs(ref))
        assert err <= 1e-5, (backend, conj, n, nrhs, b, err)


def test_solve_wait_timeout_is_reported(mh, gpu):
    """Failure injection: the flag waits of the tensor-core backend's
    triangular solve wait on a flag that nothing publishes (64 polls), so they
    expire; the solve marks the matrices, the call returns MH_ERR_TIMEOUT,
    the kernel ends and the context stays usable."""
    rng = np.random.default_rng(21)
    A = _bem_like(rng, 2, 256)
    B = rng.normal(size=(2, 256, 2)) + 1j * rng.normal(size=(2, 256, 2))
    gpu.set_wait_injection(True)
    try:
        with pytest.raises(mh.native.DeviceTimeoutError):
            gpu.lu_solve_lowp(A, B, "tcgen05")
    finally:
        gpu.set_wait_injection(False)
    X = gpu.lu_solve_lowp(A, B, "tcgen05")
    for b in range(2):
        ref = np.linalg.solve(A[b], B[b])
        assert np.max(np.abs(X[b] - ref)) / np.max(np.abs(ref)) <= 1e-2


def test_batch_falls_back_when_the_solve_times_out(mh, oracle, gpu):
    """A timed-out wait in the mixed refinement marks its frequency; the batch
    solves it with the pivoted FP64 LU instead, so the outputs stay exact."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (12, 16))
    dofs = [mh.translational_dofs(mesh, "Heave")]
    gpu.set_lu_backend("tcgen05")
    gpu.set_wait_injection(True)
    try:
        A, B, _, _, info = mh.hydro_batch(mesh, [0.7, 1.9], dofs, precision="mixed", tol=1e-12, ctx=gpu)
    finally:
        gpu.set_wait_injection(False)
    assert info.n_fallback == 2
    Ao, Bo, _, _ = oracle.hydro_coefficients(mesh, [0.7, 1.9], dofs)
    assert np.max(np.abs(A - Ao)) / np.max(np.abs(Ao)) < 1e-10
    assert np.max(np.abs(B - Bo)) / np.max(np.abs(Bo)) < 1e-10
    A2, _, _, _, info2 = mh.hydro_batch(mesh, [0.7, 1.9], dofs, precision="mixed", tol=1e-12, ctx=gpu)
    assert info2.n_fallback == 0 and np.max(np.abs(A2 - Ao)) / np.max(np.abs(Ao)) < 1e-9


def test_refinement_skips_converged_frequencies(mh, oracle, gpu):
    """Per-frequency convergence: the frequencies are refined independently,
    each to tol, and the sweep count reported is the largest any needed."""
    mesh = mh.mesh_hemisphere(1.0, (0, 0, 0), (12, 16))
    dofs = [mh.translational_dofs(mesh, "Heave")]
    om = [0.3, 1.0, 2.0, 3.0]
    for tol in (1e-6, 1e-12):
        A, B, _, _, info = mh.hydro_batch(mesh, om, dofs, precision="mixed", tol=tol, ctx=gpu)
        assert info.n_fallback == 0 and info.max_rel_residual <= tol
        assert 1 <= info.refine_iterations <= 6
    Ao, _, _, _ = oracle.hydro_coefficients(mesh, om, dofs)
    assert np.max(np.abs(A - Ao)) / np.max(np.abs(Ao)) < 1e-9


@pytest.mark.parametrize("groups,outer,update", [(1, 2, 0), (1, 4, 1), (2, 6, 0), (2, 4, 1), (3, 8, 1), (4, 4, 0),
                                                 (4, 8, 1)])
@pytest.mark.parametrize("n", [640, 641, 1100])
def test_tcgen05_lu_schedules_reconstruct(mh, gpu, groups, outer, update, n):
    """Every schedule the autotuner may pick (stream groups, 64-column panels
    per outer step, update kernel) factors the same matrices to the same
    accuracy; 1100 has several outer steps of every width and a ragged last
    tile."""
    rng = np.random.default_rng(n + 7 * outer + groups)
    A = _bem_like(rng, 5, n)
    # a context of its own: an entry for this size in its schedule table (a
    # size takes the nearest entry, so the default alone would not be used)
    ctx = mh.Context(0)
    try:
        ctx.set_lu_schedule(n, groups, outer, update)
        assert ctx.lu_schedule(n) == (groups, outer, update)
        LU, bad = ctx.lu_factor_lowp(A, "tcgen05")
    finally:
        ctx.close()
    assert not bad.any()
    for b in range(A.shape[0]):
        R = _reconstruct(LU[b].astype(np.complex128))
        assert np.max(np.abs(R - A[b])) / np.max(np.abs(A[b])) <= 4e-3, (groups, outer, n, b)


def test_builtin_lu_schedule_table(mh):
    """A new context carries the autotuner's choices per size; other sizes
    take the nearest entry (in log n)."""
    ctx = mh.Context(0)
    try:
        assert ctx.lu_schedule(512) == (1, 4, 1)
        assert ctx.lu_schedule(1024) == (1, 4, 0)
        assert ctx.lu_schedule(2048) == (2, 8, 0)
        assert ctx.lu_schedule(1640) == (1, 4, 0) and ctx.lu_schedule(64) == (1, 4, 1)
        assert ctx.lu_schedule(0) == (2, 4, 0)
    finally:
        ctx.close()


def test_lu_autotune_sets_the_fastest(mh, gpu):
    cand = [(1, 4, 0), (2, 4, 0), (2, 8, 1)]
    out = gpu.autotune_lu(512, 6, cand)
    assert set(out["ms"]) == set(cand) and all(0.0 < t < 1e4 for t in out["ms"].values())
    assert out["best"] == min(out["ms"], key=out["ms"].get)
    assert gpu.lu_schedule(512) == out["best"]
    assert gpu.lu_schedule(500) == out["best"]  # nearest entry
    assert gpu.lu_schedule(0) == (2, 4, 0)  # the default is untouched
    gpu.set_lu_schedule(512, 1, 4, 1)  # back to the built-in entry
