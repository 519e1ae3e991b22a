"""ctypes binding of ``lib/libmarinehydro_b200.so`` (declared in
``include/marinehydro_b200.h``).

There is no fallback: if the shared library is missing this module raises,
and every compute call surfaces the library's status code as an exception.
"""
from __future__ import annotations

import ctypes
import pathlib
import threading

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libmarinehydro_b200.so"

MH_OK = 0
MH_ERR_ARG = 1
MH_ERR_CUDA = 2
MH_ERR_NOT_CONVERGED = 3
MH_ERR_TIMEOUT = 4
MH_ERR_OOM = 5
MH_ERR_NO_DEVICE = 6
MH_ERR_SINGULAR = 7

MH_DELHOMMEAU_TABLE = 0
MH_DELHOMMEAU_EXACT = 1

MH_LU_SIMT_F32 = 0
MH_LU_TCGEN05_F16 = 1

MH_PRECISION_FP64 = 0
MH_PRECISION_MIXED = 1
MH_PRECISION_FP64_BATCHED = 2

_NAMES = {MH_ERR_ARG: "MH_ERR_ARG", MH_ERR_CUDA: "MH_ERR_CUDA",
          MH_ERR_NOT_CONVERGED: "MH_ERR_NOT_CONVERGED", MH_ERR_TIMEOUT: "MH_ERR_TIMEOUT",
          MH_ERR_OOM: "MH_ERR_OOM", MH_ERR_NO_DEVICE: "MH_ERR_NO_DEVICE",
          MH_ERR_SINGULAR: "MH_ERR_SINGULAR"}


class MarineHydroError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{_NAMES.get(code, code)}: {message}")
        self.code = code


class ArgumentError(MarineHydroError, ValueError):
    """Bad shapes or values (the reference raises from its @assert checks)."""


class NotConvergedError(MarineHydroError):
    pass


class DeviceTimeoutError(MarineHydroError):
    """A bounded device-side wait ran out (MH_ERR_TIMEOUT)."""


class SingularMatrixError(MarineHydroError):
    pass


_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.POINTER(ctypes.c_int64)

# name -> (restype, argtypes); every symbol include/marinehydro_b200.h declares.
SIGNATURES = {
    "mh_version": (ctypes.c_int, []),
    "mh_device_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "mh_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    "mh_ctx_destroy": (ctypes.c_int, [_P]),
    "mh_last_error": (ctypes.c_char_p, [_P]),
    "mh_ctx_kernel_launches": (ctypes.c_int, [_P, _I64]),
    "mh_ctx_set_delhommeau_method": (ctypes.c_int, [_P, ctypes.c_int]),
    "mh_ctx_stream": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    "mh_ctx_set_lu_backend": (ctypes.c_int, [_P, ctypes.c_int]),
    "mh_ctx_set_wait_injection": (ctypes.c_int, [_P, ctypes.c_int]),
    "mh_ctx_set_wave_series_fp32": (ctypes.c_int, [_P, ctypes.c_int]),
    "mh_ctx_set_lu_schedule": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "mh_ctx_get_lu_schedule": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "mh_lu_autotune": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int), _D, ctypes.POINTER(ctypes.c_int)]),
    "mh_lu_factor_lowp": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, _D,
                                         ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_int)]),
    "mh_lu_solve_lowp": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, _D, ctypes.c_int64,
                                        ctypes.c_int, _D, _D]),
    "mh_ctx_set_profiling": (ctypes.c_int, [_P, ctypes.c_int]),
    "mh_ctx_phase_times": (ctypes.c_int, [_P, ctypes.c_int, _D, _I64]),
    "mh_wave_term": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_int64, _D, _D, _D]),
    "mh_mesh_create": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int64, _D, _I64, _D, _D, _D, _D,
                                      ctypes.POINTER(_P)]),
    "mh_mesh_destroy": (ctypes.c_int, [_P, _P]),
    "mh_mesh_nfaces": (ctypes.c_int, [_P, _I64]),
    "mh_mesh_nvertices": (ctypes.c_int, [_P, _I64]),
    "mh_mesh_hemisphere": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P)]),
    "mh_mesh_wavebot": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P)]),
    "mh_mesh_combine": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    "mh_mesh_nparams": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "mh_mesh_fields": (ctypes.c_int, [_P, _P, _D, _I64, _D, _D, _D, _D]),
    "mh_mesh_tangent": (ctypes.c_int, [_P, _P, ctypes.c_int, _D, _D, _D, _D, _D]),
    "mh_mesh_param_vjp": (ctypes.c_int, [_P, _P, _D, _D, _D, _D, _D, _D]),
    "mh_assemble_matrices": (ctypes.c_int, [_P, _P, ctypes.c_double, ctypes.c_uint32, ctypes.c_int,
                                            _D, _D]),
    "mh_assemble_matrices_device": (ctypes.c_int, [_P, _P, ctypes.c_double, ctypes.c_uint32,
                                                   ctypes.c_int, _P, _P]),
    "mh_solve": (ctypes.c_int, [_P, ctypes.c_int64, _D, _D, _D, ctypes.c_int64, ctypes.c_int, _D]),
    "mh_calculate_radiation_forces": (ctypes.c_int, [_P, _P, _D, ctypes.c_int64, ctypes.c_double,
                                                     ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                                     _D]),
    "mh_diffraction_force": (ctypes.c_int, [_P, _P, ctypes.c_double, _D, ctypes.c_int64,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_uint32, ctypes.c_int, ctypes.c_int, _D]),
    "mh_hydro_batch": (ctypes.c_int, [_P, _P, ctypes.c_int64, _D, ctypes.c_int64, _D,
                                      ctypes.c_int64, _D, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_int, _D, _D, _D, _D, ctypes.c_void_p]),
    "mh_hydro_batch_vjp": (ctypes.c_int, [_P, _P, ctypes.c_int64, _D, ctypes.c_int64, _D,
                                          ctypes.c_int64, _D, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D,
                                          _D, _D, _D, _D, _D, _D, _D, _D, ctypes.c_void_p]),
    "mh_hydro_batch_jvp": (ctypes.c_int, [_P, _P, ctypes.c_int64, _D, ctypes.c_int64, _D,
                                          ctypes.c_int64, _D, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D,
                                          _D, _D, _D, _D, _D, _D, _D, ctypes.c_void_p]),
    "mh_solve_mixed_noalloc": (ctypes.c_int, [ctypes.c_int64, _P, _P, ctypes.c_int64, _P,
                                              ctypes.c_double, ctypes.c_int, _P,
                                              ctypes.POINTER(ctypes.c_int32),
                                              ctypes.POINTER(ctypes.c_double)]),
}

_lib = None
_lock = threading.Lock()


def lib():
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python marinehydro.jl_b200/build.py` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
        return L


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_D) if a is not None else None


def i64ptr(a: np.ndarray):
    return a.ctypes.data_as(_I64)


def check(rc: int, ctx=None):
    if rc == MH_OK:
        return
    msg = lib().mh_last_error(ctx)
    msg = msg.decode() if msg else ""
    if rc == MH_ERR_ARG:
        raise ArgumentError(rc, msg)
    if rc == MH_ERR_NOT_CONVERGED:
        raise NotConvergedError(rc, msg)
    if rc == MH_ERR_SINGULAR:
        raise SingularMatrixError(rc, msg)
    if rc == MH_ERR_TIMEOUT:
        raise DeviceTimeoutError(rc, msg)
    raise MarineHydroError(rc, msg)


def device_count() -> int:
    c = ctypes.c_int(0)
    check(lib().mh_device_count(ctypes.byref(c)))
    return int(c.value)


class Context:
    """One device, one CUDA stream, one workspace (``mh_ctx``)."""

    def __init__(self, device: int = 0):
        self._h = _P()
        check(lib().mh_ctx_create(int(device), ctypes.byref(self._h)), None)
        self.device = int(device)

    @property
    def handle(self):
        return self._h

    def set_delhommeau_method(self, method: str):
        """'table' (default) or 'exact' (per-pair adaptive quadrature)."""
        code = {"table": MH_DELHOMMEAU_TABLE, "exact": MH_DELHOMMEAU_EXACT}[method]
        check(lib().mh_ctx_set_delhommeau_method(self._h, code), self._h)

    def wave_term(self, which: int, r, z):
        """Dimensionless (G, dG/dr, dG/dz) at points (r, z) on the device."""
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1)
        z = np.ascontiguousarray(z, dtype=np.float64).reshape(-1)
        out = np.empty((r.shape[0], 6))
        check(lib().mh_wave_term(self._h, int(which), r.shape[0], dptr(r), dptr(z), dptr(out)),
              self._h)
        c = out[:, 0::2] + 1j * out[:, 1::2]
        return c[:, 0], c[:, 1], c[:, 2]

    PHASES = ("rankine", "wave", "rhs", "lu", "refine", "forces", "fp64_assembly", "fp64_lu",
              "adj_solve", "adj_wave", "adj_rankine", "adj_linear")

    def set_lu_backend(self, backend: str):
        """'simt' (FP32 CUDA cores) or 'tcgen05' (FP16 tensor-core trailing update)."""
        code = {"simt": MH_LU_SIMT_F32, "tcgen05": MH_LU_TCGEN05_F16}[backend]
        check(lib().mh_ctx_set_lu_backend(self._h, code), self._h)

    # candidates of the LU autotuner: (groups, 64-column panels per outer
    # step, update kernel 0 = C through shared memory after the MMAs,
    # 1 = C staged in tensor memory before them)
    LU_CANDIDATES = ((1, 4, 0), (2, 2, 0), (2, 4, 0), (2, 6, 0), (3, 4, 0), (4, 4, 0),
                     (1, 4, 1), (2, 2, 1), (2, 4, 1), (2, 6, 1), (3, 4, 1), (4, 4, 1))

    def set_lu_schedule(self, n: int, groups: int, outer_panels: int, update_kernel: int = 0):
        """Tensor-core LU schedule for matrices of n panels (n = 0: the default)."""
        check(lib().mh_ctx_set_lu_schedule(self._h, int(n), int(groups), int(outer_panels), int(update_kernel)),
              self._h)

    def lu_schedule(self, n: int = 0) -> tuple:
        g, o, u = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        check(lib().mh_ctx_get_lu_schedule(self._h, int(n), ctypes.byref(g), ctypes.byref(o), ctypes.byref(u)),
              self._h)
        return int(g.value), int(o.value), int(u.value)

    def autotune_lu(self, n: int, nbatch: int, candidates=None) -> dict:
        """Time each candidate schedule (groups, outer_panels, update_kernel)
        on nbatch synthetic n x n matrices and keep the fastest for n
        (``mh_lu_autotune``).  Returns {"n", "nbatch", "best", "ms": {candidate: ms}}."""
        cand = [tuple(c) if len(c) == 3 else (c[0], c[1], 0) for c in (candidates or self.LU_CANDIDATES)]
        g = (ctypes.c_int * len(cand))(*[c[0] for c in cand])
        o = (ctypes.c_int * len(cand))(*[c[1] for c in cand])
        u = (ctypes.c_int * len(cand))(*[c[2] for c in cand])
        ms = np.zeros(len(cand))
        best = ctypes.c_int(-1)
        check(lib().mh_lu_autotune(self._h, int(n), int(nbatch), len(cand), g, o, u, dptr(ms), ctypes.byref(best)),
              self._h)
        return {"n": int(n), "nbatch": int(nbatch), "best": cand[best.value],
                "ms": {c: float(t) for c, t in zip(cand, ms)}}

    def save_lu_table(self, path, entries):
        """Write autotuner results ({n: (groups, outer_panels, update_kernel)}) as JSON."""
        import json

        pathlib.Path(path).write_text(json.dumps({str(int(k)): list(v) for k, v in entries.items()}, indent=1))

    def load_lu_table(self, path) -> dict:
        """Set the schedules of a table written by save_lu_table on this ctx."""
        import json

        table = {int(k): tuple(v) for k, v in json.loads(pathlib.Path(path).read_text()).items()}
        for n, sched in table.items():
            self.set_lu_schedule(n, *sched)
        return table

    def wave_series_level(self) -> int:
        """The level last set with set_wave_series_fp32 on this Context (the
        library's default, 1, unless set)."""
        return getattr(self, "_wave_level", 1)

    def set_wave_series_fp32(self, level: int):
        """Reduced-precision level of the mixed path's frequency-batched
        Delhommeau pass (``mh_ctx_set_wave_series_fp32``): 0 all FP64, 1 (the
        default) the per-frequency Horner series in FP32, 2 also the alpha
        contraction."""
        check(lib().mh_ctx_set_wave_series_fp32(self._h, int(level)), self._h)
        self._wave_level = int(level)

    def set_wait_injection(self, enable: bool):
        """Failure injection (tests): the triangular solves' flag waits wait
        on a flag nothing publishes, so they expire (``mh_ctx_set_wait_injection``)."""
        check(lib().mh_ctx_set_wait_injection(self._h, int(bool(enable))), self._h)

    def lu_factor_lowp(self, A, backend: str = "tcgen05"):
        """Pivot-free low-precision LU of a batch (nbatch, n, n) of complex
        matrices; returns (LU as complex64 (nbatch, n, n), bad flags)."""
        A = np.asarray(A, dtype=np.complex128)
        if A.ndim == 2:
            A = A[None]
        nb, n, _ = A.shape
        # column-major per matrix: the transpose of each C-ordered matrix
        Af = np.ascontiguousarray(np.transpose(A, (0, 2, 1)))
        LU = np.empty((nb, n, n), dtype=np.complex64)
        bad = np.zeros(nb, dtype=np.int32)
        code = {"simt": MH_LU_SIMT_F32, "tcgen05": MH_LU_TCGEN05_F16}[backend]
        check(lib().mh_lu_factor_lowp(self._h, code, n, nb, dptr(Af),
                                      LU.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                      bad.ctypes.data_as(ctypes.POINTER(ctypes.c_int))), self._h)
        return np.transpose(LU, (0, 2, 1)), bad

    def lu_solve_lowp(self, A, B, backend: str = "tcgen05", conj_trans: bool = False):
        """Low-precision LU of A (nbatch, n, n), then op(L U) X = B with those
        factors (B: (nbatch, n, nrhs)); returns X as complex128."""
        A = np.asarray(A, dtype=np.complex128)
        B = np.asarray(B, dtype=np.complex128)
        if A.ndim == 2:
            A, B = A[None], B[None]
        nb, n, _ = A.shape
        nrhs = B.shape[2]
        Af = np.ascontiguousarray(np.transpose(A, (0, 2, 1)))
        Bf = np.ascontiguousarray(np.transpose(B, (0, 2, 1)))  # right-hand sides contiguous
        X = np.empty_like(Bf)
        code = {"simt": MH_LU_SIMT_F32, "tcgen05": MH_LU_TCGEN05_F16}[backend]
        check(lib().mh_lu_solve_lowp(self._h, code, n, nb, dptr(Af), nrhs, int(conj_trans), dptr(Bf), dptr(X)),
              self._h)
        return np.transpose(X, (0, 2, 1))

    def stream(self) -> int:
        """The ctx's cudaStream_t as an integer handle."""
        p = _P()
        check(lib().mh_ctx_stream(self._h, ctypes.byref(p)), self._h)
        return int(p.value or 0)

    def set_profiling(self, enable: bool):
        check(lib().mh_ctx_set_profiling(self._h, int(bool(enable))), self._h)

    def phase_times(self) -> dict:
        """name -> (total ms, number of timed occurrences) since profiling was enabled."""
        n = len(self.PHASES)
        ms = np.zeros(n)
        calls = np.zeros(n, dtype=np.int64)
        check(lib().mh_ctx_phase_times(self._h, n, dptr(ms), i64ptr(calls)), self._h)
        return {name: (float(ms[q]), int(calls[q])) for q, name in enumerate(self.PHASES)}

    def kernel_launches(self) -> int:
        c = ctypes.c_int64(0)
        check(lib().mh_ctx_kernel_launches(self._h, ctypes.byref(c)), self._h)
        return int(c.value)

    def close(self):
        if self._h:
            lib().mh_ctx_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx
