"""LSQR on the GPU behind the reference's Lsqr.Solve surface (Numerics/Lsqr.cs:33-152).

`solve(solver, A, b, ...)` takes a scipy-style CSR (indptr, indices, data) on the host; `solve_rows`
takes the Jacobian rows a ray call left on the device. Both return the reference's LsqrResult fields
and take the reference's `onIteration(iteration, rnorm)` callback. `self_test` is LsqrOpenCl.SelfTest
(Numerics/LsqrOpenCl.cs:541-557), whose tolerance gates LsqrOpenCl.TryCreate.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L

STOPS = ["empty system", "zero right-hand side", "Aᵀb = 0: the data do not see the model",
         "iteration budget exhausted", "residual reduced to tolerance (btol)", "normal equations satisfied (atol)",
         "condition-number limit reached (conlim)", "residual at machine precision",
         "normal equations at machine precision", "condition number at machine precision",
         "bidiagonalisation terminated"]
SELF_TEST_TOLERANCE = 1e-8   # LsqrOpenCl.SelfTestTolerance (LsqrOpenCl.cs:33)
_ITERATION_FN = C.CFUNCTYPE(None, C.c_int32, C.c_double, C.c_void_p)


class _Callback:
    """Installs `on_iteration(iteration, rnorm)` on the context for one call (Lsqr.cs:43,140)."""

    def __init__(self, solver, on_iteration):
        self.solver, self.fn = solver, None
        if on_iteration is not None:
            self.fn = _ITERATION_FN(lambda it, rnorm, _user: on_iteration(int(it), float(rnorm)))

    def __enter__(self):
        if self.fn is not None:
            L.load().ts_lsqr_set_callback(self.solver.handle, C.cast(self.fn, C.c_void_p), None)

    def __exit__(self, *exc):
        if self.fn is not None:
            L.load().ts_lsqr_set_callback(self.solver.handle, None, None)


@dataclass
class LsqrResult:
    """LsqrResult (Lsqr.cs:6-12)."""

    solution: np.ndarray
    iterations: int
    initial_residual_norm: float
    residual_norm: float
    estimated_condition_number: float
    stop_reason: str
    stop: int
    device_ms: float


def _result(x, info) -> LsqrResult:
    return LsqrResult(x, info.iterations, info.bnorm, info.rnorm, info.acond, STOPS[info.stop], info.stop,
                      info.device_ms)


def solve(solver, indptr, indices, data, n: int, b, damp: float = 0.0, max_iterations: int = 500,
          atol: float = 1e-8, btol: float = 1e-8, conlim: float = 1e8, on_iteration=None) -> LsqrResult:
    rp = np.ascontiguousarray(indptr, np.int32)
    ci = np.ascontiguousarray(indices, np.int32)
    va = np.ascontiguousarray(data, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    m = len(rp) - 1
    if len(bb) != m:
        raise ValueError("Right-hand side length differs from the row count.")
    x = np.zeros(n)
    info = L.LsqrInfo()
    P = C.POINTER
    with _Callback(solver, on_iteration):
        rc = L.load().ts_lsqr_solve(solver.handle, m, n, rp.ctypes.data_as(P(C.c_int32)),
                                    ci.ctypes.data_as(P(C.c_int32)), va.ctypes.data_as(P(C.c_double)),
                                    bb.ctypes.data_as(P(C.c_double)), damp, max_iterations, atol, btol, conlim,
                                    x.ctypes.data_as(P(C.c_double)), C.byref(info))
    if rc != L.TS_OK:
        raise L.TsError(rc, solver.last_error)
    return _result(x, info)


def solve_rows(solver, rows_handle, n: int, b, damp: float = 0.0, max_iterations: int = 500, atol: float = 1e-8,
               btol: float = 1e-8, conlim: float = 1e8, on_iteration=None) -> LsqrResult:
    """A = the device-resident rows of a ray call (a ts_rows* handle), n inversion-grid columns."""
    bb = np.ascontiguousarray(b, np.float64)
    x = np.zeros(n)
    info = L.LsqrInfo()
    P = C.POINTER
    with _Callback(solver, on_iteration):
        rc = L.load().ts_lsqr_solve_rows(solver.handle, rows_handle, n, bb.ctypes.data_as(P(C.c_double)), damp,
                                         max_iterations, atol, btol, conlim, x.ctypes.data_as(P(C.c_double)),
                                         C.byref(info))
    if rc != L.TS_OK:
        raise L.TsError(rc, solver.last_error)
    return _result(x, info)


def self_test(solver) -> tuple[float, str]:
    """LsqrOpenCl.SelfTest: (max |dx| / max |x_host|, message); the gate passes at <= 1e-8."""
    rel = C.c_double()
    msg = C.create_string_buffer(256)
    rc = L.load().ts_lsqr_selftest(solver.handle, C.byref(rel), msg, 256)
    if rc not in (L.TS_OK, L.TS_E_SELFTEST):
        raise L.TsError(rc, solver.last_error)
    return rel.value, msg.value.decode()
