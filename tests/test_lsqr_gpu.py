"""LSQR on the GPU (Lsqr.cs) against the oracle's restatement: the same iterates to rounding over a
fixed number of iterations, the same stopping rule and the solution within the reference's own
device-versus-host bar (LsqrOpenCl.SelfTestTolerance = 1e-8 relative) at convergence, bitwise
repeatable on the device; and on the Jacobian rows a ray call leaves on the device."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import lsqr
from tomostar_b200 import synthetic as syn
from tomostar_b200.rays import _fetch

pytestmark = pytest.mark.gpu


def system(seed=4, m=400, n=150, density=0.04):
    A = sp.random(m, n, density=density, random_state=seed, format="csr")
    b = np.random.default_rng(seed).standard_normal(m)
    return A, b


@pytest.mark.parametrize("damp", [0.0, 0.3])
def test_lsqr_matches_oracle(solver, damp):
    A, b = system()
    m, n = A.shape
    # Fixed iteration count: the same recurrences, differing only by the order of the sums.
    d5 = lsqr.solve(solver, A.indptr, A.indices, A.data, n, b, damp=damp, max_iterations=5, atol=0, btol=0, conlim=0)
    o5, code5, _ = O.lsqr(m, n, A.indptr, A.indices, A.data, b, damp=damp, max_iterations=5, atol=0, btol=0,
                          conlim=0)
    assert d5.stop == code5 == 3
    assert np.max(np.abs(d5.solution - o5)) <= 1e-12 * np.max(np.abs(o5))
    # To convergence.
    d = lsqr.solve(solver, A.indptr, A.indices, A.data, n, b, damp=damp)
    o, code, info = O.lsqr(m, n, A.indptr, A.indices, A.data, b, damp=damp)
    assert d.stop == code and abs(d.iterations - info["iterations"]) <= 2
    assert np.max(np.abs(d.solution - o)) <= 1e-8 * np.max(np.abs(o))
    assert abs(d.residual_norm - info["rnorm"]) <= 1e-8 * info["rnorm"]
    # Repeatable to the bit.
    again = lsqr.solve(solver, A.indptr, A.indices, A.data, n, b, damp=damp)
    assert np.array_equal(again.solution, d.solution) and again.iterations == d.iterations


def test_lsqr_self_test_gate(solver):
    """LsqrOpenCl.SelfTest's gate: the device and the sequential host solver on a random damped
    3000 x 1200 system, 12 non-zeros per row, agree within SelfTestTolerance = 1e-8."""
    rel, message = lsqr.self_test(solver)
    assert rel <= lsqr.SELF_TEST_TOLERANCE, message
    assert "iterations" in message


def test_lsqr_on_iteration(solver):
    """onIteration (Lsqr.cs:140): one call per iteration, numbered from 1, with the ‖r‖ the result
    reports last; LSQR's ‖r‖ never increases. Removed after the call."""
    A, b = system()
    seen = []
    r = lsqr.solve(solver, A.indptr, A.indices, A.data, A.shape[1], b, damp=0.1,
                   on_iteration=lambda it, rn: seen.append((it, rn)))
    assert [it for it, _ in seen] == list(range(1, r.iterations + 1))
    assert seen[-1][1] == r.residual_norm
    rn = np.array([v for _, v in seen])
    assert np.all(np.diff(rn) <= 1e-12 * rn[0])
    calls = len(seen)
    lsqr.solve(solver, A.indptr, A.indices, A.data, A.shape[1], b, damp=0.1)
    assert len(seen) == calls


def test_lsqr_degenerate_systems(solver):
    A, b = system()
    m, n = A.shape
    r = lsqr.solve(solver, A.indptr, A.indices, A.data, n, np.zeros(m))
    assert r.stop_reason == "zero right-hand side" and not r.solution.any()
    empty = sp.csr_matrix((m, n))
    r = lsqr.solve(solver, empty.indptr, empty.indices, empty.data, n, b)
    assert r.stop == 2


def test_lsqr_on_device_resident_rays(solver):
    """Rays of the 61×61×31 model traced to their Jacobian rows on the device, then LSQR on those rows
    without a copy (ts_lsqr_solve_rows), against the oracle on the same rows copied to the host."""
    p = syn.single_source_61()
    lib = L.load()
    fs, is_ = p.grid.struct(), p.inv.struct()
    s = np.ascontiguousarray(p.slowness)
    st = np.ascontiguousarray(p.stations)
    ev = np.ascontiguousarray(p.events)
    ar = np.ascontiguousarray(p.arrivals, np.int32)
    ae, ast, ap = (np.ascontiguousarray(ar[:, q]) for q in range(3))
    P = C.POINTER
    h = C.c_void_p()
    stats = L.EikStats()
    rc = lib.ts_forward(solver.handle, C.byref(fs), s.ctypes.data_as(P(C.c_double)), len(s), C.byref(is_), len(st),
                        st.ctypes.data_as(P(C.c_double)), len(ev), ev.ctypes.data_as(P(C.c_double)), len(ar),
                        ae.ctypes.data_as(P(C.c_int32)), ast.ctypes.data_as(P(C.c_int32)),
                        ap.ctypes.data_as(P(C.c_int32)), 64, L.MODE_ENGINE, 0.0, C.byref(h), C.byref(stats))
    assert rc == 0, solver.last_error
    n = p.inv.count
    b = np.random.default_rng(9).standard_normal(len(ar)) * 0.05
    with pytest.raises(L.TsError):  # columns beyond n are refused, not written
        lsqr.solve_rows(solver, h, 10, b)
    d = lsqr.solve_rows(solver, h, n, b, damp=0.1)
    rows = _fetch(h)  # copies the rows to the host and frees them
    # The transpose built on the device equals the host's (the reference's order): the same system
    # given as host CSR runs the same device arithmetic, so the solutions agree to the bit.
    h_res = lsqr.solve(solver, rows.row_ptr, rows.col, rows.len.astype(np.float64), n, b, damp=0.1)
    assert np.array_equal(h_res.solution, d.solution) and h_res.iterations == d.iterations
    o, code, info = O.lsqr(len(ar), n, rows.row_ptr, rows.col, rows.len.astype(np.float64), b, damp=0.1)
    assert d.stop == code
    assert np.max(np.abs(d.solution - o)) <= 1e-8 * np.max(np.abs(o))
