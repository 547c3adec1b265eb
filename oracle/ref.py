"""ctypes front end of oracle/_ref/libref.so — TEST INFRASTRUCTURE ONLY.

libref.so is the reference's own OpenCL kernel text (EikonalOpenCl.cs:387-624, LsqrOpenCl.cs:41-176)
compiled as C++ under oracle/ref_shim.h and driven in the reference host's launch order
(oracle/ref_eik.cpp, oracle/ref_lsqr.cpp). It is built from the reference tree by `make -C oracle ref`
(oracle/ref_extract.py copies the kernel literals into oracle/_ref/, which is never committed); on a
machine without the reference only a prebuilt libref.so can be used. It pins the C++ restatement
(oracle.cpp) and, through it, the CUDA engine: same inputs, same bits.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "libref.so")
REFERENCE_ROOT = os.environ.get("TOMOSTAR_REFERENCE", "/root/reference")


def build() -> str | None:
    """Builds libref.so when the reference tree is present; returns its path, or None when neither the
    tree nor a prebuilt library is there."""
    src = os.path.join(REFERENCE_ROOT, "src", "TomoStar.Core", "Forward", "EikonalOpenCl.cs")
    if os.path.exists(src):
        subprocess.run(["make", "-C", HERE, "ref", f"REF={REFERENCE_ROOT}"], check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH if os.path.exists(LIB_PATH) else None


def available() -> bool:
    try:
        return build() is not None
    except (OSError, subprocess.CalledProcessError):
        return False


_lib = None


def lib():
    global _lib
    if _lib is None:
        if build() is None:
            raise RuntimeError("oracle/_ref/libref.so is not built (no reference tree here)")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        i32, d = C.c_int32, C.c_double
        dp, ip, fp = P(C.c_double), P(C.c_int32), P(C.c_float)
        solve = (i32, [i32, i32, i32, dp, dp, d, dp, i32, ip, ip, dp, i32, dp, ip])
        sig = {
            "ref_eik_solve_f64": solve,
            "ref_eik_solve_paired": solve,
            "ref_spmv_f64": (None, [i32, ip, ip, dp, dp, dp]),
            "ref_xmby_f64": (None, [i32, dp, d, dp]),
            "ref_axpy_f64": (None, [i32, d, dp, dp]),
            "ref_scal_f64": (None, [i32, dp, d]),
            "ref_spmv_paired": (None, [i32, ip, ip, fp, fp, fp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def eik_solve(g: O.Grid, slowness, seed_sets, precision: int = 64, cap: int = 0):
    """EikonalOpenCl.TrySolve + Sweep with the reference's kernel, on one grid and one slowness for a
    batch of seed sets. precision 64 runs the QV_FP64 kernel, 32 the paired-float one. Returns
    (fields (batch, n) float64, status, rounds[2]): status 0 settled, 1 refused as unsettled, 2 no seed."""
    if g.depth is not None:
        raise ValueError("the reference kernel has uniform depth spacing only")
    hlon, hlat, hr, _ = O.metric(g)
    s = np.ascontiguousarray(slowness, np.float64)
    off, idx, t = O._seed_arrays(seed_sets)
    out = np.empty((len(seed_sets), g.count))
    rounds = np.zeros(2, np.int32)
    fn = lib().ref_eik_solve_f64 if precision == 64 else lib().ref_eik_solve_paired
    st = fn(g.nx, g.ny, g.nz, _p(hlon, C.c_double), _p(hlat, C.c_double), hr, _p(s, C.c_double), len(seed_sets),
            _p(off, C.c_int32), _p(idx, C.c_int32), _p(t, C.c_double), cap, _p(out, C.c_double),
            _p(rounds, C.c_int32))
    return out, int(st), rounds


def pairs(v) -> np.ndarray:
    """LsqrOpenCl.PairBits: each double as the floats (hi, lo), hi = (float)v, lo = (float)(v − hi)."""
    v = np.asarray(v, np.float64)
    hi = v.astype(np.float32)
    lo = np.where(np.isfinite(hi), (v - hi.astype(np.float64)).astype(np.float32), np.float32(0))
    return np.ascontiguousarray(np.stack([hi, lo], axis=-1).reshape(-1))


def unpair(p) -> np.ndarray:
    """LsqrOpenCl.Unpair: (double)hi + lo."""
    p = np.asarray(p, np.float32).reshape(-1, 2)
    return p[:, 0].astype(np.float64) + p[:, 1].astype(np.float64)


def spmv(row_ptr, col, val, x, precision: int = 64) -> np.ndarray:
    """The reference's `spmv` kernel (one work item per row, sequential sum) on a CSR matrix."""
    rs = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col, np.int32)
    rows = len(rs) - 1
    if precision == 64:
        va = np.ascontiguousarray(val, np.float64)
        xv = np.ascontiguousarray(x, np.float64)
        y = np.zeros(rows)
        lib().ref_spmv_f64(rows, _p(rs, C.c_int32), _p(ci, C.c_int32), _p(va, C.c_double), _p(xv, C.c_double),
                           _p(y, C.c_double))
        return y
    va, xv = pairs(val), pairs(x)
    y = np.zeros(2 * rows, np.float32)
    lib().ref_spmv_paired(rows, _p(rs, C.c_int32), _p(ci, C.c_int32), _p(va, C.c_float), _p(xv, C.c_float),
                          _p(y, C.c_float))
    return unpair(y)


def xmby(x, b: float, y) -> np.ndarray:
    """The reference's `xmby` kernel: y ← x − b·y."""
    xv = np.ascontiguousarray(x, np.float64)
    yv = np.array(y, np.float64)
    lib().ref_xmby_f64(len(xv), _p(xv, C.c_double), b, _p(yv, C.c_double))
    return yv
