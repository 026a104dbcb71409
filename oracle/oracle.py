"""ctypes wrapper of the C oracle (gustavson.c) — TEST INFRASTRUCTURE ONLY.

Matrices are (n, rowptr int32, col int32, val float64) numpy tuples or any
object with those attributes.  See gustavson.c for the semantics and the
reference lines each function restates.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            subprocess.run(["make", "-C", _HERE, "_build/liboracle.so"], check=True,
                           capture_output=True)
        L = ctypes.CDLL(_LIB)
        L.oracle_count.restype = ctypes.c_int64
        L.oracle_count.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, _i64p, ctypes.c_int]
        L.oracle_fill.restype = ctypes.c_int
        L.oracle_fill.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p, _i64p,
                                  _i32p, _f64p, ctypes.c_int]
        L.oracle_transpose.restype = None
        L.oracle_transpose.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.oracle_products.restype = ctypes.c_int64
        L.oracle_products.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p]
        L.oracle_checksum.restype = None
        L.oracle_checksum.argtypes = [_f64p, ctypes.c_int64, _f64p]
        L.oracle_rows_stream.restype = ctypes.c_int64
        L.oracle_rows_stream.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p,
                                         ctypes.c_int32, ctypes.c_int32, ctypes.c_int, _f64p]
        L.oracle_rows_count.restype = ctypes.c_int64
        L.oracle_rows_count.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, _i32p,
                                        ctypes.c_int32, _i64p, ctypes.c_int]
        L.oracle_rows_fill.restype = ctypes.c_int
        L.oracle_rows_fill.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p,
                                       _i32p, ctypes.c_int32, _i64p, _i32p, _f64p, ctypes.c_int]
        L.oracle_gen_stencil27.restype = ctypes.c_int64
        L.oracle_gen_stencil27.argtypes = [ctypes.c_int32, ctypes.c_uint64, _i32p, _i32p, _f64p]
        L.oracle_max_threads.restype = ctypes.c_int
        L.oracle_max_threads.argtypes = []
        _lib = L
    return _lib


def _arrs(A):
    n = int(A.n)
    rp = np.ascontiguousarray(A.rowptr, dtype=np.int32)
    col = np.ascontiguousarray(A.col, dtype=np.int32)
    val = np.ascontiguousarray(A.val, dtype=np.float64)
    return n, rp, col, val


def _p(a, t):
    return a.ctypes.data_as(t)


class _Csr:
    def __init__(self, n, rowptr, col, val):
        self.n, self.rowptr, self.col, self.val = n, rowptr, col, val

    @property
    def nnz(self) -> int:
        return int(len(self.col))


def transpose(A):
    """Aᵀ by a sequential stable counting sort (rows of Aᵀ ascending)."""
    n, rp, col, val = _arrs(A)
    tp = np.zeros(n + 1, dtype=np.int32)
    tc = np.zeros(max(len(col), 1), dtype=np.int32)
    tv = np.zeros(max(len(col), 1), dtype=np.float64)
    _load().oracle_transpose(n, _p(rp, _i32p), _p(col, _i32p), _p(val, _f64p), _p(tp, _i32p),
                             _p(tc, _i32p), _p(tv, _f64p))
    return _Csr(n, tp, tc[: len(col)], tv[: len(col)])


def multiply(A, task: str = "AA", nthreads: int = 0):
    """C = A·B (B = A for "AA", Aᵀ for "AAt"/"AAtS"): (rowptr int64, col int32, val float64)."""
    n, rp, col, val = _arrs(A)
    B = _Csr(n, rp, col, val) if task == "AA" else transpose(A)
    bn, brp, bcol, bval = _arrs(B)
    L = _load()
    rownnz = np.zeros(max(n, 1), dtype=np.int64)
    tot = L.oracle_count(n, _p(rp, _i32p), _p(col, _i32p), _p(brp, _i32p), _p(bcol, _i32p),
                         _p(rownnz, _i64p), nthreads)
    if tot < 0:
        raise MemoryError("oracle count failed")
    cp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(rownnz[:n], out=cp[1:])
    ci = np.zeros(max(tot, 1), dtype=np.int32)
    cx = np.zeros(max(tot, 1), dtype=np.float64)
    rc = L.oracle_fill(n, _p(rp, _i32p), _p(col, _i32p), _p(val, _f64p), _p(brp, _i32p),
                       _p(bcol, _i32p), _p(bval, _f64p), _p(cp, _i64p), _p(ci, _i32p),
                       _p(cx, _f64p), nthreads)
    if rc != 0:
        raise RuntimeError("oracle fill failed")
    return cp, ci[:tot], cx[:tot]


def products(A, task: str = "AA") -> int:
    """Intermediate products Σ_{(i,k)} nnz(B_k)."""
    n, rp, col, val = _arrs(A)
    B = _Csr(n, rp, col, val) if task == "AA" else transpose(A)
    return int(_load().oracle_products(n, _p(rp, _i32p), _p(col, _i32p),
                                       _p(np.ascontiguousarray(B.rowptr, dtype=np.int32), _i32p)))


def checksum(vals) -> tuple:
    v = np.ascontiguousarray(vals, dtype=np.float64)
    out = np.zeros(3, dtype=np.float64)
    _load().oracle_checksum(_p(v, _f64p), len(v), _p(out, _f64p))
    return (float(out[0]), float(out[1]), float(out[2]))


def rows_stream(A, B, r0: int, r1: int, nthreads: int = 0):
    """CPU baseline: rows [r0, r1) of A·B with bounded memory; (nnz, (s, as, sq))."""
    n, rp, col, val = _arrs(A)
    _, brp, bcol, bval = _arrs(B)
    chk = np.zeros(3, dtype=np.float64)
    m = _load().oracle_rows_stream(n, _p(rp, _i32p), _p(col, _i32p), _p(val, _f64p),
                                   _p(brp, _i32p), _p(bcol, _i32p), _p(bval, _f64p), r0, r1,
                                   nthreads, _p(chk, _f64p))
    if m < 0:
        raise MemoryError("oracle rows_stream failed")
    return int(m), (float(chk[0]), float(chk[1]), float(chk[2]))


def multiply_rows(A, rows, task: str = "AA", B=None, nthreads: int = 0):
    """Rows `rows` (int array, any order) of C = A·B, B as in multiply() unless
    given: (rowptr int64 over the sample, col int32, val float64) — the check
    for products too large to compute whole."""
    n, rp, col, val = _arrs(A)
    if B is None:
        B = _Csr(n, rp, col, val) if task == "AA" else transpose(A)
    _, brp, bcol, bval = _arrs(B)
    r = np.ascontiguousarray(rows, dtype=np.int32)
    m = len(r)
    L = _load()
    cnt = np.zeros(max(m, 1), dtype=np.int64)
    tot = L.oracle_rows_count(n, _p(rp, _i32p), _p(col, _i32p), _p(brp, _i32p), _p(bcol, _i32p),
                              _p(r, _i32p), m, _p(cnt, _i64p), nthreads)
    if tot < 0:
        raise MemoryError("oracle rows count failed")
    cp = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(cnt[:m], out=cp[1:])
    ci = np.zeros(max(tot, 1), dtype=np.int32)
    cx = np.zeros(max(tot, 1), dtype=np.float64)
    rc = L.oracle_rows_fill(n, _p(rp, _i32p), _p(col, _i32p), _p(val, _f64p), _p(brp, _i32p),
                            _p(bcol, _i32p), _p(bval, _f64p), _p(r, _i32p), m, _p(cp, _i64p),
                            _p(ci, _i32p), _p(cx, _f64p), nthreads)
    if rc != 0:
        raise RuntimeError("oracle rows fill failed")
    return cp, ci[:tot], cx[:tot]


def gen_stencil27(side: int, seed: int):
    """The benchmark's 27-point stencil on side³ (gustavson.c: oracle_gen_stencil27),
    built without the engine library: an object with n, rowptr, col, val."""
    n = side ** 3
    nnz = (3 * side - 2) ** 3
    rp = np.zeros(n + 1, dtype=np.int32)
    col = np.zeros(nnz, dtype=np.int32)
    val = np.zeros(nnz, dtype=np.float64)
    got = _load().oracle_gen_stencil27(side, seed, _p(rp, _i32p), _p(col, _i32p), _p(val, _f64p))
    if got != nnz:
        raise RuntimeError(f"stencil generator wrote {got} entries, expected {nnz}")
    return _Csr(n, rp, col, val)


def max_threads() -> int:
    return int(_load().oracle_max_threads())
