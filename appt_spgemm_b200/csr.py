"""Host-side CSR container, CSR1 files and the seeded synthetic generators.

``load_bin`` / ``write_bin`` mirror the reference's CSR1 reader and writer
(src/spgemm_engine.cuh:21-32, src/export_bin.py:20-29); the generators build
the matrix families of the benchmark configurations.  All of it runs in the
engine library's host code (C++), reached through the C ABI.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import SpgHostCsr, check, lib


@dataclass
class CsrHost:
    """Square n×n CSR on the host: int32 rowptr/col, float64 val."""

    n: int
    rowptr: np.ndarray
    col: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def _struct(self) -> SpgHostCsr:
        self.rowptr = np.ascontiguousarray(self.rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(self.col, dtype=np.int32)
        self.val = np.ascontiguousarray(self.val, dtype=np.float64)
        return SpgHostCsr(
            self.n, self.nnz,
            self.rowptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            self.col.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            self.val.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def validate(self) -> None:
        """Raise SpgemmError(SPG_ERR_INVALID_CSR) unless rows are sorted and unique."""
        s = self._struct()
        check(lib().spg_host_csr_validate(ctypes.byref(s)), "validate")

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.rowptr), shape=(self.n, self.n))

    def transpose(self) -> "CsrHost":
        """Aᵀ on the host (numpy stable sort), rows sorted."""
        rows = np.repeat(np.arange(self.n, dtype=np.int32), np.diff(self.rowptr))
        order = np.argsort(self.col, kind="stable")
        cnt = np.bincount(self.col, minlength=self.n)
        rp = np.zeros(self.n + 1, dtype=np.int32)
        np.cumsum(cnt, out=rp[1:])
        return CsrHost(self.n, rp, rows[order].astype(np.int32), self.val[order].copy())


def _take(h: SpgHostCsr) -> CsrHost:
    """Copy a library-allocated host CSR into numpy arrays and free it."""
    try:
        n, nnz = int(h.n), int(h.nnz)
        rp = np.ctypeslib.as_array(h.rowptr, shape=(n + 1,)).copy()
        if nnz > 0:
            col = np.ctypeslib.as_array(h.col, shape=(nnz,)).copy()
            val = np.ctypeslib.as_array(h.val, shape=(nnz,)).copy()
        else:
            col = np.zeros(0, dtype=np.int32)
            val = np.zeros(0, dtype=np.float64)
        return CsrHost(n, rp, col, val)
    finally:
        lib().spg_host_csr_free(ctypes.byref(h))


def load_bin(path: str) -> CsrHost:
    """Read a CSR1 file (the reference's load_bin)."""
    h = SpgHostCsr()
    check(lib().spg_csr1_read(str(path).encode(), ctypes.byref(h)), f"read {path}")
    return _take(h)


def write_bin(A: CsrHost, path: str) -> None:
    """Write a CSR1 file (the reference's write_bin; rows must already be sorted)."""
    s = A._struct()
    check(lib().spg_csr1_write(str(path).encode(), ctypes.byref(s)), f"write {path}")


def laplace2d(side: int) -> CsrHost:
    """2-D 5-point Laplacian on side×side: 4.0 diagonal, −1.0 neighbours."""
    h = SpgHostCsr()
    check(lib().spg_gen_laplace2d(side, ctypes.byref(h)), "laplace2d")
    return _take(h)


def stencil27(side: int, seed: int) -> CsrHost:
    """3-D 27-point stencil on side³, values uniform(−1,1) from mt19937_64(seed)."""
    h = SpgHostCsr()
    check(lib().spg_gen_stencil27(side, seed, ctypes.byref(h)), "stencil27")
    return _take(h)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 3) -> CsrHost:
    """R-MAT with duplicates merged, self-loops kept, values uniform(0,1)."""
    h = SpgHostCsr()
    check(lib().spg_gen_rmat(scale, edge_factor, a, b, c, seed, ctypes.byref(h)), "rmat")
    return _take(h)


def banded(n: int, bw: int, fill: float, seed: int) -> CsrHost:
    """Random banded: half-bandwidth bw, in-band fill, diagonal always present."""
    h = SpgHostCsr()
    check(lib().spg_gen_banded(n, bw, fill, seed, ctypes.byref(h)), "banded")
    return _take(h)


def erdos_renyi(n: int, lam: float, seed: int) -> CsrHost:
    """Erdős–Rényi: row nnz ~ Poisson(lam), uniform distinct columns."""
    h = SpgHostCsr()
    check(lib().spg_gen_er(n, lam, seed, ctypes.byref(h)), "erdos_renyi")
    return _take(h)


def uniform(n: int, per_row: int, seed: int) -> CsrHost:
    """Exactly min(per_row, n) random distinct columns per row."""
    h = SpgHostCsr()
    check(lib().spg_gen_uniform(n, per_row, seed, ctypes.byref(h)), "uniform")
    return _take(h)


def batch_mix(count: int = 512, seed: int = 4, n_min: int = 1000, n_max: int = 64000):
    """The batched workload: `count` matrices with n = floor(exp(U(ln n_min,
    ln n_max))); even indices random banded (half-bandwidth U{3..64}, 30%
    in-band fill), odd indices Erdős–Rényi (row nnz ~ Poisson(λ), λ ~ U(4, 32));
    values uniform(−1, 1).  Parameters come from numpy's PCG64(seed); each
    matrix gets its own generator seed.  Returns (matrices, parameter dicts)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    mats, params = [], []
    for b in range(count):
        n = int(np.floor(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        sub = int(rng.integers(0, 2**63 - 1))
        if b % 2 == 0:
            bw = int(rng.integers(3, 65))
            mats.append(banded(n, bw, 0.3, sub))
            params.append({"kind": "banded", "n": n, "bw": bw, "seed": sub})
        else:
            lam = float(rng.uniform(4.0, 32.0))
            mats.append(erdos_renyi(n, lam, sub))
            params.append({"kind": "er", "n": n, "lambda": lam, "seed": sub})
    return mats, params


def products(A: CsrHost, task: str) -> int:
    """Intermediate products: A·A Σ_{(i,k)} nnz(A_k); A·Aᵀ Σ_k colcount(k)²
    (est_outputs, bench/run_baseline.py:38-44)."""
    if task == "AA":
        deg = np.diff(A.rowptr).astype(np.int64)
        return int(deg[A.col].sum())
    cc = np.bincount(A.col, minlength=A.n).astype(np.int64)
    return int((cc * cc).sum())


__all__ = ["CsrHost", "load_bin", "write_bin", "laplace2d", "stencil27", "rmat", "banded",
           "erdos_renyi", "uniform", "products", "_capi"]
