"""The CPU oracle, pinned against the reference's own outputs (golden fixtures
made by the reference's Python with scipy) and against closed forms."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from appt_spgemm_b200 import csr

TASKS = ("AA", "AAt")


def rel_close(a, b, rtol):
    return abs(a - b) <= rtol * max(1.0, abs(b))


@pytest.mark.parametrize("task", TASKS)
def test_oracle_matches_reference_checksums(golden, golden_dir, task):
    """nnz equals the structural product; checksums equal checksum(scipy A@A)
    (src/export_bin.py:31-35) within 1e-12 when summed sequentially, and bit
    for bit when summed the way that function sums (numpy's pairwise sum over
    the entries scipy keeps, i.e. without exact zeros) — which holds only if
    every value equals scipy's bit for bit."""
    exact = 0
    for name, g in golden["cases"].items():
        A = csr.load_bin(os.path.join(golden_dir, name + ".csr"))
        cp, ci, cx = oracle.multiply(A, task)
        ref = g[task]
        assert len(ci) == ref["nnz_structural"], name
        assert len(ci) >= ref["nnz_scipy"], name
        assert np.count_nonzero(cx) == ref["nnz_scipy"], name
        s, a, q = oracle.checksum(cx)
        for mine, theirs in ((s, ref["sum"]), (a, ref["abssum"]), (q, ref["sq"])):
            assert rel_close(mine, theirs, 1e-12), (name, task, mine, theirs)
        nz = cx[cx != 0]
        pairwise = (float(nz.sum()), float(np.abs(nz).sum()), float((nz * nz).sum()))
        exact += pairwise == (ref["sum"], ref["abssum"], ref["sq"])
        assert oracle.products(A, task) == g["products"][task]
        assert csr.products(A, task) == g["products"][task]
    assert exact == len(golden["cases"])


@pytest.mark.parametrize("task", TASKS)
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_structure_and_values_vs_scipy(task, seed):
    A = csr.erdos_renyi(700, 5.0 + seed, seed=seed)
    cp, ci, cx = oracle.multiply(A, task)
    S = A.to_scipy()
    P = S.copy()
    P.data[:] = 1.0
    pat = (P @ P if task == "AA" else P @ P.T).tocsr()
    pat.sort_indices()
    assert np.array_equal(cp, pat.indptr)
    assert np.array_equal(ci, pat.indices)
    num = (S @ S if task == "AA" else S @ S.T).tocsr()
    num.sort_indices()
    dense_o = sp.csr_matrix((cx, ci, cp), shape=(A.n, A.n)).toarray()
    assert np.array_equal(dense_o, num.toarray())


def test_laplacian_square_closed_form():
    """(4I − adjacency)² of the 2-D grid: interior rows are the 13-point stencil
    20 / −8 (distance 1) / +2 (diagonal) / +1 (distance 2), exactly."""
    side = 64
    A = csr.laplace2d(side)
    cp, ci, cx = oracle.multiply(A, "AA")
    assert len(ci) == 51972
    want = {0: 20.0, 1: -8.0, -1: -8.0, side: -8.0, -side: -8.0, 2: 1.0, -2: 1.0,
            2 * side: 1.0, -2 * side: 1.0, side + 1: 2.0, side - 1: 2.0, -side + 1: 2.0,
            -side - 1: 2.0}
    for y in range(2, side - 2):
        for x in range(2, side - 2):
            i = y * side + x
            row = dict(zip(ci[cp[i]:cp[i + 1]] - i, cx[cp[i]:cp[i + 1]]))
            assert row == want


def test_gram_is_symmetric_bitwise():
    A = csr.uniform(400, 6, seed=5)
    cp, ci, cx = oracle.multiply(A, "AAt")
    M = sp.csr_matrix((cx, ci, cp), shape=(A.n, A.n))
    assert (M != M.T).nnz == 0


def test_transpose_matches_scipy():
    A = csr.rmat(10, 8, seed=21)
    T = oracle.transpose(A)
    S = A.to_scipy().T.tocsr()
    S.sort_indices()
    assert np.array_equal(T.rowptr, S.indptr)
    assert np.array_equal(T.col, S.indices)
    assert np.array_equal(T.val, S.data)
    H = A.transpose()
    assert np.array_equal(H.rowptr, T.rowptr) and np.array_equal(H.col, T.col)


def test_rows_stream_matches_full_product():
    A = csr.banded(2000, 12, 0.3, seed=3)
    cp, ci, cx = oracle.multiply(A, "AA")
    m, chk = oracle.rows_stream(A, A, 100, 900, nthreads=2)
    assert m == cp[900] - cp[100]
    s, a, q = chk
    ref = cx[cp[100]:cp[900]]
    assert abs(s - ref.sum()) <= 1e-9 * max(1, abs(ref.sum()))
    assert abs(a - np.abs(ref).sum()) <= 1e-9 * np.abs(ref).sum()


def test_empty_and_tiny():
    E = csr.CsrHost(0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    cp, ci, cx = oracle.multiply(E, "AA")
    assert len(cp) == 1 and len(ci) == 0
    one = csr.CsrHost(1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([3.0]))
    cp, ci, cx = oracle.multiply(one, "AAt")
    assert list(ci) == [0] and cx[0] == 9.0
    Z = csr.CsrHost(5, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0))
    cp, ci, cx = oracle.multiply(Z, "AA")
    assert list(cp) == [0] * 6


def test_multiply_rows_matches_full_product():
    """The row-sample oracle (used to check products too large to compute
    whole) gives exactly the rows of the full product, in the order asked."""
    A = csr.rmat(11, 8, seed=5)
    rng = np.random.default_rng(3)
    rows = rng.integers(0, A.n, 300)
    for task in ("AA", "AAt"):
        cp, ci, cx = oracle.multiply(A, task)
        sp, si, sx = oracle.multiply_rows(A, rows, task)
        for t, r in enumerate(rows):
            a, b = slice(cp[r], cp[r + 1]), slice(sp[t], sp[t + 1])
            assert np.array_equal(ci[a], si[b])
            assert np.array_equal(cx[a].view(np.int64), sx[b].view(np.int64))
