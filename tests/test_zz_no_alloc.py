"""spg_transpose_noalloc — the transpose for callers that may not allocate device
memory (applications that carve all GPU memory up front and forbid libraries
from calling cudaMalloc/cudaFree, or latency-critical paths where an allocation
may synchronise the device).  It keeps its scratch in a static device array, so
this file checks it against the allocating entry point spg_transpose over two
calls in a row (the second call reuses whatever the first left in the shared
scratch) and checks that inputs beyond its fixed limits are refused.

Named so pytest collects it last; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from appt_spgemm_b200 import _capi, csr
from appt_spgemm_b200._capi import SpgCsrDev, SpgemmError

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def transpose_noalloc(A):
    """Call the entry point through the C ABI with caller-owned torch buffers."""
    dev = torch.device("cuda:0")
    rp = torch.from_numpy(A.rowptr).to(dev)
    col = torch.from_numpy(A.col).to(dev)
    val = torch.from_numpy(A.val).to(dev)
    t_rp = torch.empty(A.n + 1, dtype=torch.int32, device=dev)
    t_col = torch.empty(max(A.nnz, 1), dtype=torch.int32, device=dev)
    t_val = torch.empty(max(A.nnz, 1), dtype=torch.float64, device=dev)
    s = SpgCsrDev(A.n, A.nnz, rp.data_ptr(), col.data_ptr(), val.data_ptr())
    stream = torch.cuda.current_stream().cuda_stream
    _capi.check(_capi.lib().spg_transpose_noalloc(ctypes.byref(s), t_rp.data_ptr(),
                                                  t_col.data_ptr(), t_val.data_ptr(), stream),
                "spg_transpose_noalloc")
    torch.cuda.synchronize()
    return (t_rp.cpu().numpy(), t_col[: A.nnz].cpu().numpy(), t_val[: A.nnz].cpu().numpy())


def transpose_allocating(A):
    from appt_spgemm_b200.engine import CsrDevice, Engine
    with Engine("cuda:0") as eng:
        T = eng.transpose(CsrDevice.from_host(A, "cuda:0"))
        torch.cuda.synchronize()
        return (T.rowptr.cpu().numpy(), T.col.cpu().numpy(), T.val.cpu().numpy())


def test_noalloc_transpose_matches_allocating_entry_point():
    # an R-MAT matrix (columns longer than 256 take the long-segment sort) and
    # a uniform one, back to back through the same static scratch
    cases = [csr.rmat(12, 16, seed=41), csr.uniform(3000, 20, seed=42)]
    for A in cases:
        got = transpose_noalloc(A)
        want = transpose_allocating(A)
        assert np.array_equal(got[0], want[0])
        assert np.array_equal(got[1], want[1])
        assert np.array_equal(got[2].view(np.int64), want[2].view(np.int64))  # bit-exact


def test_noalloc_at_its_limits_and_empty():
    # n = 65,536 rows and nnz = 524,288 entries use the whole static scratch;
    # then matrices with no entries, and one with no rows
    cases = [csr.uniform(65536, 8, seed=43),
             csr.CsrHost(5, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0)),
             csr.CsrHost(0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))]
    assert cases[0].n == 65536 and cases[0].nnz == 524288
    for A in cases:
        for _ in range(2):
            got = transpose_noalloc(A)
            want = transpose_allocating(A)
            assert np.array_equal(got[0], want[0])
            assert np.array_equal(got[1], want[1])
            assert np.array_equal(got[2].view(np.int64), want[2].view(np.int64))


def test_noalloc_refuses_inputs_beyond_its_scratch():
    # one row too many
    n = 65537
    A = csr.CsrHost(n, np.zeros(n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    with pytest.raises(SpgemmError) as e:
        transpose_noalloc(A)
    assert e.value.status == _capi.SPG_ERR_UNSUPPORTED
    # one entry too many (refused on its sizes, before anything runs)
    n, nnz = 65536, 524289
    rp = np.full(n + 1, nnz, np.int32)
    rp[0] = 0
    A = csr.CsrHost(n, rp, np.zeros(nnz, np.int32), np.zeros(nnz))
    with pytest.raises(SpgemmError) as e:
        transpose_noalloc(A)
    assert e.value.status == _capi.SPG_ERR_UNSUPPORTED
