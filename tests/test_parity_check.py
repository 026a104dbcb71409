"""The parity check catches what it must: mistakes planted in the oracle's
own output (on the CPU) — a value one ulp off, a zero of the other sign, two
column indices swapped inside a row, a cancelled entry dropped — each fail it,
and the untouched output passes."""
import numpy as np
import pytest

import oracle
from appt_spgemm_b200 import csr
from parity import assert_same_csr


@pytest.fixture(scope="module")
def product():
    A = csr.erdos_renyi(300, 6.0, seed=8)
    return A, oracle.multiply(A, "AA")


def copy(ref):
    return tuple(np.array(x, copy=True) for x in ref)


def test_untouched_output_passes(product):
    _, ref = product
    assert_same_csr(copy(ref), ref, "same")


def test_one_ulp_fails(product):
    _, ref = product
    got = copy(ref)
    got[2][len(got[2]) // 2] = np.nextafter(got[2][len(got[2]) // 2], np.inf)
    with pytest.raises(AssertionError, match="values"):
        assert_same_csr(got, ref, "ulp")


def test_sign_of_zero_fails():
    rp = np.array([0, 1], np.int64)
    ci = np.array([0], np.int32)
    with pytest.raises(AssertionError, match="values"):
        assert_same_csr((rp, ci, np.array([-0.0])), (rp, ci, np.array([0.0])), "zero")


def test_swapped_columns_fail(product):
    _, ref = product
    got = copy(ref)
    rp = got[0]
    row = int(np.argmax(np.diff(rp)))
    a = int(rp[row])
    got[1][a], got[1][a + 1] = got[1][a + 1], got[1][a]
    with pytest.raises(AssertionError, match="col"):
        assert_same_csr(got, ref, "order")


def test_dropped_cancelled_entry_fails():
    """Structural semantics: an entry whose products cancel stays, as 0.0."""
    A = csr.CsrHost(2, np.array([0, 2, 3], np.int32), np.array([0, 1, 0], np.int32),
                    np.array([1.0, 1.0, -1.0]))
    ref = oracle.multiply(A, "AA")
    zero = np.nonzero(ref[2] == 0.0)[0]
    assert len(zero) == 1  # (0,0): 1·1 + 1·(−1)
    keep = np.ones(len(ref[1]), bool)
    keep[zero] = False
    rp = ref[0].copy()
    rp[1:] -= np.cumsum(np.bincount(np.repeat(np.arange(2), np.diff(ref[0])), weights=~keep,
                                    minlength=2)).astype(rp.dtype)
    with pytest.raises(AssertionError, match="rowptr"):
        assert_same_csr((rp, ref[1][keep], ref[2][keep]), ref, "pruned")
