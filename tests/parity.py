"""The parity check of the GPU tests: a product equals the oracle's when its row
pointers and column indices are equal and its values are equal bit for bit
(compared as int64 words, so a one-ulp difference or the sign of a zero
counts)."""
import numpy as np


def assert_same_csr(got, ref, label):
    """got, ref: (rowptr, col, val) host arrays."""
    rp, ci, cx = got
    orp, oci, ocx = ref
    assert rp.shape == orp.shape, label
    assert np.array_equal(rp, orp), f"{label}: rowptr"
    assert np.array_equal(ci, oci), f"{label}: col"
    cx = np.ascontiguousarray(cx, dtype=np.float64)
    ocx = np.ascontiguousarray(ocx, dtype=np.float64)
    assert np.array_equal(cx.view(np.int64), ocx.view(np.int64)), (
        f"{label}: values, max |diff| {np.abs(cx - ocx).max() if len(cx) else 0}")
