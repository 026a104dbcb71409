"""The power-law benchmark matrix at full size: R-MAT 2^20 (edge factor 16,
(a,b,c,d) = (.57,.19,.19,.05), seed 3), whose C has about 9.7e9 entries
(≈116 GB on the device, more than host memory holds).  The engine computes
the whole product; a seeded sample of rows — 4,096 uniform rows, 512 heavy
rows and the 16 rows with the most products — is checked bit for bit
against the CPU oracle, and the row pointers against the plan's count.
A·Aᵀ through the Gram path is checked the same way at 2^18 (its temporary
lower store would not fit beside a 2^20 C)."""
import numpy as np
import pytest

import oracle
from appt_spgemm_b200 import csr

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def sample_rows(A, B, seed):
    deg_b = np.diff(B.rowptr).astype(np.int64)
    cs = np.concatenate([[0], np.cumsum(deg_b[A.col])])
    f = cs[A.rowptr[1:]] - cs[A.rowptr[:-1]]
    rng = np.random.default_rng(seed)
    heavy = np.flatnonzero(f > 8192)
    rows = [rng.integers(0, A.n, 4096), rng.choice(heavy, min(512, len(heavy)), replace=False),
            np.argsort(f)[-16:]]
    return np.unique(np.concatenate(rows)).astype(np.int32)


def check_sample(C, A, task, rows):
    rp = C.rowptr.cpu().numpy()
    assert rp[0] == 0 and rp[-1] == C.nnz and np.all(np.diff(rp) >= 0)
    B = A if task == "AA" else oracle.transpose(A)
    orp, oci, ocx = oracle.multiply_rows(A, rows, task, B=B)
    assert np.array_equal(np.diff(rp)[rows], np.diff(orp)), f"{task}: row lengths"
    idx = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows])
    ti = torch.from_numpy(idx).to(C.col.device)
    gc = C.col[ti].cpu().numpy()
    gv = C.val[ti].cpu().numpy()
    assert np.array_equal(gc, oci), f"{task}: columns"
    assert np.array_equal(gv.view(np.int64), ocx.view(np.int64)), f"{task}: values"


@pytest.mark.parametrize("scale,task", [(20, "AA"), (20, "AAt"), (18, "AAtS")])
def test_rmat_full_size_sampled_rows(scale, task):
    from appt_spgemm_b200.engine import CsrDevice, Engine
    A = csr.rmat(scale, 16, seed=3)
    rows = sample_rows(A, A if task == "AA" else A.transpose(), seed=scale)
    with Engine("cuda:0") as eng:
        dA = CsrDevice.from_host(A, "cuda:0")
        plan = eng.plan(dA, task)
        nnz_c = plan.nnz_c
        C = plan.execute()
        torch.cuda.synchronize()
        plan.close()
        assert C.nnz == nnz_c
        check_sample(C, A, task, rows)
        del C
        torch.cuda.empty_cache()
