"""GPU parity: the engine, called through the C ABI, against the CPU oracle.

The bar is bit-exact everywhere: row pointers, sorted column indices and every
FP64 value (the engine and the oracle both add the rounded products of each
entry in increasing position of k in row i of A).  The 1e-12 relative bound
of the task is therefore met with zero error.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from appt_spgemm_b200 import _capi, csr
from appt_spgemm_b200._capi import SpgemmError
from parity import assert_same_csr

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TASKS = ("AA", "AAt", "AAtS")


# Every engine test runs twice: with the default configuration (A·A and A·Aᵀ
# of matrices up to 2^20 entries take the one-readback plan: one warp-per-row
# launch per phase) and with that plan switched off (the binned kernels).
@pytest.fixture(scope="module", params=["default", "binned"])
def eng(request):
    from appt_spgemm_b200.engine import Engine
    e = Engine("cuda:0", **({} if request.param == "default" else {"small_max_nnz": -1}))
    yield e
    e.check_device_status()
    e.close()


def dev(A):
    from appt_spgemm_b200.engine import CsrDevice
    return CsrDevice.from_host(A, "cuda:0")


def assert_same(C, ref, label):
    assert_same_csr(C.to_host(), ref, label)


def run_case(eng, A, task, label):
    C = eng.multiply(dev(A), task)
    torch.cuda.synchronize()
    assert_same(C, oracle.multiply(A, task), f"{label}/{task}")


@pytest.mark.parametrize("task", TASKS)
def test_golden_cases(eng, golden, golden_dir, task):
    for name in golden["cases"]:
        A = csr.load_bin(os.path.join(golden_dir, name + ".csr"))
        run_case(eng, A, task, name)


@pytest.mark.parametrize("task", TASKS)
def test_laplacian_64(eng, task):
    run_case(eng, csr.laplace2d(64), task, "laplace2d_64")


# per-row widths that put rows in every shared-table bin and on the heavy path
@pytest.mark.parametrize("per_row", [1, 2, 3, 5, 8, 12, 16, 24, 32, 48, 64, 96, 128])
@pytest.mark.parametrize("task", TASKS)
def test_every_bin(eng, per_row, task):
    n = 2500 if per_row <= 64 else 4000
    run_case(eng, csr.uniform(n, per_row, seed=per_row), task, f"uniform{per_row}")


# rows of roughly 300 to 5000 entries spread over 70,000 columns: the radix
# sorts of the 512/1024-slot warp tables and of the 2048- to 8192-slot CTA
# tables, with three 8-bit digit passes over 17-bit column fields
@pytest.mark.parametrize("deg", [18.0, 30.0, 60.0])
@pytest.mark.parametrize("task", TASKS)
def test_wide_rows_three_digit_passes(eng, deg, task):
    run_case(eng, csr.erdos_renyi(70000, deg, seed=int(deg)), task, f"er70k_d{int(deg)}")


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
def test_lanes_per_row(lanes):
    from appt_spgemm_b200.engine import Engine
    with Engine("cuda:0", lanes_per_row=lanes, small_max_nnz=-1) as e:
        for task in TASKS:
            run_case(e, csr.erdos_renyi(3000, 9.0, seed=lanes), task, f"er/lanes{lanes}")


@pytest.mark.parametrize("window,split", [(0, 1 << 30), (4096, 1 << 30), (3072, 1 << 30),
                                          (0, 1), (4096, 1), (0, 0)])
def test_force_heavy_dense_windows(window, split):
    """Every row through the heavy path (the reference's debugging trick of
    forcing all rows onto its global path): symbolic bitmap windows of 2^20,
    4096 and 3072 columns (the last cuts rows into 1024-column blocks instead
    of 4096); numeric rows through the windowed warp kernel (split 2^30:
    every row of at most 2^17 products), all through the CTA kernel (split 1)
    or divided by the default rule."""
    from appt_spgemm_b200.engine import Engine
    with Engine("cuda:0", force_heavy=1, window_bits=window, heavy_split=split) as e:
        for A, lab in ((csr.laplace2d(40), "lap40"), (csr.rmat(11, 8, seed=2), "rmat11"),
                       (csr.erdos_renyi(20000, 4.0, seed=3), "er20k")):
            for task in TASKS:
                run_case(e, A, task, f"forced/{lab}/w{window}")


@pytest.mark.parametrize("vcap", [1024, 8192, -1])
def test_heavy_shared_value_windows(vcap):
    """Heavy CTA rows with their values in shared memory window by window:
    1024 values per window (many windows per row; blocks above it cut into
    fixed 1024-column sub-windows), the default 8192, and -1 (the kernel that
    accumulates in place in C); every row forced heavy and onto the CTA kernel,
    then R-MAT heavy rows and 32768-column blocks under the default rules."""
    from appt_spgemm_b200.engine import Engine
    with Engine("cuda:0", force_heavy=1, heavy_split=1, heavy_vcap=vcap) as e:
        for A, lab in ((csr.laplace2d(40), "lap40"), (csr.rmat(11, 8, seed=2), "rmat11"),
                       (csr.erdos_renyi(20000, 4.0, seed=3), "er20k")):
            for task in TASKS:
                run_case(e, A, task, f"win{vcap}/{lab}")
    with Engine("cuda:0", heavy_vcap=vcap) as e:
        for task in TASKS:
            run_case(e, csr.rmat(13, 16, seed=3), task, f"win{vcap}/rmat13")
    with Engine("cuda:0", heavy_vcap=vcap, heavy_block_budget=1 << 16) as e:
        run_case(e, csr.erdos_renyi(30000, 90.0, seed=6), "AA", f"win{vcap}/er30k")


@pytest.mark.parametrize("task", TASKS)
def test_rmat_heavy_rows(eng, task):
    run_case(eng, csr.rmat(13, 16, seed=3), task, "rmat13")


@pytest.mark.parametrize("budget", [1 << 18, 1 << 16, 1])
def test_heavy_block_budget(budget):
    """A small block-count budget widens the column blocks of the heavy rows
    (30,000 rows of ~7,000 entries over 30,000 columns: 4096-column blocks at
    2^18, one 32768-column block per row at 2^16, cut into fixed 1024-column
    windows); a budget below one count per row leaves no counts, and every
    heavy row takes the CTA kernel."""
    from appt_spgemm_b200.engine import Engine
    A = csr.erdos_renyi(30000, 90.0, seed=6)
    with Engine("cuda:0", heavy_block_budget=budget) as e:
        for task in TASKS:
            run_case(e, A, task, f"er30k/budget{budget}")


@pytest.mark.parametrize("split", [1, 1 << 30])
@pytest.mark.parametrize("task", TASKS)
def test_rmat_heavy_split(split, task):
    """R-MAT heavy rows of at most 2^17 products through the windowed warp
    kernel (split 2^30) or all heavy rows through the CTA kernel (split 1)."""
    from appt_spgemm_b200.engine import Engine
    with Engine("cuda:0", heavy_split=split) as e:
        run_case(e, csr.rmat(14, 16, seed=4), task, f"rmat14/split{split}")


def test_one_readback_plan(eng):
    """Small A·A and A·Aᵀ plans: with the default configuration one launch per
    phase (a single bin), and a matrix with a row of more than 1536 products
    planned again on the binned path — both bit-exact."""
    A = csr.laplace2d(64)
    default = eng.get_config()["small_max_nnz"] > 0
    for task in ("AA", "AAt"):
        p = eng.plan(dev(A), task)
        if default:
            assert p.info["bins_used"] == 1 and p.info["heavy_rows"] == 0
        p.close()
        run_case(eng, A, task, "small/laplace64")
    # one dense row: 1,999 products in row 0
    n = 3000
    rows = [np.arange(n, dtype=np.int32)] + [np.array([i], np.int32) for i in range(1, n)]
    rows[0] = np.arange(0, n, 3, dtype=np.int32)
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    B = csr.CsrHost(n, rp, np.concatenate(rows),
                    np.random.default_rng(5).uniform(-1, 1, int(rp[-1])))
    for task in TASKS:
        run_case(eng, B, task, "small/fallback")


def strided(n, entries, step):
    """Row i holds columns i + step·c, c = −entries..entries, inside [0, n):
    C rows of 4·entries + 1 columns over a span of 4·entries·step."""
    rows = [np.array([i + step * c for c in range(-entries, entries + 1)
                      if 0 <= i + step * c < n], np.int32) for i in range(n)]
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    val = np.random.default_rng(n + step).uniform(-1, 1, int(rp[-1]))
    return csr.CsrHost(n, rp, np.concatenate(rows), val)


@pytest.mark.parametrize("words", [256, 512, 1024, 2048, -1])
def test_dense_bitmap_rows(words):
    """Rows over a bitmap of their output span (bitmap bins of up to 256, 512,
    1024 and 2048 words, or switched off): stencils, banded matrices, rows of
    far-apart columns (spans of 375 and 563 words) and a random graph (whose
    spans are too wide, so it stays on the hash tables), all tasks (the Gram
    path never takes the bitmap bins)."""
    from appt_spgemm_b200.engine import Engine
    cases = [(csr.stencil27(12, 5), "st12"), (csr.stencil27(30, 6), "st30"),
             (csr.banded(3000, 30, 0.3, 7), "band30"), (csr.banded(20000, 64, 0.3, 8), "band64"),
             (csr.uniform(4000, 40, seed=9), "uni40"), (csr.laplace2d(50), "lap50")]
    with Engine("cuda:0", small_max_nnz=-1, dense_max_words=words) as e:
        for A, lab in cases:
            for task in TASKS:
                run_case(e, A, task, f"dense{words}/{lab}")
        # 61 entries 100 or 150 columns apart: the 512- and 1024-word bins
        for A, lab in ((strided(30000, 30, 100), "far100"), (strided(30000, 30, 150), "far150")):
            for task in ("AA", "AAt"):
                run_case(e, A, task, f"dense{words}/{lab}")
        e.check_device_status()


@pytest.mark.parametrize("task", TASKS)
def test_stencil27_small(eng, task):
    run_case(eng, csr.stencil27(18, seed=2), task, "stencil27_18")


@pytest.mark.parametrize("task", TASKS)
def test_banded_and_er(eng, task):
    run_case(eng, csr.banded(5000, 40, 0.3, seed=4), task, "banded")
    run_case(eng, csr.erdos_renyi(6000, 20.0, seed=5), task, "er")


def test_edge_shapes(eng):
    cases = [
        csr.CsrHost(0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)),
        csr.CsrHost(1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([-2.5])),
        csr.CsrHost(1, np.array([0, 0], np.int32), np.zeros(0, np.int32), np.zeros(0)),
        csr.CsrHost(7, np.zeros(8, np.int32), np.zeros(0, np.int32), np.zeros(0)),
    ]
    n = 3000  # one dense row, one dense column, everything else empty
    rp = np.zeros(n + 1, np.int32)
    cols = []
    for i in range(n):
        c = list(range(n)) if i == 17 else ([17] if i % 3 == 0 else [])
        cols.extend(c)
        rp[i + 1] = len(cols)
    cases.append(csr.CsrHost(n, rp, np.array(cols, np.int32),
                             np.linspace(-1, 1, len(cols))))
    for k, A in enumerate(cases):
        for task in TASKS:
            run_case(eng, A, task, f"edge{k}")


def test_exact_cancellation_kept(eng):
    """Structural semantics: products that cancel to 0.0 stay as explicit
    entries (report/CORRECTNESS_NOTES.md:3-16)."""
    A = csr.CsrHost(2, np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32),
                    np.array([1.0, 1.0, 1.0, -1.0]))
    C = eng.multiply(dev(A), "AA")
    rp, ci, cx = C.to_host()
    assert list(rp) == [0, 2, 4] and list(ci) == [0, 1, 0, 1]
    assert list(cx) == [2.0, 0.0, 0.0, 2.0]


def test_invalid_csr_rejected_on_device(eng):
    from appt_spgemm_b200.engine import CsrDevice
    A = csr.laplace2d(8)
    bad = [A.col.copy(), A.col.copy(), A.col.copy()]
    bad[0][[1, 2]] = bad[0][[2, 1]]          # unsorted row
    bad[1][2] = bad[1][1]                    # duplicate column
    bad[2][-1] = 64                          # out of range
    for c in bad:
        M = CsrDevice(A.n, torch.from_numpy(A.rowptr).cuda(), torch.from_numpy(c).cuda(),
                      torch.from_numpy(A.val).cuda())
        for task in TASKS:
            with pytest.raises(SpgemmError) as e:
                eng.multiply(M, task)
            assert e.value.status == _capi.SPG_ERR_INVALID_CSR
    # row pointers out of range and decreasing (the one-readback plan runs its
    # kernels before it sees the verdict: they must stay inside the arrays)
    far, swapped = A.rowptr.copy(), A.rowptr.copy()
    far[3] = 10**6
    swapped[5], swapped[6] = swapped[6], swapped[5]
    for rp in (far, swapped):
        M = CsrDevice(A.n, torch.from_numpy(rp).cuda(), torch.from_numpy(A.col).cuda(),
                      torch.from_numpy(A.val).cuda())
        for task in TASKS:
            with pytest.raises(SpgemmError) as e:
                eng.multiply(M, task)
            assert e.value.status == _capi.SPG_ERR_INVALID_CSR
    with pytest.raises(SpgemmError):
        eng.multiply(dev(A), "AB")


def test_transpose_matches_oracle(eng):
    for A in (csr.rmat(12, 16, seed=8), csr.laplace2d(30), csr.uniform(1000, 40, seed=2)):
        T = eng.transpose(dev(A))
        torch.cuda.synchronize()
        O = oracle.transpose(A)
        assert np.array_equal(T.rowptr.cpu().numpy(), O.rowptr)
        assert np.array_equal(T.col.cpu().numpy(), O.col)
        assert np.array_equal(T.val.cpu().numpy(), O.val)


def test_transpose_path_selection(eng):
    """A·Aᵀ reuses A's pattern when it is structurally symmetric (values gathered)
    and runs the counting-sort transpose otherwise (the one-readback plan of a
    small A·Aᵀ always transposes: it does not wait for the pattern check); every
    path gives the oracle's C."""
    small = eng.get_config()["small_max_nnz"] > 0
    for A, sym in ((csr.laplace2d(20), 1), (csr.stencil27(7, seed=3), 1),
                   (csr.rmat(10, 8, seed=4), 0), (csr.uniform(500, 6, seed=5), 0)):
        for task in ("AAt", "AAtS"):
            p = eng.plan(dev(A), task)
            assert p.info["symmetric_pattern"] == (0 if small and task == "AAt" else sym)
            out = p.execute()
            torch.cuda.synchronize()
            assert_same(out, oracle.multiply(A, task), f"path{sym}/{task}")
            p.close()
    # one missing mirror entry forces the general path
    A = csr.laplace2d(12)
    keep = np.ones(A.nnz, bool)
    keep[7] = False
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))[keep]
    rp = np.zeros(A.n + 1, np.int32)
    np.cumsum(np.bincount(rows, minlength=A.n), out=rp[1:])
    B = csr.CsrHost(A.n, rp, A.col[keep].copy(), A.val[keep].copy())
    p = eng.plan(dev(B), "AAt")
    assert p.info["symmetric_pattern"] == 0
    out = p.execute()
    torch.cuda.synchronize()
    assert_same(out, oracle.multiply(B, "AAt"), "asymmetric-by-one")
    p.close()


def test_descriptors(eng):
    A = csr.rmat(11, 8, seed=6)
    d = eng.describe(dev(A))
    deg = np.diff(A.rowptr)
    assert d["products_aa"] == csr.products(A, "AA")
    assert d["products_aat"] == csr.products(A, "AAt")
    assert d["max_deg"] == deg.max()
    assert abs(d["deg_cv"] - deg.std() / deg.mean()) < 1e-9
    rows = np.repeat(np.arange(A.n), deg)
    assert d["bandwidth"] == np.abs(rows - A.col).max()
    S = A.to_scipy()
    P = S.copy()
    P.data[:] = 1
    sym = P.multiply(P.T).nnz / A.nnz
    assert abs(d["pattern_symmetry"] - sym) < 1e-12
    L = eng.describe(dev(csr.laplace2d(16)))
    assert L["pattern_symmetry"] == 1.0 and L["bandwidth"] == 16


def test_plan_execute_info_and_caller_buffers(eng):
    A = csr.erdos_renyi(5000, 10.0, seed=12)
    p = eng.plan(dev(A), "AA")
    ref = oracle.multiply(A, "AA")
    assert p.info["nnz_c"] == len(ref[1])
    assert p.info["products"] == csr.products(A, "AA")
    out = p.execute()
    torch.cuda.synchronize()
    assert_same(out, ref, "plan/execute")
    out2 = p.execute()  # a plan can execute again
    torch.cuda.synchronize()
    assert_same(out2, ref, "plan/execute twice")
    p.close()


def test_deterministic_repeats(eng):
    A = csr.rmat(12, 16, seed=9)
    first = None
    for _ in range(5):
        C = eng.multiply(dev(A), "AAt")
        torch.cuda.synchronize()
        h = C.to_host()
        if first is None:
            first = h
        else:
            for a, b in zip(first, h):
                assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_run_ours_record(golden, golden_dir):
    """spg_run_ours reproduces run_ours: nnz(C) and Σv, Σ|v|, Σv² (here bit-equal
    to the oracle's sequential checksum, since the values are)."""
    from appt_spgemm_b200.engine import run_ours
    A = csr.load_bin(os.path.join(golden_dir, "rmat_s9_ef8.csr"))
    d = dev(A)
    for task in TASKS:
        r = run_ours(task, d.rowptr, d.col, d.val, A.n, A.nnz, 3)
        cp, ci, cx = oracle.multiply(A, task)
        assert r.nnz == len(ci)
        assert (r.s, r.as_, r.sq) == oracle.checksum(cx)
        assert r.ms > 0


def test_cli_protocol(golden_dir):
    """The CLI prints the reference's __chk / RESULT lines (src/spgemm.cu:223-224),
    parsed here with the reference sweep's patterns (bench/run_compare.py:30-40)."""
    path = os.path.join(golden_dir, "banded_500_bw8.csr")
    A = csr.load_bin(path)
    for task in TASKS:
        out = subprocess.run([_capi.CLI_PATH, "banded", path, task, "2"], capture_output=True,
                             text=True, timeout=120, check=True).stdout
        chk = re.findall(r"__chk s=(\S+) as=(\S+) sq=(\S+)", out)
        res = [ln.split(",") for ln in out.splitlines() if ln.startswith("RESULT,")]
        assert len(chk) == 1 and len(res) == 1
        f = res[0]
        cp, ci, cx = oracle.multiply(A, task)
        assert f[1] == "banded" and f[2] == task and int(f[3]) == A.n and int(f[4]) == A.nnz
        assert int(f[5]) == len(ci) and float(f[6]) > 0
        s, a, q = oracle.checksum(cx)
        for got, want in zip(chk[0], (s, a, q)):
            assert abs(float(got) - want) <= 1e-6 * max(1.0, abs(want))


def test_stencil27_full_size_properties(eng):
    """The 27-point stencil on 96³ at full size, both products of the benchmark
    step: A·A and A·Aᵀ bit-exact against the oracle, nnz(C) equal to the
    5×5×5-stencil count, and the Gram path bit-identical to the plain A·Aᵀ."""
    A = csr.stencil27(96, seed=2)
    d = dev(A)
    s = np.array([3, 4] + [5] * 92 + [4, 3], dtype=np.int64)  # reachable offsets per axis
    want_nnz = int(s.sum()) ** 3
    assert want_nnz == 106496424
    for task in ("AA", "AAt"):
        C = eng.multiply(d, task)
        torch.cuda.synchronize()
        assert C.nnz == want_nnz, task
        assert_same(C, oracle.multiply(A, task, nthreads=0), f"stencil27_96/{task}")
        del C
    G = eng.multiply(d, "AAtS")
    P = eng.multiply(d, "AAt")
    torch.cuda.synchronize()
    assert G.nnz == P.nnz == want_nnz
    assert torch.equal(G.rowptr, P.rowptr) and torch.equal(G.col, P.col)
    assert torch.equal(G.val.view(torch.int64), P.val.view(torch.int64))


REF_ENGINE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                          "oracle", "_ref", "spgemm_ref")


def rel_ok(a, b, rt=1e-6):
    """The reference sweep's checksum tolerance (bench/run_compare.py:42-43)."""
    return abs(a - b) <= rt * max(1.0, abs(b))


@pytest.mark.parametrize("name", ["laplace2d_64", "stencil27_96"])
def test_against_reference_engine(eng, name, tmp_path):
    """The benchmark matrices through the reference's own CUDA engine
    (src/spgemm.cu, built unmodified into oracle/_ref/): nnz(C) equal and the
    three checksums within the reference's own tolerance, for every task,
    with the engine's C checksummed like the reference's run_ours does
    (src/spgemm_engine.cuh:116-118)."""
    if not os.path.exists(REF_ENGINE):
        pytest.skip("the reference engine was not built (oracle/Makefile REF=...)")
    A = csr.laplace2d(64) if name == "laplace2d_64" else csr.stencil27(96, seed=2)
    path = str(tmp_path / "a.csr")
    csr.write_bin(A, path)
    d = dev(A)
    for task in TASKS:
        out = subprocess.run([REF_ENGINE, name, path, task, "1"], capture_output=True, text=True,
                             timeout=600, check=True).stdout
        chk = re.findall(r"__chk s=(\S+) as=(\S+) sq=(\S+)", out)
        res = [ln.split(",") for ln in out.splitlines() if ln.startswith("RESULT,")]
        assert len(chk) == 1 and len(res) == 1, out
        C = eng.multiply(d, task)
        torch.cuda.synchronize()
        assert C.nnz == int(res[0][5]), f"{name}/{task}: nnz {C.nnz} vs {res[0][5]}"
        ours = oracle.checksum(C.val.cpu().numpy())
        for got, want in zip(ours, (float(x) for x in chk[0])):
            assert rel_ok(got, want), f"{name}/{task}: checksum {got} vs reference {want}"
        del C


def prune(ref):
    """The oracle's product with exact zeros removed (scipy's eliminate_zeros)."""
    rp, ci, cx = ref
    keep = cx != 0.0
    ck = np.concatenate([[0], np.cumsum(keep)]).astype(np.int64)
    return ck[rp], ci[keep], cx[keep]


def signed_ones(A, seed):
    """A's pattern with values ±1: products of such matrices cancel often."""
    rng = np.random.default_rng(seed)
    return csr.CsrHost(A.n, A.rowptr, A.col, rng.choice([-1.0, 1.0], A.nnz))


@pytest.mark.parametrize("task", TASKS)
def test_drop_zeros_matches_pruned_oracle(eng, task):
    """The numeric-zero switch leaves exactly the entries scipy keeps, also
    when the product is compacted through several row chunks."""
    cases = [signed_ones(csr.stencil27(14, 1), 3), signed_ones(csr.rmat(12, 8, seed=4), 5),
             csr.CsrHost(2, np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32),
                         np.array([1.0, 1.0, 1.0, -1.0])),
             csr.laplace2d(30)]
    for k, A in enumerate(cases):
        C = eng.multiply(dev(A), task)
        before = C.nnz
        eng.drop_zeros(C)
        torch.cuda.synchronize()
        ref = prune(oracle.multiply(A, task))
        assert_same(C, ref, f"drop_zeros{k}/{task}")
        assert C.nnz <= before
        eng.drop_zeros(C)  # idempotent
        torch.cuda.synchronize()
        assert_same(C, ref, f"drop_zeros{k}/{task}/again")


def test_drop_zeros_multi_chunk(eng):
    """A product of ±1 values with 42.9M entries: more than one 2^25-entry
    compaction chunk, about a third of the values exactly zero."""
    A = signed_ones(csr.stencil27(70, 1), 9)
    C = eng.multiply(dev(A), "AA")
    eng.drop_zeros(C)
    torch.cuda.synchronize()
    ref = prune(oracle.multiply(A, "AA"))
    assert C.nnz < len(oracle.multiply(A, "AA")[1])
    assert_same(C, ref, "drop_zeros/stencil70")
