"""The request server: every result equals its standalone product (and the
oracle) bit for bit while requests of different sizes run concurrently and
small ones are merged into batches; the memory budget rejects what can never
fit and holds back what does not fit yet."""
import time

import numpy as np
import pytest

import oracle
from appt_spgemm_b200 import _capi, csr

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(A):
    from appt_spgemm_b200.engine import CsrDevice
    return CsrDevice.from_host(A, "cuda:0")


def request_mix():
    mats = [csr.laplace2d(20), csr.uniform(800, 6, 1), csr.banded(3000, 9, 0.3, 2),
            csr.erdos_renyi(2000, 8.0, 3), csr.stencil27(30, 4), csr.rmat(13, 16, seed=5),
            csr.laplace2d(300), csr.banded(1500, 30, 0.3, 6)]
    mats += csr.batch_mix(10, seed=7, n_min=300, n_max=5000)[0]
    tasks = ["AA" if i % 2 == 0 else ("AAt" if i % 4 == 1 else "AAtS") for i in range(len(mats))]
    return mats, tasks


def test_server_results_equal_standalone_and_oracle():
    from appt_spgemm_b200.engine import Engine, Server
    mats, tasks = request_mix()
    ds = [dev(A) for A in mats]
    with Server(workers=3, batch_rows=8192, batch_max=8) as srv:
        ids = [srv.submit(d, t) for d, t in zip(ds, tasks)]
        infos = [srv.wait(i, timeout_ms=120000) for i in ids]
        assert all(inf["status"] == _capi.SPG_OK for inf in infos)
        st = srv.stats()
        assert st["completed"] == len(mats) and st["rejected"] == 0
        assert st["batches"] >= 1 and any(inf["batched"] for inf in infos)
        assert st["p99_ms"] >= st["p50_ms"] > 0
        for inf in infos:
            assert inf["submit_ms"] <= inf["start_ms"] <= inf["planned_ms"] <= inf["run_ms"]
            assert inf["run_ms"] <= inf["done_ms"]
        with Engine("cuda:0") as eng:
            for i, (A, d, t, rid) in enumerate(zip(mats, ds, tasks, ids)):
                got = srv.result(rid)
                alone = eng.multiply(d, t)
                torch.cuda.synchronize()
                g, a = got.to_host(), alone.to_host()
                o = oracle.multiply(A, t)
                for x, y, z in zip(g, a, o):
                    assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), (i, t)
                    assert np.array_equal(x.view(np.uint8), np.ascontiguousarray(z).view(np.uint8))
                srv.release(rid)
        assert srv.stats()["reserved_bytes"] == 0


def test_server_budget_rejects_and_holds_back():
    from appt_spgemm_b200.engine import Server
    big = csr.stencil27(40, 8)            # output ~ 14 MB
    small = csr.laplace2d(30)             # output ~ 28 KB
    out_big = 8 * (big.n + 1) + 12 * len(oracle.multiply(big, "AA")[1])
    # a budget below the big request's output: it is rejected, the small one runs
    with Server(workers=2, memory_budget_bytes=out_big // 2, batch_rows=1) as srv:
        rb = srv.submit(dev(big), "AA")
        rs = srv.submit(dev(small), "AA")
        assert srv.wait(rb, 60000)["status"] == _capi.SPG_ERR_BUDGET
        assert srv.wait(rs, 60000)["status"] == _capi.SPG_OK
        assert srv.stats()["rejected"] == 1
    # a budget that holds one big result at a time: the second waits for a release
    with Server(workers=2, memory_budget_bytes=int(out_big * 1.6), batch_rows=1) as srv:
        d = dev(big)
        r1 = srv.submit(d, "AA")
        assert srv.wait(r1, 60000)["status"] == _capi.SPG_OK
        r2 = srv.submit(d, "AA")
        with pytest.raises(_capi.SpgemmError) as e:
            srv.wait(r2, timeout_ms=1500)
        assert e.value.status == _capi.SPG_ERR_TIMEOUT
        srv.release(r1)
        assert srv.wait(r2, 60000)["status"] == _capi.SPG_OK
        assert srv.stats()["peak_reserved_bytes"] <= int(out_big * 1.6)


def test_small_requests_pass_a_large_one_waiting_for_budget():
    """A large request that does not fit the budget yet waits, planned, while
    the workers (and the small-request lane) keep serving small requests; it
    runs once the client releases the result that holds the budget."""
    from appt_spgemm_b200.engine import Server
    big = csr.rmat(15, 16, seed=11)               # n = 32768 >= batch_rows below: a large request
    out_big = 8 * (big.n + 1) + 12 * len(oracle.multiply(big, "AA")[1])
    smalls = [csr.laplace2d(20 + i) for i in range(12)]
    with Server(workers=3, memory_budget_bytes=int(out_big * 1.5), batch_rows=4096,
                batch_max=4) as srv:
        d = dev(big)
        r1 = srv.submit(d, "AA")
        assert srv.wait(r1, 60000)["status"] == _capi.SPG_OK
        r2 = srv.submit(d, "AA")                 # cannot fit until r1 is released
        ids = [srv.submit(dev(A), "AA") for A in smalls]
        for A, rid in zip(smalls, ids):
            info = srv.wait(rid, 60000)
            assert info["status"] == _capi.SPG_OK
            g = srv.result(rid).to_host()
            o = oracle.multiply(A, "AA")
            for x, z in zip(g, o):
                assert np.array_equal(x.view(np.uint8), np.ascontiguousarray(z).view(np.uint8))
            srv.release(rid)
        assert srv.poll(r2)["status"] == _capi.SPG_ERR_NOT_READY
        srv.release(r1)
        assert srv.wait(r2, 60000)["status"] == _capi.SPG_OK
        g = srv.result(r2).to_host()
        o = oracle.multiply(big, "AA")
        for x, z in zip(g, o):
            assert np.array_equal(x.view(np.uint8), np.ascontiguousarray(z).view(np.uint8))
        srv.release(r2)
        assert srv.stats()["rejected"] == 0


def test_batch_over_budget_is_split_into_requests():
    """Small requests merged into a batch whose outputs together exceed the
    budget are split and run one by one, each within the budget."""
    from appt_spgemm_b200.engine import Server
    mats = [csr.stencil27(30, 20 + i) for i in range(4)]
    out = 8 * (mats[0].n + 1) + 12 * len(oracle.multiply(mats[0], "AA")[1])
    ds = [dev(A) for A in mats]
    with Server(workers=1, memory_budget_bytes=int(out * 2.5), batch_rows=1 << 20,
                batch_max=8) as srv:
        ids = [srv.submit(d, "AA") for d in ds]
        for A, rid in zip(mats, ids):
            info = srv.wait(rid, 60000)
            assert info["status"] == _capi.SPG_OK
            assert not info["batched"]
            g = srv.result(rid).to_host()
            o = oracle.multiply(A, "AA")
            for x, z in zip(g, o):
                assert np.array_equal(x.view(np.uint8), np.ascontiguousarray(z).view(np.uint8))
            srv.release(rid)
        assert srv.stats()["rejected"] == 0


@pytest.mark.timeout(120, method="thread")
def test_close_with_a_request_waiting_for_budget():
    """Closing the server while a planned request still waits for budget
    ends that request with an error status instead of hanging."""
    from appt_spgemm_b200.engine import Server
    big = csr.stencil27(40, 8)
    out_big = 8 * (big.n + 1) + 12 * len(oracle.multiply(big, "AA")[1])
    srv = Server(workers=2, memory_budget_bytes=int(out_big * 1.6), batch_rows=1)
    d = dev(big)
    r1 = srv.submit(d, "AA")
    assert srv.wait(r1, 60000)["status"] == _capi.SPG_OK
    r2 = srv.submit(d, "AA")
    with pytest.raises(_capi.SpgemmError):
        srv.wait(r2, timeout_ms=1000)
    srv.close()


def workspace_bound(eng, As, task, batched):
    import ctypes
    from appt_spgemm_b200._capi import SpgCsrDev, check, lib
    arr = (SpgCsrDev * len(As))(*[A.struct() for A in As])
    out = ctypes.c_int64()
    check(lib().spg_plan_workspace_bound(eng._h, _capi.TASKS[task], len(As), arr,
                                         1 if batched else 0, ctypes.byref(out)), "bound")
    return out.value


def test_plan_workspace_bound_covers_every_plan():
    """The host-side bound a budgeted caller reserves before planning is at
    least the workspace the plan then holds, single and batched, for every
    task, heavy rows and the windowed heavy kernel included."""
    from appt_spgemm_b200.engine import Engine
    mats, _ = request_mix()
    mats = mats + [csr.erdos_renyi(1 << 14, 80.0, 9), csr.rmat(14, 16, seed=11)]
    with Engine("cuda:0") as eng:
        ds = [dev(A) for A in mats]
        for task in ("AA", "AAt", "AAtS"):
            for d in ds:
                p = eng.plan(d, task)
                assert workspace_bound(eng, [d], task, False) >= p.info["workspace_bytes"], task
                p.close()
            p = eng.plan_batched(ds[:6], task)
            assert workspace_bound(eng, ds[:6], task, True) >= p.info["workspace_bytes"], task
            p.close()


def test_server_holds_at_most_its_budget():
    """Several large requests at once under a budget of about two and a half of
    them: plans are only made once their workspace bound is reserved, a job
    that cannot run yet holds nothing, so the bytes the server actually holds
    (plans, execute workspace, results) never exceed the budget; every request
    still completes, equal to its standalone product."""
    from appt_spgemm_b200.engine import Engine, Server
    big = csr.stencil27(40, 8)
    d = dev(big)
    with Engine("cuda:0") as eng:
        p = eng.plan(d, "AA")
        need = (p.info["workspace_bytes"] + p.info["exec_workspace_bytes"] +
                p.info["output_bytes"])
        bound = workspace_bound(eng, [d], "AA", False)
        p.close()
        alone = eng.multiply(d, "AA").to_host()
    budget = int(max(need, bound) * 2.5)
    with Server(workers=3, memory_budget_bytes=budget, batch_rows=1) as srv:
        ids = [srv.submit(d, "AA") for _ in range(6)]
        # results are checked and released as they complete: the workers may
        # finish requests out of submission order, and a client that kept later
        # results while waiting for an earlier one could hold the budget that
        # the earlier one needs
        pending, deadline = set(ids), time.time() + 120
        while pending:
            assert time.time() < deadline, f"requests {sorted(pending)} did not complete"
            for rid in sorted(pending):
                info = srv.poll(rid)
                if info["status"] == _capi.SPG_ERR_NOT_READY:
                    continue
                assert info["status"] == _capi.SPG_OK
                got = srv.result(rid).to_host()
                for x, y in zip(got, alone):
                    assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
                srv.release(rid)
                pending.discard(rid)
            time.sleep(0.001)
        st = srv.stats()
        assert st["completed"] == 6 and st["rejected"] == 0
        assert 0 < st["peak_held_bytes"] <= budget
        assert st["peak_held_bytes"] <= st["peak_reserved_bytes"] <= budget
        assert st["held_bytes"] == 0 and st["reserved_bytes"] == 0
