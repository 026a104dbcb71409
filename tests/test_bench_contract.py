"""The benchmark's reference arm (the CPU oracle on the host cores) prints the
one JSON line its callers parse: the contract keys, an end-to-end block with
no host↔device bytes, and nothing at all from ranks other than 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--steps", "3", "--warmup", "3", "--cpu-seconds", "0.5"]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_the_contract_line():
    p = run_bench()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["unit"] == "GFLOP/s" and d["higher_is_better"] is True
    assert d["dtype"] == "f64"
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["cores"] >= 1 and cb["kind"] in ("port", "reference") and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_loads_no_engine_code_and_keeps_the_config():
    """The reference arm maps only the oracle's library (never the engine's),
    and its config is the one the GPU arm prints for the same workload."""
    import types

    import bench
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', "
            "'--warmup', '3']; runpy.run_path('bench.py', run_name='__main__'); "
            "print(open('/proc/self/maps').read(), file=sys.stderr)")
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "liboracle.so" in p.stderr
    assert "libspgemm_b200" not in p.stderr
    d = json.loads(p.stdout.strip().splitlines()[-1])
    side = 96
    A = types.SimpleNamespace(n=side ** 3, nnz=(3 * side - 2) ** 3)
    args = types.SimpleNamespace(side=side, gpus=1)
    assert d["config"] == json.loads(json.dumps(bench.config(args, A)))
    assert "every row" in d["cpu_baseline"]["sample"]


def test_reference_arm_other_ranks_print_nothing():
    p = run_bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def run_entry(rate, server, p50, gflops, small=None):
    return {"rate_per_s": rate, "server": server, "requests": 10, "completed": 10,
            "rejected": 0, "failed": 0, "batches": 1, "small_requests": 4,
            "p50_ms": p50, "p99_ms": 2 * p50, "small_p50_ms": small, "small_p99_ms": small,
            "sustained_gflops": gflops, "peak_reserved_gb": 1.0}


def test_serve_aggregation_one_stream_is_that_stream():
    import bench
    r = run_entry(50.0, "queue_only", 120.0, 40.0, small=5.0)
    a = bench.aggregate_serve([r])
    for k, v in r.items():
        assert a[k] == v, k
    assert a["streams"] == 1 and "p50_ms_range" not in a


def test_serve_aggregation_medians_ranges_and_sums():
    import bench
    runs = [run_entry(500.0, "continuous_batching", p, g, small=s)
            for p, g, s in ((300.0, 50.0, None), (100.0, 70.0, 8.0), (200.0, 60.0, 2.0))]
    a = bench.aggregate_serve(runs)
    assert a["p50_ms"] == 200.0 and a["p50_ms_range"] == [100.0, 300.0]
    assert a["sustained_gflops"] == 60.0 and a["sustained_gflops_range"] == [50.0, 70.0]
    # a figure missing from a stream (no small requests there) is left out
    assert a["small_p50_ms"] == 5.0 and a["small_p50_ms_range"] == [2.0, 8.0]
    assert a["requests"] == 30 and a["completed"] == 30 and a["batches"] == 3
    assert a["streams"] == 3
    even = bench.aggregate_serve(runs[:2])
    assert even["p50_ms"] == 200.0 and even["sustained_gflops"] == 60.0


def test_serve_loop_runs_a_stream_through_a_server(monkeypatch):
    """The serving loop's host side: every request is submitted at its arrival
    time, polled to completion and released, and the entry counts them."""
    import time
    import types

    import numpy as np

    import bench
    from appt_spgemm_b200 import _capi, engine

    class FakeServer:
        def __init__(self, memory_budget_bytes=0, workers=1, batch_rows=1, batch_max=1):
            self.t0 = time.perf_counter()
            self.submitted = {}
            self.released = set()
            FakeServer.last = self

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def submit(self, A, task):
            rid = len(self.submitted) + 1
            self.submitted[rid] = ((time.perf_counter() - self.t0) * 1e3, task)
            return rid

        def poll(self, rid):
            sub = self.submitted[rid][0]
            return {"status": _capi.SPG_OK, "submit_ms": sub, "done_ms": sub + 1.0 + rid % 3}

        def release(self, rid):
            self.released.add(rid)

        def stats(self):
            return {"rejected": 0, "failed": 0, "batches": 0, "peak_reserved_bytes": 5e8}

    monkeypatch.setattr(engine, "Server", FakeServer)
    pool = [(types.SimpleNamespace(n=1000), "small"), (types.SimpleNamespace(n=100000), "large")]
    prods = {(i, t): 1000 * (i + 1) for i in range(2) for t in ("AA", "AAt")}
    picks = np.array([0, 1, 0, 1, 0])
    tasks = np.array(["AA", "AAt", "AA", "AA", "AAt"])
    gaps = np.full(5, 0.002)
    r = bench.serve_once(pool, [None, None], prods, 500.0, "continuous_batching", {},
                         picks, tasks, gaps)
    assert r["requests"] == 5 and r["completed"] == 5 and r["small_requests"] == 3
    assert r["rate_per_s"] == 500.0 and r["server"] == "continuous_batching"
    assert FakeServer.last.released == {1, 2, 3, 4, 5}
    assert [t for _, t in FakeServer.last.submitted.values()] == list(tasks)
    assert r["p50_ms"] >= 1.0 and r["sustained_gflops"] > 0
    assert r["peak_reserved_gb"] == 0.5


def test_single_matrix_workloads():
    """The matrices of --mode laplace / rmat: the 5-point Laplacian 64² of the
    small plain configuration (n 4,096, nnz 20,224, 100,104 products), R-MAT and
    Erdős–Rényi at the requested scale."""
    import types

    import bench
    from appt_spgemm_b200 import csr

    args = types.SimpleNamespace(mode="laplace", laplace_side=64, rmat_scale=10, er_degree=0.0)
    A, desc, label = bench.single_matrix(args)
    assert (A.n, A.nnz) == (4096, 20224) and csr.products(A, "AA") == 100104
    assert "Laplacian" in desc and label == "2-D 5-point Laplacian"
    args.mode = "rmat"
    A, desc, label = bench.single_matrix(args)
    assert A.n == 1024 and label == "power-law graph" and "R-MAT scale 10" in desc
    args.er_degree = 8.0
    A, desc, label = bench.single_matrix(args)
    assert A.n == 1024 and label == "random graph"


def test_serve_pool_follows_its_recipe():
    """The serving pool: each matrix one of the three families, its size from
    n log-uniform in [2k, 2M] rounded to the family's shape (grid side or
    R-MAT scale), and the pool fixed by its seed."""
    import re

    import bench
    pool = bench.serve_pool(12, seed=5)
    assert len(pool) == 12
    for A, desc in pool:
        A.validate()
        m = re.fullmatch(r"(laplace2d|stencil27|rmat) (\d+)\^(\d+)", desc)
        assert m, desc
        fam, base, exp = m.group(1), int(m.group(2)), int(m.group(3))
        assert A.n == base ** exp
        assert 2000 <= A.n <= 2 ** 21  # rounding of the side or scale can pass 2M a little
        assert (fam == "rmat") == (base == 2)
    first = bench.serve_pool(3, seed=5)
    assert [d for _, d in first] == [d for _, d in pool[:3]]
    assert all(a.nnz == b.nnz for (a, _), (b, _) in zip(first, pool))


def test_serve_streams_are_seeded_per_rate_and_stream():
    """Every arrival stream comes from (55, rate index, stream): the same
    arguments give the same requests, the rate changes only the gaps (so the
    back-to-back leg replays the first rate's first stream exactly), and the
    tasks are A·A / A·Aᵀ with the gaps' mean near 1 / rate."""
    import numpy as np

    import bench
    p1, t1, g1 = bench.serve_stream(0, 0, 2000, 40, 500.0)
    p2, t2, g2 = bench.serve_stream(0, 0, 2000, 40, 1.0)
    assert np.array_equal(p1, p2) and np.array_equal(t1, t2)
    assert np.allclose(g2, g1 * 500.0)
    assert set(np.unique(t1)) == {"AA", "AAt"} and 0.4 < np.mean(t1 == "AA") < 0.6
    assert p1.min() >= 0 and p1.max() < 40
    assert abs(np.mean(g1) * 500.0 - 1.0) < 0.1
    p3, _, _ = bench.serve_stream(1, 0, 2000, 40, 500.0)
    p4, _, _ = bench.serve_stream(0, 1, 2000, 40, 500.0)
    assert not np.array_equal(p1, p3) and not np.array_equal(p1, p4)
