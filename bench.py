#!/usr/bin/env python3
"""SpGEMM benchmark: GFLOP/s (2 × intermediate products / s) of C = A·A and
C = A·Aᵀ on one B200, with the roofline of the dominant kernel, the CPU oracle
timed on the host cores, cuSPARSE on the same GPU, and an end-to-end number
through the public API with host buffers.

Workload: the 3-D 27-point stencil on a 96³ grid (n = 884,736, nnz = 23.4M,
values uniform(−1,1) from a seed), structurally symmetric, numerically
unsymmetric; one step = one A·A plus one A·Aᵀ (through Aᵀ; the Gram path,
which gives the same C, is timed per call beside the line).
Inputs (284 MB) and outputs (2 × 1.3 GB) exceed the 126 MB L2, so no flush
is needed between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: the product has no exchange step, so N GPUs run N independent
replicas (weak scaling); the time is the max over ranks.  --impl reference
times the CPU oracle (the reference's algorithm, restated) on the host cores.

Other workloads, one GPU each: --mode rmat (R-MAT 2^20, heavy rows; or an
Erdős–Rényi graph with --er-degree), --mode laplace (the 2-D 5-point
Laplacian 64², microseconds per call), --mode batch (512 matrices in one
batched product and in graph replay against back-to-back calls), --mode serve
(Poisson request streams through the request server and a one-worker queue;
--serve-seeds repeats each rate over several streams).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIDE = 96
SEED = 2
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC = os.path.join(ROOT, "profiles", "ncu_traffic.json")
FALLBACK_HBM_GBS = 6650.0
METRIC = "GFLOP/s (2×intermediate products/s) A·A & A·Aᵀ"


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--side", type=int, default=SIDE, help="stencil grid side (96 = the benchmark)")
    ap.add_argument("--aat-task", default="AAt", choices=["AAt", "AAtS"],
                    help="engine task used for A·Aᵀ (AAt: the product through Aᵀ, the faster "
                         "path on this matrix; AAtS: the Gram path, upper triangle + mirror, "
                         "also timed beside the line)")
    ap.add_argument("--no-baselines", action="store_true",
                    help="skip the CPU oracle, cuSPARSE and reference-GPU baselines")
    ap.add_argument("--no-sub", action="store_true",
                    help="skip the sub-results of the default line (the 5-point Laplacian 64^2 "
                         "per call and the 512-matrix batch)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU work of the oracle baseline sample")
    ap.add_argument("--mode", choices=["plain", "rmat", "laplace", "batch", "serve"],
                    default="plain",
                    help="plain: the headline stencil benchmark; rmat: the power-law graph "
                         "(R-MAT 2^20, heavy rows); laplace: the 2-D 5-point Laplacian "
                         "(64^2, launch-latency-bound: µs per call); batch: 512 matrices in one "
                         "batched product vs back-to-back calls; serve: Poisson request stream")
    ap.add_argument("--laplace-side", type=int, default=64,
                    help="grid side of --mode laplace")
    ap.add_argument("--rmat-scale", type=int, default=20, help="R-MAT scale of --mode rmat")
    ap.add_argument("--er-degree", type=float, default=0.0,
                    help="--mode rmat on an Erdős–Rényi graph of n = 2^scale with this mean "
                         "degree instead (heavy rows fed by short B rows)")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--serve-requests", type=int, default=300,
                    help="requests per arrival rate in --mode serve")
    ap.add_argument("--serve-rates", default="50,500,5000")
    ap.add_argument("--serve-pool", type=int, default=40, help="distinct matrices in the pool")
    ap.add_argument("--serve-workers", type=int, default=0,
                    help="workers of the continuous-batching server (0: its default)")
    ap.add_argument("--serve-seeds", type=int, default=1,
                    help="arrival streams per rate in --mode serve (each run through both "
                         "servers); figures are medians over the streams")
    return ap.parse_args()


def workload(side):
    from appt_spgemm_b200 import csr
    A = csr.stencil27(side, seed=SEED)
    return A, csr.products(A, "AA"), csr.products(A, "AAt")


def config(args, A, extra=None):
    c = {"workload": f"27-point stencil {args.side}^3 (n={A.n}, nnz={A.nnz}), FP64, "
                     f"one step = A·A + A·Aᵀ",
         "matrix": "stencil27", "grid_side": args.side, "n": A.n, "nnz": A.nnz,
         "tasks": ["AA", "AAt"], "index": "int32 in / int64 C rowptr", "values": "fp64",
         "l2": "inputs (284 MB) and outputs (2.6 GB) exceed L2; no flush needed",
         "parallelism": f"replicas x{args.gpus}"}
    if extra:
        c.update(extra)
    return c


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [ln.split(",") for ln in open(self.path).read().strip().splitlines()]
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for name, flag in zip(names, r[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx),
                       reasons=sorted(reasons), samples=len(sm))
        try:
            os.unlink(self.path)
        except Exception:
            pass
        return out


# ---------------------------------------------------------------------------
# CPU baselines (the oracle: test infrastructure, timed here as the baseline)
# ---------------------------------------------------------------------------
def row_products(A, B):
    import numpy as np
    deg_b = np.diff(B.rowptr).astype(np.int64)
    per_entry = deg_b[A.col]
    cs = np.concatenate([[0], np.cumsum(per_entry)])
    return cs[A.rowptr[1:]] - cs[A.rowptr[:-1]]


def cpu_oracle_rate(A, seconds, nthreads, label_rows=None):
    """Time the oracle on leading row blocks of A·A and A·Aᵀ for about
    `seconds`; returns (GFLOP/s, products timed, description)."""
    import numpy as np

    import oracle
    B_t = A.transpose()
    total_products = 0
    total_time = 0.0
    parts = []
    for task, B in (("AA", A), ("AAt", B_t)):
        f = row_products(A, B)
        budget = seconds / 2
        r0, r = 0, 256
        while r0 < A.n and budget > 0:
            r1 = min(A.n, r0 + r)
            t0 = time.perf_counter()
            oracle.rows_stream(A, B, r0, r1, nthreads)
            dt = time.perf_counter() - t0
            total_time += dt
            total_products += int(f[r0:r1].sum())
            budget -= dt
            rate = (r1 - r0) / max(dt, 1e-6)
            r0 = r1
            r = int(max(256, min(rate * min(budget, 2.0), A.n)))
        parts.append(f"{task}: rows [0, {r0}) of {A.n}")
    gflops = 2.0 * total_products / total_time / 1e9
    return gflops, total_products, total_time, "; ".join(parts)


def run_reference(args):
    """--impl reference: the reference's algorithm on the host cores (the CPU
    oracle restating it, all threads), same workload, metric and config.  Each
    step computes every row of A·A and of A·Aᵀ.  This arm loads no engine code:
    the stencil comes from the oracle's own generator (byte-identical to the
    engine's) and Aᵀ from the oracle's transpose."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    A = oracle.gen_stencil27(args.side, SEED)
    B_t = oracle.transpose(A)
    nthreads = os.cpu_count() or 1
    f_aa, f_aat = row_products(A, A), row_products(A, B_t)
    prods = int(f_aa.sum() + f_aat.sum())
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.rows_stream(A, A, 0, A.n, nthreads)
        oracle.rows_stream(A, B_t, 0, A.n, nthreads)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
    gflops = 2.0 * prods * len(times) / sum(times) / 1e9
    sample = (f"every row of A·A and of A·Aᵀ each step ({A.n} rows, {prods} products per "
              f"step, {nthreads} threads)")
    line = {"metric": METRIC, "value": round(gflops, 3),
            "unit": "GFLOP/s", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * statistics.mean(times), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator)",
            "config": config(args, A),
            "cpu_baseline": {"value": round(gflops, 3), "unit": "GFLOP/s", "cores": nthreads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(gflops, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU baselines outside the timed region: cuSPARSE, the reference's CUDA engine
# ---------------------------------------------------------------------------
def cusparse_baseline(dA, A, p_aa, p_aat, reps=5):
    import ctypes

    from appt_spgemm_b200 import _capi
    try:
        L = ctypes.CDLL(_capi.CUSPARSE_LIB_PATH)
    except OSError as e:
        return {"error": str(e)}
    fn = L.spgb_cusparse_time
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                   ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                   ctypes.POINTER(ctypes.c_longlong),
                   ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_int]
    out = {}
    for task, tid, prods in (("AA", 0, p_aa), ("AAt", 1, p_aat)):
        mean, mn, med = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        nnz = ctypes.c_longlong()
        chk = (ctypes.c_double * 3)()
        err = ctypes.create_string_buffer(256)
        rc = fn(tid, dA.rowptr.data_ptr(), dA.col.data_ptr(), dA.val.data_ptr(), A.n, A.nnz, reps, 2,
                ctypes.byref(mean), ctypes.byref(mn), ctypes.byref(med), ctypes.byref(nnz), chk,
                err, 256)
        if rc != 0:
            out[task] = {"error": err.value.decode()}
        else:
            out[task] = {"ms_mean": round(mean.value, 4), "ms_min": round(mn.value, 4),
                         "ms_median": round(med.value, 4),
                         "nnz_c": nnz.value,
                         "gflops": round(2.0 * prods / (mean.value * 1e-3) / 1e9, 3)}
    return out


def reference_gpu_baseline(A, p_aa, p_aat, reps=5):
    """The reference's own CUDA engine (src/spgemm.cu built unmodified for sm_80,
    JIT-run on the B200) on a CSR1 file of the same matrix, `reps` timed calls
    (its RESULT line reports their mean)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "spgemm_ref")
    if not os.path.exists(exe):
        return {"error": "reference engine binary not built"}
    from appt_spgemm_b200 import csr
    out = {}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "a.csr")
        csr.write_bin(A, path)
        for task, prods in (("AA", p_aa), ("AAt", p_aat), ("AAtS", p_aat)):
            try:
                r = subprocess.run([exe, "bench", path, task, str(reps)], capture_output=True, text=True,
                                   timeout=300)
                res = [ln.split(",") for ln in r.stdout.splitlines() if ln.startswith("RESULT,")]
                if r.returncode != 0 or not res:
                    out[task] = {"error": (r.stderr or r.stdout).strip()[-200:]}
                    continue
                ms = float(res[0][6])
                out[task] = {"ms_mean": ms, "nnz_c": int(res[0][5]),
                             "gflops": round(2.0 * prods / (ms * 1e-3) / 1e9, 3)}
            except subprocess.TimeoutExpired:
                out[task] = {"error": "timeout"}
    return out


# ---------------------------------------------------------------------------
# single matrices timed per call: the power-law graph R-MAT 2^20 (edge factor
# 16, (.57,.19,.19,.05), seed 3), an Erdős–Rényi graph, or the 2-D 5-point
# Laplacian 64^2
# ---------------------------------------------------------------------------
def single_matrix(args):
    """The matrix of --mode rmat / laplace: (A, description, metric label)."""
    from appt_spgemm_b200 import csr
    if args.mode == "laplace":
        A = csr.laplace2d(args.laplace_side)
        return A, (f"2-D 5-point Laplacian {args.laplace_side}^2 (n={A.n}, nnz={A.nnz}), 4.0 "
                   "diagonal, -1.0 neighbours"), "2-D 5-point Laplacian"
    if args.er_degree > 0:
        A = csr.erdos_renyi(1 << args.rmat_scale, args.er_degree, seed=3)
        return A, (f"Erdős–Rényi n=2^{args.rmat_scale} (n={A.n}, nnz={A.nnz}), mean degree "
                   f"{args.er_degree:g}, seed 3"), "random graph"
    A = csr.rmat(args.rmat_scale, 16, seed=3)
    return A, (f"R-MAT scale {args.rmat_scale} (n={A.n}, nnz={A.nnz}), edge factor 16, "
               "(a,b,c,d)=(.57,.19,.19,.05), seed 3, duplicates merged, self-loops kept, "
               "values uniform(0,1)"), "power-law graph"


def run_rmat(args):
    import torch

    from appt_spgemm_b200 import csr
    from appt_spgemm_b200.engine import CsrDevice, Engine

    t0 = time.time()
    A, graph, label = single_matrix(args)
    gen_s = time.time() - t0
    prods = {"AA": csr.products(A, "AA"), "AAt": csr.products(A, "AAt")}
    n, nnz = A.n, A.nnz
    dA = CsrDevice.from_host(A, "cuda:0")
    eng = Engine("cuda:0")
    stream = torch.cuda.current_stream()
    peak, peak_kind = hbm_peak()
    tasks = {}
    kernels = {}
    with ClockSampler(0) as clocks:
        for task in ("AA", "AAt"):
            plan = eng.plan(dA, task)
            info = dict(plan.info)
            plan.close()
            for _ in range(max(args.warmup, 0)):
                C = eng.multiply(dA, task)
                torch.cuda.synchronize()
                del C
            eng.profile_reset()
            eng.profile_enable(True)
            ts = []
            for _ in range(max(args.steps, 1)):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                C = eng.multiply(dA, task)
                e1.record(stream)
                torch.cuda.synchronize()
                del C
                ts.append(e0.elapsed_time(e1))
            eng.profile_enable(False)
            prof = eng.profile_read()
            ms = statistics.median(ts)
            alg = 4 * (n + 1) + 12 * nnz + 8 * (n + 1) + 12 * info["nnz_c"]
            tasks[task] = {"ms_median": round(ms, 3), "ms_mean": round(statistics.mean(ts), 3),
                           "us_per_call": round(ms * 1e3, 1),
                           "gflops": round(2.0 * prods[task] / (ms * 1e-3) / 1e9, 3),
                           "products": prods[task], "nnz_c": info["nnz_c"],
                           "heavy_rows": info["heavy_rows"],
                           "alg_bytes": int(alg),
                           "hbm_frac": round(alg / (ms * 1e-3) / 1e9 / peak, 4)}
            kernels[task] = {k: round(v["ms"] / len(ts), 3) for k, v in
                             sorted(prof["kernels"].items(), key=lambda kv: -kv[1]["ms"])[:8]}
            launches = int(prof.get("launches", 0))
    total_ms = tasks["AA"]["ms_median"] + tasks["AAt"]["ms_median"]
    value = 2.0 * (prods["AA"] + prods["AAt"]) / (total_ms * 1e-3) / 1e9
    top_label, top_ms = max(kernels["AA"].items(), key=lambda kv: kv[1])
    line = {"metric": "GFLOP/s (2×intermediate products/s) A·A & A·Aᵀ, " + label,
            "value": round(value, 3), "unit": "GFLOP/s", "mode": args.mode, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms, 3),
            "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": graph + "; one step = A·A + A·Aᵀ",
                       "generation_s": round(gen_s, 1),
                       "l2": ("inputs and C fit in L2: warm-cache calls, launch-latency-bound"
                              if args.mode == "laplace" else
                              "C exceeds L2 by far; no flush needed")},
            "tasks": tasks, "kernels_ms_per_call": kernels,
            "roofline": {"bound": "hbm", "kernel": "whole call (A·A)",
                         "achieved": round(tasks["AA"]["alg_bytes"] /
                                           (tasks["AA"]["ms_median"] * 1e-3) / 1e9, 1),
                         "peak": peak, "unit": "GB/s", "frac": tasks["AA"]["hbm_frac"],
                         "peak_source": peak_kind, "traffic": None,
                         "top_kernel": top_label, "top_kernel_share": round(
                             top_ms / tasks["AA"]["ms_median"], 3)},
            "gpu_launches_per_call": launches // max(args.steps, 1),
            "clocks": clocks.summary()}
    del dA
    eng.close()
    torch.cuda.empty_cache()
    if not args.no_baselines:
        big = max(t["nnz_c"] for t in tasks.values()) >= 2**31
        if big:
            why = ("not run: C has more than 2^31 - 1 entries, which cusparseSpGEMM's "
                   "32-bit CSR and the reference engine's int32 C row offsets "
                   "(src/spgemm_engine.cuh:91) cannot index")
            line["baselines"] = {"cusparse": {"unsupported": why},
                                 "reference_gpu_engine": {"unsupported": why}}
        else:
            dA = CsrDevice.from_host(A, "cuda:0")
            line["baselines"] = {"cusparse": cusparse_baseline(dA, A, prods["AA"], prods["AAt"]),
                                 "reference_gpu_engine": reference_gpu_baseline(
                                     A, prods["AA"], prods["AAt"])}
            del dA
        nthreads = os.cpu_count() or 1
        gf, p, secs, sample = cpu_oracle_rate(A, args.cpu_seconds, nthreads)
        line["cpu_baseline"] = {"value": round(gf, 3), "unit": "GFLOP/s", "cores": nthreads,
                                "kind": "port", "sample": sample + f" ({p} products, {secs:.1f} s)"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# batched products: 512 matrices, one batched plan vs back-to-back plain calls
# ---------------------------------------------------------------------------
def run_batch(args):
    import torch

    from appt_spgemm_b200 import csr
    from appt_spgemm_b200.engine import CsrDevice, Engine

    t0 = time.time()
    mats, params = csr.batch_mix(args.batch_count, seed=4)
    gen_s = time.time() - t0
    prods = sum(csr.products(A, "AA") for A in mats)
    ds = [CsrDevice.from_host(A, "cuda:0") for A in mats]
    eng = Engine("cuda:0")
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            a, b = ev(), ev()
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.median(ms)

    def back_to_back():
        for d in ds:
            eng.multiply(d, "AA")

    reps = max(1, min(args.steps, 3))
    ms_plain = timed(back_to_back, reps)
    ms_batch = timed(lambda: eng.multiply_batched(ds, "AA"), reps)
    # plan once, then replay the execute phase as a CUDA graph
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        p = eng.plan_batched(ds, "AA", stream=side)
        out = p.execute(stream=side)
        g = p.capture_graph(out, side)
    side.synchronize()

    def replay():
        with torch.cuda.stream(side):
            g.launch(side)
        side.synchronize()

    ms_graph = timed(replay, reps)
    g.close()
    p.close()
    t1 = time.time()
    tuned = eng.autotune(ds, "AA", reps=1)
    tune_s = time.time() - t1
    ms_tuned = timed(lambda: eng.multiply_batched(ds, "AA"), reps)
    gf = lambda ms: round(2.0 * prods / (ms * 1e-3) / 1e9, 3)  # noqa: E731
    line = {"metric": "GFLOP/s (2×intermediate products/s), batched A·A", "unit": "GFLOP/s",
            "mode": "batch", "value": gf(min(ms_batch, ms_tuned)), "higher_is_better": True,
            "data": "synthetic (seeded generator)", "dtype": "f64",
            "config": {"workload": f"{len(mats)} matrices, n log-uniform [1k, 64k], half banded "
                                   "(bw U{3..64}, 30% fill), half Erdős–Rényi (λ U(4,32)), A·A",
                       "total_nnz": int(sum(A.nnz for A in mats)), "total_products": int(prods),
                       "generation_s": round(gen_s, 1)},
            "back_to_back": {"ms": round(ms_plain, 3), "gflops": gf(ms_plain)},
            "batched": {"ms": round(ms_batch, 3), "gflops": gf(ms_batch),
                        "speedup_vs_back_to_back": round(ms_plain / ms_batch, 2)},
            "batched_graph_replay": {"ms": round(ms_graph, 3), "gflops": gf(ms_graph),
                                     "speedup_vs_back_to_back": round(ms_plain / ms_graph, 2),
                                     "note": "plan reused; execute phase replayed as a CUDA graph"},
            "batched_autotuned": {"ms": round(ms_tuned, 3), "gflops": gf(ms_tuned),
                                  "speedup_vs_back_to_back": round(ms_plain / ms_tuned, 2),
                                  "tuning_s": round(tune_s, 1),
                                  "config": {k: tuned[k] for k in ("lanes_per_row",
                                             "max_smem_slots", "num_load_pct", "sym_load_pct",
                                             "heavy_threads", "window_bits")}}}
    eng.close()
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# serving: Poisson arrivals of A·A / A·Aᵀ requests over the generator families
# ---------------------------------------------------------------------------
def serve_pool(count, seed):
    """Distinct request matrices: family uniform over {5-pt Laplacian,
    27-pt stencil, R-MAT}, n log-uniform in [2k, 2M]."""
    import numpy as np

    from appt_spgemm_b200 import csr
    rng = np.random.Generator(np.random.PCG64(seed))
    pool = []
    for i in range(count):
        n = float(np.exp(rng.uniform(np.log(2000), np.log(2_000_000))))
        fam = int(rng.integers(0, 3))
        if fam == 0:
            side = max(2, int(round(n ** 0.5)))
            A, desc = csr.laplace2d(side), f"laplace2d {side}^2"
        elif fam == 1:
            side = max(2, int(round(n ** (1 / 3))))
            A, desc = csr.stencil27(side, int(rng.integers(1, 2**31))), f"stencil27 {side}^3"
        else:
            sc = max(1, int(round(np.log2(n))))
            A, desc = csr.rmat(sc, 16, seed=int(rng.integers(1, 2**31))), f"rmat 2^{sc}"
        pool.append((A, desc))
    return pool


SERVE_FIGURES = ("p50_ms", "p99_ms", "small_p50_ms", "small_p99_ms", "sustained_gflops",
                 "peak_reserved_gb")


def aggregate_serve(runs):
    """One (rate, server) entry from its runs over several arrival streams:
    counts summed, each latency / throughput figure the median over the
    streams, with its [min, max] under `<figure>_range` when there are two or
    more."""
    out = {"rate_per_s": runs[0]["rate_per_s"], "server": runs[0]["server"]}
    for k in ("requests", "completed", "rejected", "failed", "batches", "small_requests"):
        out[k] = sum(r[k] for r in runs)
    for k in SERVE_FIGURES:
        v = sorted(r[k] for r in runs if r[k] is not None)
        if not v:
            out[k] = None
        elif len(v) % 2:
            out[k] = v[len(v) // 2]
        else:
            out[k] = round((v[len(v) // 2 - 1] + v[len(v) // 2]) / 2, 3)
        if len(runs) > 1:
            out[k + "_range"] = [v[0], v[-1]] if v else None
    out["streams"] = len(runs)
    splits = [r["small_split"] for r in runs if r.get("small_split")]
    if splits:  # the time split of small requests, per stream
        out["small_split"] = splits[0] if len(splits) == 1 else splits
    return out


SERVERS = (("continuous_batching", dict(workers=4, batch_rows=65536, batch_max=64)),
           ("queue_only", dict(workers=1, batch_rows=1, batch_max=1)))


def serve_once(pool, ds, prods, rate, label, kw, picks, tasks, gaps):
    """Run one arrival stream (request k: matrix picks[k], task tasks[k],
    arriving gaps[k] after request k-1) through a server; the result entry."""
    import threading

    from appt_spgemm_b200 import _capi
    from appt_spgemm_b200.engine import Server

    nreq = len(picks)
    with Server(memory_budget_bytes=150 * 10**9, **kw) as srv:
        ids = [None] * nreq
        done = []

        def consumer():
            # release results in completion order: a request waiting for
            # budget may need the memory of later ones
            pending = set()
            nxt = 0
            while len(done) < nreq:
                while nxt < nreq and ids[nxt] is not None:
                    pending.add(nxt)
                    nxt += 1
                finished = []
                for k in pending:
                    info = srv.poll(ids[k])
                    if info["status"] != _capi.SPG_ERR_NOT_READY:
                        finished.append((k, info))
                for k, info in finished:
                    pending.discard(k)
                    done.append((k, info))
                    if info["status"] == _capi.SPG_OK:
                        srv.release(ids[k])
                if not finished:
                    time.sleep(0.0002)

        th = threading.Thread(target=consumer)
        th.start()
        start = time.perf_counter()
        t_next = 0.0
        for k in range(nreq):
            t_next += gaps[k]
            delay = start + t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids[k] = srv.submit(ds[picks[k]], str(tasks[k]))
        th.join()
        st = srv.stats()
    ok = [(k, i) for k, i in done if i["status"] == _capi.SPG_OK]
    lat = sorted(i["done_ms"] - i["submit_ms"] for _, i in ok)
    small = sorted(i["done_ms"] - i["submit_ms"] for k, i in ok
                   if pool[int(picks[k])][0].n < 65536)

    def pct(v, q):
        return round(v[min(len(v) - 1, int(q * len(v)))], 3) if v else None

    # where a small request's latency goes: queued until a worker took it,
    # its symbolic pass, waiting for budget after it, and the numeric run
    def split(sel):
        parts = {"queued": ("submit_ms", "start_ms"), "planning": ("start_ms", "planned_ms"),
                 "admission": ("planned_ms", "run_ms"), "running": ("run_ms", "done_ms")}
        out = {}
        for name, (a, b) in parts.items():
            v = sorted(i[b] - i[a] for k, i in ok
                       if sel(k) and a in i and b in i and i[b] >= i[a] > 0)
            out[name + "_p50_ms"] = pct(v, 0.5)
        return out
    work = sum(2.0 * prods[(int(picks[k]), str(tasks[k]))] for k, _ in ok)
    span_s = (max(i["done_ms"] for _, i in ok) - min(i["submit_ms"] for _, i in ok)) / 1e3 \
        if ok else 0.0
    return {"rate_per_s": rate, "server": label, "requests": nreq,
            "completed": len(ok), "rejected": int(st["rejected"]),
            "failed": int(st["failed"]), "batches": int(st["batches"]),
            "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99),
            "small_requests": len(small),
            "small_p50_ms": pct(small, 0.5), "small_p99_ms": pct(small, 0.99),
            "small_split": split(lambda k: pool[int(picks[k])][0].n < 65536),
            "sustained_gflops": round(work / span_s / 1e9, 3) if ok and span_s > 0 else None,
            "peak_reserved_gb": round(st["peak_reserved_bytes"] / 1e9, 2)}


def serve_stream(rate_index, stream, nreq, npool, rate):
    """One arrival stream of the serving bench: matrix picks (indices into the
    pool), tasks ("AA" / "AAt", 50/50) and exponential gaps at `rate` per
    second, from numpy's PCG64 seeded with (55, rate_index, stream)."""
    import numpy as np

    rng = np.random.Generator(np.random.PCG64([55, rate_index, stream]))
    picks = rng.integers(0, npool, nreq)
    tasks = np.where(rng.random(nreq) < 0.5, "AA", "AAt")
    gaps = rng.exponential(1.0 / rate, nreq)
    return picks, tasks, gaps


def serve_back_to_back(ds, prods, nreq):
    """The request mix as back-to-back plain calls: the first arrival stream's
    requests (matrix and task as the servers got them, no arrival gaps) through
    Engine.multiply one after another on one stream, each result freed before
    the next call; CUDA events around the whole sequence."""
    import torch

    from appt_spgemm_b200.engine import Engine

    picks, tasks, _ = serve_stream(0, 0, nreq, len(ds), 1.0)
    work = sum(2.0 * prods[(int(i), str(t))] for i, t in zip(picks, tasks))
    with Engine("cuda:0") as eng:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for i, t in zip(picks, tasks):
            C = eng.multiply(ds[int(i)], str(t))
            del C
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
    torch.cuda.empty_cache()
    return {"requests": int(nreq), "ms": round(ms, 3), "gflops": round(work / (ms * 1e-3) / 1e9, 3),
            "note": "the requests of the first rate's first arrival stream, executed back "
                    "to back without arrival gaps"}


def run_serve(args):
    from appt_spgemm_b200 import csr
    from appt_spgemm_b200.engine import CsrDevice

    t0 = time.time()
    pool = serve_pool(args.serve_pool, seed=5)
    gen_s = time.time() - t0
    ds = [CsrDevice.from_host(A, "cuda:0") for A, _ in pool]
    prods = {(i, t): csr.products(A, "AA" if t == "AA" else "AAt")
             for i, (A, _) in enumerate(pool) for t in ("AA", "AAt")}
    rates = [float(r) for r in args.serve_rates.split(",")]
    runs = {}
    for ri, rate in enumerate(rates):
        for stream in range(args.serve_seeds):
            # one arrival stream per (rate, stream), run through both servers
            nreq = args.serve_requests
            picks, tasks, gaps = serve_stream(ri, stream, nreq, len(pool), rate)
            for label, kw in SERVERS:
                if label == "continuous_batching" and args.serve_workers > 0:
                    kw = dict(kw, workers=args.serve_workers)
                r = serve_once(pool, ds, prods, rate, label, kw, picks, tasks, gaps)
                runs.setdefault((rate, label), []).append(r)
                print(json.dumps(dict(r, stream=stream)), file=sys.stderr, flush=True)
    results = [aggregate_serve(runs[(rate, label)]) for rate in rates for label, _ in SERVERS]
    best = max((r["sustained_gflops"] or 0) for r in results)
    plain = serve_back_to_back(ds, prods, args.serve_requests)
    line = {"metric": "served GFLOP/s and p50/p99 latency, A·A / A·Aᵀ requests", "unit": "GFLOP/s",
            "mode": "serve", "value": best, "higher_is_better": True,
            "data": "synthetic (seeded generator)", "dtype": "f64",
            "config": {"workload": "Poisson arrivals; requests drawn uniformly from a pool of "
                                   f"{len(pool)} matrices (families 5-pt Laplacian / 27-pt stencil"
                                   " / R-MAT, n log-uniform [2k, 2M]); task A·A or A·Aᵀ 50/50; "
                                   "budget 150 GB; each arrival stream runs through both servers",
                       "streams_per_rate": args.serve_seeds, "pool": [d for _, d in pool],
                       "pool_generation_s": round(gen_s, 1)},
            "rates": results, "back_to_back_plain": plain}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# sub-results of the default line: the other configurations that fit one GPU
# ---------------------------------------------------------------------------
def time_calls(fn, reps, warm=3):
    """CUDA-event times (ms) of `reps` calls of fn() on the current stream, after
    `warm` untimed ones; a synchronize on both sides of each call."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return out


def ms_summary(ts):
    return {"ms_median": round(statistics.median(ts), 4), "ms_mean": round(statistics.mean(ts), 4),
            "ms_min": round(min(ts), 4), "calls": len(ts)}


def laplace_subresult(eng, reps=50):
    """The 2-D 5-point Laplacian 64² (n = 4,096, 4.0 diagonal, −1.0 neighbours):
    full calls (plan + execute) of A·A and A·Aᵀ in µs, beside cuSPARSE and the
    reference's CUDA engine on the same matrix; launch-latency-bound."""
    from appt_spgemm_b200 import csr
    from appt_spgemm_b200.engine import CsrDevice
    A = csr.laplace2d(64)
    dA = CsrDevice.from_host(A, "cuda:0")
    prods = {"AA": csr.products(A, "AA"), "AAt": csr.products(A, "AAt")}
    out = {"workload": f"2-D 5-point Laplacian 64^2 (n={A.n}, nnz={A.nnz}), one full call "
                       "(plan + execute) per product", "products": prods, "ours": {}}
    for task in ("AA", "AAt"):
        ts = time_calls(lambda: eng.multiply(dA, task), reps)
        m = ms_summary(ts)
        m["us_per_call"] = round(1e3 * m["ms_median"], 1)
        m["gflops"] = round(2.0 * prods[task] / (m["ms_median"] * 1e-3) / 1e9, 3)
        pl = eng.plan(dA, task)
        m["nnz_c"] = pl.nnz_c
        pl.close()
        out["ours"][task] = m
    # the same calls through the reference-compatible C entry point: spg_run_ours
    # times `reps` full calls with CUDA events in C++, as the reference's
    # run_ours does (src/spgemm_engine.cuh:199-202), with no Python in the loop
    from appt_spgemm_b200.engine import run_ours
    out["ours_run_ours"] = {}
    for task in ("AA", "AAt"):
        r = run_ours(task, dA.rowptr, dA.col, dA.val, A.n, A.nnz, reps)
        out["ours_run_ours"][task] = {"ms_mean": round(r.ms, 4),
                                      "us_per_call": round(1e3 * r.ms, 1), "nnz_c": r.nnz}
    out["cusparse"] = cusparse_baseline(dA, A, prods["AA"], prods["AAt"], reps=20)
    out["reference_gpu_engine"] = reference_gpu_baseline(A, prods["AA"], prods["AAt"], reps=20)
    for k in ("cusparse", "reference_gpu_engine"):
        for task in ("AA", "AAt"):
            r = out[k].get(task, {})
            if "ms_mean" in r:
                r["us_per_call"] = round(1e3 * r.get("ms_min", r["ms_mean"]), 1)
    return out


def batch_subresult(eng, reps=3):
    """512 matrices (n log-uniform [1k, 64k]; half random banded, half
    Erdős–Rényi), A·A of each, with the same work on both sides of each ratio:
    one batched plan + execute against 512 full calls, and one graph replay of
    the batched execute against 512 graph replays of per-instance executes."""
    import torch

    from appt_spgemm_b200 import csr
    from appt_spgemm_b200.engine import CsrDevice
    t0 = time.time()
    mats, _ = csr.batch_mix(512, seed=4)
    gen_s = time.time() - t0
    prods = sum(csr.products(A, "AA") for A in mats)
    ds = [CsrDevice.from_host(A, "cuda:0") for A in mats]
    gf = lambda ms: round(2.0 * prods / (ms * 1e-3) / 1e9, 3)  # noqa: E731

    def back_to_back():
        for d in ds:
            eng.multiply(d, "AA")

    full_each = statistics.median(time_calls(back_to_back, reps, warm=1))
    full_batched = statistics.median(time_calls(lambda: eng.multiply_batched(ds, "AA"), reps,
                                                warm=1))
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        plans = [eng.plan(d, "AA", stream=side) for d in ds]
        outs = [p.execute(stream=side) for p in plans]
        graphs = [p.capture_graph(o, side) for p, o in zip(plans, outs)]
        bp = eng.plan_batched(ds, "AA", stream=side)
        bout = bp.execute(stream=side)
        bg = bp.capture_graph(bout, side)
    side.synchronize()

    def replay_each():
        for g in graphs:
            g.launch(side)
        torch.cuda.current_stream().wait_stream(side)

    def replay_batched():
        bg.launch(side)
        torch.cuda.current_stream().wait_stream(side)

    rep_each = statistics.median(time_calls(replay_each, reps, warm=1))
    rep_batched = statistics.median(time_calls(replay_batched, reps, warm=1))
    for g in graphs + [bg]:
        g.close()
    for p in plans + [bp]:
        p.close()
    return {"workload": "512 matrices, n log-uniform [1k, 64k], half banded (bw U{3..64}, 30% "
                        "fill), half Erdős–Rényi (λ U(4,32)), A·A of each",
            "total_nnz": int(sum(A.nnz for A in mats)), "total_products": int(prods),
            "generation_s": round(gen_s, 1),
            "full_calls": {"back_to_back_ms": round(full_each, 3), "batched_ms": round(full_batched, 3),
                           "back_to_back_gflops": gf(full_each), "batched_gflops": gf(full_batched),
                           "speedup": round(full_each / full_batched, 2),
                           "note": "plan + execute on both sides"},
            "graph_replay": {"per_instance_ms": round(rep_each, 3),
                             "batched_ms": round(rep_batched, 3),
                             "per_instance_gflops": gf(rep_each), "batched_gflops": gf(rep_batched),
                             "speedup": round(rep_each / rep_batched, 2),
                             "note": "execute phase of reused plans, replayed as CUDA graphs on "
                                     "both sides"},
            "batched_replay_vs_back_to_back_calls": round(full_each / rep_batched, 2)}


# ---------------------------------------------------------------------------
# replicas: every rank runs the whole workload; the job's step time is the
# slowest rank's, its throughput the sum of the replicas' work over that time
# ---------------------------------------------------------------------------
def replica_step_time(ms, device):
    """Max over ranks of this rank's step time in ms (the rank's own time
    when no process group is running)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(work_per_step, ms, world):
    """Whole-job GFLOP/s: `world` replicas, each 2·products = work_per_step
    per step, over the slowest rank's step time."""
    return world * work_per_step / (ms * 1e-3) / 1e9


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.mode in ("rmat", "laplace"):
        run_rmat(args)
        return
    if args.mode == "batch":
        run_batch(args)
        return
    if args.mode == "serve":
        run_serve(args)
        return
    import torch
    import torch.distributed as dist

    from appt_spgemm_b200.engine import CsrDevice, Engine

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    A, p_aa, p_aat = workload(args.side)
    work_per_step = 2.0 * (p_aa + p_aat)
    dA = CsrDevice.from_host(A, dev)
    eng = Engine(dev)
    stream = torch.cuda.current_stream()

    def step():
        C1 = eng.multiply(dA, "AA")
        C2 = eng.multiply(dA, args.aat_task)
        return C1, C2

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    eng.profile_reset()
    eng.profile_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            C = step()
            del C
        e1.record(stream)
        torch.cuda.synchronize()
    eng.profile_enable(False)
    prof = eng.profile_read()
    ms = replica_step_time(e0.elapsed_time(e1) / max(args.steps, 1), dev)
    if world > 1:
        dist.barrier()
    value = replica_value(work_per_step, ms, world)

    # per-task info, dominant kernel and its roofline
    infos = {}
    for task in ("AA", args.aat_task):
        p = eng.plan(dA, task)
        infos[task] = dict(p.info)
        p.close()
    kernels = prof.get("kernels", {})
    top = max(kernels.items(), key=lambda kv: kv[1]["ms"]) if kernels else None
    peak, peak_kind = hbm_peak()
    n, nnz = A.n, A.nnz
    roofline = None
    if top:
        label, rec = top
        per_launch_ms = rec["ms"] / max(rec["count"], 1)
        # algorithmic bytes per launch (per call of the phase): numeric kernels
        # read A once and write C once; symbolic kernels read A's structure and
        # write one count per row; the transpose reads and writes A once.
        nnz_c_mean = statistics.mean(i["nnz_c"] for i in infos.values())
        if label.startswith("num/"):
            alg = 4 * (n + 1) + 12 * nnz + 8 * (n + 1) + 12 * nnz_c_mean
        elif label.startswith("sym/"):
            alg = 4 * (n + 1) + 4 * nnz + 4 * n
        elif label == "plan/transpose":
            alg = 2 * (4 * (n + 1) + 12 * nnz)
        else:
            alg = 4 * (n + 1) + 12 * nnz
        achieved = alg / (per_launch_ms * 1e-3) / 1e9
        traffic = None
        try:
            with open(TRAFFIC) as f:
                traffic = json.load(f).get(label)
        except Exception:
            pass
        roofline = {"bound": "hbm", "kernel": label, "achieved": round(achieved, 1),
                    "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                    "peak_source": peak_kind, "traffic": traffic,
                    "alg_bytes_per_launch": int(alg), "ms_per_launch": round(per_launch_ms, 4),
                    "share_of_step": round(rec["ms"] / (ms * args.steps), 4)}
    call_alg = sum(4 * (n + 1) + 12 * nnz + 8 * (n + 1) + 12 * i["nnz_c"] for i in infos.values())

    # per-call times of the three tasks (the Gram path gives the same C as
    # A·Aᵀ; it is timed here beside the line, not inside the step)
    per_task_ms = {}
    for task in ("AA", "AAt", "AAtS"):
        ts = []
        for _ in range(3):
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            C = eng.multiply(dA, task)
            a1.record(stream)
            torch.cuda.synchronize()
            del C
            ts.append(a0.elapsed_time(a1))
        per_task_ms[task] = round(statistics.median(ts), 4)

    result = {"metric": METRIC,
              "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world,
              "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
              "data": "synthetic (seeded generator)",
              "config": config(args, A), "aat_task": args.aat_task,
              "roofline": roofline,
              "call_roofline": {"alg_bytes_per_step": int(call_alg),
                                "achieved": round(call_alg / (ms * 1e-3) / 1e9, 1),
                                "frac": round(call_alg / (ms * 1e-3) / 1e9 / peak, 4),
                                "unit": "GB/s"},
              "gpu_launches": int(prof.get("launches", 0)),
              "kernels_ms_per_step": {k: round(v["ms"] / args.steps, 4)
                                      for k, v in sorted(kernels.items())},
              "products": {"AA": p_aa, "AAt": p_aat},
              "ms_per_call": per_task_ms,
              "nnz_c": {t: i["nnz_c"] for t, i in infos.items()},
              "clocks": clocks.summary()}

    # end to end through the public API: host CSR in pinned memory → device,
    # both products, C back to pinned host buffers, every step.  The copies run
    # on their own streams: a product's C goes back while the next product is
    # computed, and the next step's A comes in (into the other of two input
    # buffers) while this step computes.
    if rank == 0 or world > 1:
        pin = lambda x: torch.from_numpy(x).pin_memory()  # noqa: E731
        h_rp, h_col, h_val = pin(A.rowptr), pin(A.col), pin(A.val)
        inputs = [(torch.empty_like(dA.rowptr), torch.empty_like(dA.col), torch.empty_like(dA.val))
                  for _ in range(2)]
        in_free = [torch.cuda.Event(), torch.cuda.Event()]  # buffer read by its last step
        outs = {t: (torch.empty(n + 1, dtype=torch.int64).pin_memory(),
                    torch.empty(infos[t]["nnz_c"], dtype=torch.int32).pin_memory(),
                    torch.empty(infos[t]["nnz_c"], dtype=torch.float64).pin_memory())
                for t in infos}
        h2d = h_rp.numel() * 4 + h_col.numel() * 4 + h_val.numel() * 8
        d2h = sum((n + 1) * 8 + infos[t]["nnz_c"] * 12 for t in infos)
        up, down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        for ev in in_free:
            ev.record(stream)

        def e2e_step(k):
            d_rp, d_col, d_val = inputs[k % 2]
            up.wait_event(in_free[k % 2])
            with torch.cuda.stream(up):
                d_rp.copy_(h_rp, non_blocking=True)
                d_col.copy_(h_col, non_blocking=True)
                d_val.copy_(h_val, non_blocking=True)
            stream.wait_stream(up)
            M = CsrDevice(n, d_rp, d_col, d_val)
            for t in ("AA", args.aat_task):
                C = eng.multiply(M, t)
                down.wait_stream(stream)
                with torch.cuda.stream(down):
                    o = outs[t]
                    o[0].copy_(C.rowptr, non_blocking=True)
                    o[1].copy_(C.col, non_blocking=True)
                    o[2].copy_(C.val, non_blocking=True)
                for x in (C.rowptr, C.col, C.val):
                    x.record_stream(down)
            in_free[k % 2].record(stream)

        e2e_steps = max(1, min(args.steps, 5))
        e2e_step(0)
        torch.cuda.synchronize()
        e0.record(stream)
        for k in range(e2e_steps):
            e2e_step(k + 1)
        stream.wait_stream(down)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / e2e_steps
        result["e2e"] = {"value": round(work_per_step / (e2e_ms * 1e-3) / 1e9, 3),
                         "unit": "GFLOP/s", "h2d_bytes_per_step": int(h2d),
                         "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms, 3),
                         "api": "Engine.multiply (spg_plan_create + spg_execute); copies on "
                                "their own streams, overlapped with the products"}

    if rank == 0 and world == 1 and not args.no_baselines:
        nthreads = os.cpu_count() or 1
        gf, prods, secs, sample = cpu_oracle_rate(A, args.cpu_seconds, nthreads)
        result["cpu_baseline"] = {"value": round(gf, 3), "unit": "GFLOP/s", "cores": nthreads,
                                  "kind": "port", "sample": sample + f" ({prods} products, "
                                  f"{secs:.1f} s)"}
        result["baselines"] = {"cusparse": cusparse_baseline(dA, A, p_aa, p_aat),
                               "reference_gpu_engine": reference_gpu_baseline(A, p_aa, p_aat)}
        cs = result["baselines"]["cusparse"]
        if all("ms_mean" in cs.get(t, {}) for t in ("AA", "AAt")):
            cms = cs["AA"]["ms_mean"] + cs["AAt"]["ms_mean"]
            result["baselines"]["cusparse_step_gflops"] = round(work_per_step / (cms * 1e-3) / 1e9, 3)
    if rank == 0 and world == 1 and not args.no_sub:
        del dA
        torch.cuda.empty_cache()
        result["sub_results"] = {"laplace2d_64": laplace_subresult(eng),
                                 "batch_512": batch_subresult(eng)}

    eng.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
