"""Device-side API of the engine over the C ABI, with torch as the memory plumbing.

``run_ours`` mirrors the reference entry point
``run_ours(task, dOff, dCol, dVal, n, nnz, reps)`` (src/spgemm_engine.cuh:132-210):
same task names ("AA", "AAt", "AAtS"), same result record {ms, nnz, s, as, sq}.
``Engine`` exposes what the reference kept internal: the product C itself as
CSR with int64 row pointers, a plan/execute split, the transpose and the
structural descriptors.  Every call goes to the CUDA library; there is no
CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import torch

from . import _capi
from ._capi import (SpgConfig, SpgCsrDev, SpgCsrOut, SpgDescriptors, SpgEngResult, SpgPlanInfo,
                    check, lib)
from .csr import CsrHost


@dataclass
class EngResult:
    """The reference's EngResult (src/spgemm_engine.cuh:129)."""

    ms: float
    nnz: int
    s: float
    as_: float
    sq: float


@dataclass
class CsrDevice:
    """Square CSR on a CUDA device: int32 rowptr/col, float64 val."""

    n: int
    rowptr: torch.Tensor
    col: torch.Tensor
    val: torch.Tensor

    @property
    def nnz(self) -> int:
        return int(self.col.numel())

    @classmethod
    def from_host(cls, A: CsrHost, device="cuda", pin: bool = False) -> "CsrDevice":
        def up(x):
            t = torch.from_numpy(x)
            if pin:
                t = t.pin_memory()
            return t.to(device, non_blocking=pin)
        return cls(A.n, up(A.rowptr), up(A.col), up(A.val))

    def struct(self) -> SpgCsrDev:
        return SpgCsrDev(self.n, self.nnz, self.rowptr.data_ptr(),
                         self.col.data_ptr() if self.nnz else 0,
                         self.val.data_ptr() if self.nnz else 0)

    def to_host(self) -> CsrHost:
        return CsrHost(self.n, self.rowptr.cpu().numpy(), self.col.cpu().numpy(),
                       self.val.cpu().numpy())


@dataclass
class CsrResult:
    """C on the device: int64 rowptr, int32 col, float64 val."""

    n: int
    nnz: int
    rowptr: torch.Tensor
    col: torch.Tensor
    val: torch.Tensor

    def to_host(self):
        """(rowptr int64, col int32, val float64) numpy arrays."""
        return (self.rowptr.cpu().numpy(), self.col.cpu().numpy(), self.val.cpu().numpy())


def _stream_handle(stream: Optional[torch.cuda.Stream]) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _task_id(task) -> int:
    if isinstance(task, int):
        return task
    if task not in _capi.TASKS:
        raise _capi.SpgemmError(_capi.SPG_ERR_INVALID_ARG, f"unknown task {task!r}")
    return _capi.TASKS[task]


def make_config(**kw) -> SpgConfig:
    c = SpgConfig()
    c.struct_size = ctypes.sizeof(SpgConfig)
    for k, v in kw.items():
        if not hasattr(c, k):
            raise ValueError(f"unknown config field {k}")
        setattr(c, k, v)
    return c


class Plan:
    """Pre-pass, binning and symbolic phase done; nnz(C) known (``info``)."""

    def __init__(self, engine: "Engine", handle: ctypes.c_void_p, A, task: str, count: int = 0):
        self._engine = engine
        self._h = handle
        self._A = A  # keep the input(s) alive for execute
        self.task = task
        self.count = count
        info = SpgPlanInfo()
        check(lib().spg_plan_get_info(self._h, ctypes.byref(info)), "plan info")
        self.info = {f: getattr(info, f) for f, _ in SpgPlanInfo._fields_ if f != "reserved"}

    @property
    def nnz_c(self) -> int:
        return int(self.info["nnz_c"])

    def execute(self, out: Optional[CsrResult] = None, stream=None) -> CsrResult:
        n = self.info["n"]
        dev = (self._A[0] if isinstance(self._A, (list, tuple)) else self._A).rowptr.device
        if out is None:
            out = CsrResult(
                n, self.nnz_c,
                torch.empty(n + 1, dtype=torch.int64, device=dev),
                torch.empty(max(self.nnz_c, 1), dtype=torch.int32, device=dev)[: self.nnz_c],
                torch.empty(max(self.nnz_c, 1), dtype=torch.float64, device=dev)[: self.nnz_c])
        c = SpgCsrOut(n, 0, out.rowptr.data_ptr(),
                      out.col.data_ptr() if out.col.numel() or self.nnz_c == 0 else 0,
                      out.val.data_ptr() if out.val.numel() or self.nnz_c == 0 else 0)
        if self.nnz_c == 0:
            c.col = out.rowptr.data_ptr()  # never written; any valid address
            c.val = out.rowptr.data_ptr()
        check(lib().spg_execute(self._h, ctypes.byref(c), _stream_handle(stream)), "execute")
        out.nnz = int(c.nnz)
        return out

    def offsets(self):
        """Batched plans: (row_off, nnz_off) int64 arrays of count+1 entries —
        instance b owns rows [row_off[b], row_off[b+1]) and entries
        [nnz_off[b], nnz_off[b+1]) of the concatenated C."""
        import numpy as np
        n = self.count + 1
        ro = np.zeros(n, dtype=np.int64)
        no = np.zeros(n, dtype=np.int64)
        check(lib().spg_plan_batch_offsets(self._h, ro.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                           no.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
              "batch offsets")
        return ro, no

    def capture_graph(self, out: CsrResult, stream: torch.cuda.Stream) -> "Graph":
        """CUDA graph of execute() into `out` on `stream` (a created stream)."""
        c = SpgCsrOut(out.n, 0, out.rowptr.data_ptr(), out.col.data_ptr(), out.val.data_ptr())
        g = ctypes.c_void_p()
        check(lib().spg_graph_capture(self._h, ctypes.byref(c), int(stream.cuda_stream),
                                      ctypes.byref(g)), "graph capture")
        return Graph(g, self, out)

    def close(self) -> None:
        if self._h:
            lib().spg_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """An instantiated CUDA graph of one plan's execute phase."""

    def __init__(self, handle, plan: Plan, out: CsrResult):
        self._h = handle
        self._plan = plan  # the graph reads the plan's workspace
        self.out = out

    def launch(self, stream: Optional[torch.cuda.Stream] = None) -> CsrResult:
        check(lib().spg_graph_launch(self._h, _stream_handle(stream)), "graph launch")
        return self.out

    def close(self) -> None:
        if self._h:
            lib().spg_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class BatchResult:
    """Concatenated C of a batched product and the instance offsets."""

    C: CsrResult
    row_off: "object"
    nnz_off: "object"

    def instance(self, b: int):
        """(rowptr int64 rebased to 0, col, val) device views of instance b."""
        r0, r1 = int(self.row_off[b]), int(self.row_off[b + 1])
        e0, e1 = int(self.nnz_off[b]), int(self.nnz_off[b + 1])
        return (self.C.rowptr[r0:r1 + 1] - e0, self.C.col[e0:e1], self.C.val[e0:e1])


class Engine:
    """One engine context (memory pool, status word) on one CUDA device."""

    def __init__(self, device=None, **config):
        if not torch.cuda.is_available():
            raise RuntimeError("the SpGEMM engine needs a CUDA device")
        dev = torch.device(device) if device is not None else torch.device("cuda")
        self.device = torch.device("cuda", dev.index if dev.index is not None
                                   else torch.cuda.current_device())
        torch.cuda.set_device(self.device)
        torch.cuda.init()
        cfg = make_config(**config)
        if self.device.index:
            cfg.device = self.device.index
        h = ctypes.c_void_p()
        check(lib().spg_create(ctypes.byref(h), ctypes.byref(cfg)), "create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().spg_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def plan(self, A: CsrDevice, task: str = "AA", stream=None) -> Plan:
        s = A.struct()
        p = ctypes.c_void_p()
        check(lib().spg_plan_create(self._h, _task_id(task), ctypes.byref(s),
                                    _stream_handle(stream), ctypes.byref(p)), "plan")
        return Plan(self, p, A, task)

    def multiply(self, A: CsrDevice, task: str = "AA", stream=None) -> CsrResult:
        """C = A·A, A·Aᵀ ("AAt") or A·Aᵀ via the Gram path ("AAtS").

        The plan/execute pair of plan().execute() without the Plan object: one
        stream lookup, only n and nnz(C) read from the plan's info, so that a
        call on a small matrix spends little beyond the library's own time."""
        sh = _stream_handle(stream)
        s = A.struct()
        L = lib()
        p = ctypes.c_void_p()
        check(L.spg_plan_create(self._h, _task_id(task), ctypes.byref(s), sh, ctypes.byref(p)),
              "plan")
        try:
            info = SpgPlanInfo()
            check(L.spg_plan_get_info(p, ctypes.byref(info)), "plan info")
            n, nnz = int(info.n), int(info.nnz_c)
            dev = A.rowptr.device
            rp = torch.empty(n + 1, dtype=torch.int64, device=dev)
            col = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
            val = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
            c = SpgCsrOut(n, 0, rp.data_ptr(), col.data_ptr(), val.data_ptr())
            check(L.spg_execute(p, ctypes.byref(c), sh), "execute")
        finally:
            L.spg_plan_destroy(p)
        if nnz != col.numel():
            col, val = col[:nnz], val[:nnz]
        return CsrResult(n, int(c.nnz), rp, col, val)

    def plan_batched(self, As, task: str = "AA", stream=None) -> Plan:
        """One plan for many independent products (block-diagonal layout)."""
        arr = (SpgCsrDev * len(As))(*[A.struct() for A in As])
        p = ctypes.c_void_p()
        check(lib().spg_plan_create_batched(self._h, _task_id(task), len(As), arr,
                                            _stream_handle(stream), ctypes.byref(p)),
              "batched plan")
        return Plan(self, p, list(As), task, count=len(As))

    def multiply_batched(self, As, task: str = "AA", stream=None) -> BatchResult:
        p = self.plan_batched(As, task, stream)
        try:
            C = p.execute(stream=stream)
            ro, no = p.offsets()
            return BatchResult(C, ro, no)
        finally:
            p.close()

    def get_config(self) -> dict:
        c = SpgConfig()
        check(lib().spg_get_config(self._h, ctypes.byref(c)), "get_config")
        return {f: getattr(c, f) for f, _ in SpgConfig._fields_
                if not f.startswith("reserved") and f != "struct_size"}

    def set_config(self, **kw) -> None:
        cur = self.get_config()
        cur.update(kw)
        cur.pop("device", None)
        c = make_config(**cur)
        check(lib().spg_set_config(self._h, ctypes.byref(c)), "set_config")

    def autotune(self, A, task: str = "AA", reps: int = 3, stream=None) -> dict:
        """Coordinate-descent search over bin thresholds, table loads, lanes per
        row and heavy-path shapes, timed on A (a matrix or a list of matrices,
        tuned as one batch); the best tuning stays in this engine."""
        As = list(A) if isinstance(A, (list, tuple)) else [A]
        arr = (SpgCsrDev * len(As))(*[M.struct() for M in As])
        best = SpgConfig()
        check(lib().spg_autotune(self._h, _task_id(task), len(As), arr, reps, ctypes.byref(best),
                                 _stream_handle(stream)), "autotune")
        return self.get_config()

    def autotune_trials(self) -> dict:
        """Candidates of the last autotune: timed, and pruned by the descriptors."""
        t, p = ctypes.c_int32(), ctypes.c_int32()
        check(lib().spg_autotune_trials(self._h, ctypes.byref(t), ctypes.byref(p)), "trials")
        return {"timed": t.value, "pruned": p.value}

    def transpose(self, A: CsrDevice, stream=None) -> CsrDevice:
        dev = A.rowptr.device
        tp = torch.empty(A.n + 1, dtype=torch.int32, device=dev)
        tc = torch.empty(max(A.nnz, 1), dtype=torch.int32, device=dev)
        tv = torch.empty(max(A.nnz, 1), dtype=torch.float64, device=dev)
        s = A.struct()
        check(lib().spg_transpose(self._h, ctypes.byref(s), tp.data_ptr(), tc.data_ptr(),
                                  tv.data_ptr(), _stream_handle(stream)), "transpose")
        return CsrDevice(A.n, tp, tc[: A.nnz], tv[: A.nnz])

    def drop_zeros(self, C: CsrResult, stream=None) -> CsrResult:
        """Drop C's exact zero values in place (scipy's eliminate_zeros()
        pattern); returns C with its nnz and col/val views shortened."""
        c = SpgCsrOut(C.n, C.nnz, C.rowptr.data_ptr(), C.col.data_ptr() if C.nnz else 0,
                      C.val.data_ptr() if C.nnz else 0)
        check(lib().spg_drop_zeros(self._h, ctypes.byref(c), _stream_handle(stream)),
              "drop zeros")
        C.nnz = int(c.nnz)
        C.col = C.col[: C.nnz]
        C.val = C.val[: C.nnz]
        return C

    def describe(self, A: CsrDevice, stream=None) -> dict:
        d = SpgDescriptors()
        s = A.struct()
        check(lib().spg_describe(self._h, ctypes.byref(s), ctypes.byref(d),
                                 _stream_handle(stream)), "describe")
        return {f: getattr(d, f) for f, _ in SpgDescriptors._fields_ if f != "reserved"}

    def check_device_status(self, stream=None) -> None:
        check(lib().spg_check_device_status(self._h, _stream_handle(stream)), "device status")

    # per-kernel CUDA events on the launching stream, and the launch counter
    def profile_enable(self, on: bool = True) -> None:
        check(lib().spg_profile_enable(self._h, 1 if on else 0), "profile_enable")

    def profile_reset(self) -> None:
        check(lib().spg_profile_reset(self._h), "profile_reset")

    def profile_read(self) -> dict:
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        check(lib().spg_profile_read(self._h, buf, len(buf)), "profile_read")
        return json.loads(buf.value.decode())


def run_ours(task: str, dOff: torch.Tensor, dCol: torch.Tensor, dVal: torch.Tensor, n: int,
             nnz: int, reps: int) -> EngResult:
    """The reference's run_ours on device CSR tensors: one checked call, then
    ``reps`` timed full calls (mean ms); nnz(C) and checksums Σv, Σ|v|, Σv²."""
    r = SpgEngResult()
    check(lib().spg_run_ours(task.encode(), dOff.data_ptr(), dCol.data_ptr() if nnz else 0,
                             dVal.data_ptr() if nnz else 0, n, nnz, reps, ctypes.byref(r)),
          "run_ours")
    return EngResult(float(r.ms), int(r.nnz), float(r.s), float(r.as_), float(r.sq))


def checksum(vals: torch.Tensor):
    """Σv, Σ|v|, Σv² of a device FP64 array, summed in index order on the host."""
    s, a, q = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    check(lib().spg_checksum(vals.data_ptr() if vals.numel() else 0, vals.numel(),
                             ctypes.byref(s), ctypes.byref(a), ctypes.byref(q)), "checksum")
    return (s.value, a.value, q.value)


class Server:
    """Request server (spg_server_*): continuous batching of A·A / A·Aᵀ requests
    with admission by a device-memory budget from the symbolic pass."""

    def __init__(self, workers: int = 4, memory_budget_bytes: int = 0, batch_rows: int = 0,
                 batch_max: int = 0, device=None):
        if device is not None:
            torch.cuda.set_device(torch.device(device))
        torch.cuda.init()
        cfg = _capi.SpgServerConfig()
        cfg.struct_size = ctypes.sizeof(_capi.SpgServerConfig)
        cfg.workers = workers
        cfg.memory_budget_bytes = memory_budget_bytes
        cfg.batch_rows = batch_rows
        cfg.batch_max = batch_max
        h = ctypes.c_void_p()
        check(lib().spg_server_create(ctypes.byref(cfg), ctypes.byref(h)), "server create")
        self._h = h
        self._inputs = {}  # request id → input kept alive until the request is done

    @staticmethod
    def _info(i) -> dict:
        return {f: getattr(i, f) for f, _ in _capi.SpgRequestInfo._fields_}

    def submit(self, A: CsrDevice, task: str = "AA") -> int:
        s = A.struct()
        rid = ctypes.c_uint64()
        check(lib().spg_server_submit(self._h, _task_id(task), ctypes.byref(s), ctypes.byref(rid)),
              "submit")
        self._inputs[rid.value] = A
        return rid.value

    def poll(self, rid: int) -> dict:
        i = _capi.SpgRequestInfo()
        check(lib().spg_server_poll(self._h, rid, ctypes.byref(i)), "poll")
        return self._info(i)

    def wait(self, rid: int, timeout_ms: int = -1) -> dict:
        i = _capi.SpgRequestInfo()
        check(lib().spg_server_wait(self._h, rid, timeout_ms, ctypes.byref(i)), "wait")
        self._inputs.pop(rid, None)
        return self._info(i)

    def result(self, rid: int, device=None) -> CsrResult:
        """Copy a finished result into new device tensors (the server keeps its copy)."""
        info = self.wait(rid)
        if info["status"] != _capi.SPG_OK:
            raise _capi.SpgemmError(info["status"], f"request {rid} did not complete")
        dev = torch.device(device) if device is not None else torch.device("cuda")
        n, nnz = info["n"], info["nnz_c"]
        rp = torch.empty(n + 1, dtype=torch.int64, device=dev)
        col = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        val = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
        check(lib().spg_server_copy_result(self._h, rid, rp.data_ptr(), col.data_ptr(),
                                           val.data_ptr()), "copy result")
        return CsrResult(n, nnz, rp, col[:nnz], val[:nnz])

    def release(self, rid: int) -> None:
        check(lib().spg_server_release(self._h, rid), "release")

    def stats(self) -> dict:
        st = _capi.SpgServerStats()
        check(lib().spg_server_stats_get(self._h, ctypes.byref(st)), "stats")
        return {f: getattr(st, f) for f, _ in _capi.SpgServerStats._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().spg_server_destroy(self._h)
            self._h = None
            self._inputs.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
