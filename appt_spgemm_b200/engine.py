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

    def __init__(self, engine: "Engine", handle: ctypes.c_void_p, A: CsrDevice, task: str):
        self._engine = engine
        self._h = handle
        self._A = A  # keep the input alive for execute
        self.task = task
        info = SpgPlanInfo()
        check(lib().spg_plan_get_info(self._h, ctypes.byref(info)), "plan info")
        self.info = {f: getattr(info, f) for f, _ in SpgPlanInfo._fields_ if f != "reserved"}

    @property
    def nnz_c(self) -> int:
        return int(self.info["nnz_c"])

    def execute(self, out: Optional[CsrResult] = None, stream=None) -> CsrResult:
        n = self.info["n"]
        dev = self._A.rowptr.device
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

    def close(self) -> None:
        if self._h:
            lib().spg_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


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
        """C = A·A, A·Aᵀ ("AAt") or A·Aᵀ via the Gram path ("AAtS")."""
        p = self.plan(A, task, stream)
        try:
            return p.execute(stream=stream)
        finally:
            p.close()

    def transpose(self, A: CsrDevice, stream=None) -> CsrDevice:
        dev = A.rowptr.device
        tp = torch.empty(A.n + 1, dtype=torch.int32, device=dev)
        tc = torch.empty(max(A.nnz, 1), dtype=torch.int32, device=dev)
        tv = torch.empty(max(A.nnz, 1), dtype=torch.float64, device=dev)
        s = A.struct()
        check(lib().spg_transpose(self._h, ctypes.byref(s), tp.data_ptr(), tc.data_ptr(),
                                  tv.data_ptr(), _stream_handle(stream)), "transpose")
        return CsrDevice(A.n, tp, tc[: A.nnz], tv[: A.nnz])

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
