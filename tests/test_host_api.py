"""Host-side checks that need no GPU: the C-ABI library loads and exports every
declared entry point, CSR1 files, host validation and the generators."""
import ctypes
import os
import re

import numpy as np
import pytest

from appt_spgemm_b200 import _capi, csr
from appt_spgemm_b200._capi import SpgemmError

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "spgemm_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(spg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers the same set
    assert set(names) <= set(_capi.SIGNATURES), set(names) - set(_capi.SIGNATURES)


def test_abi_version_and_status_strings():
    L = _capi.lib()
    assert L.spg_abi_version() == 1
    assert L.spg_status_string(0) == b"ok"
    assert L.spg_status_string(2) == b"invalid CSR"


def test_csr1_reader_reads_reference_files(golden, golden_dir):
    for name, g in golden["cases"].items():
        A = csr.load_bin(os.path.join(golden_dir, name + ".csr"))
        assert A.n == g["n"] and A.nnz == g["nnz"]
        A.validate()


def test_csr1_writer_is_byte_identical_to_reference_writer(golden, golden_dir, tmp_path):
    for name in golden["cases"]:
        src = os.path.join(golden_dir, name + ".csr")
        A = csr.load_bin(src)
        dst = tmp_path / (name + ".csr")
        csr.write_bin(A, str(dst))
        assert open(src, "rb").read() == open(dst, "rb").read(), name


def test_generators_regenerate_golden_inputs(golden_dir):
    for name, A in (("laplace2d_64", csr.laplace2d(64)), ("stencil27_6", csr.stencil27(6, 2)),
                    ("uniform_300x7", csr.uniform(300, 7, 11)),
                    ("banded_500_bw8", csr.banded(500, 8, 0.3, 12)),
                    ("er_400_l6", csr.erdos_renyi(400, 6.0, 13)),
                    ("rmat_s9_ef8", csr.rmat(9, 8, seed=14))):
        B = csr.load_bin(os.path.join(golden_dir, name + ".csr"))
        assert np.array_equal(A.rowptr, B.rowptr) and np.array_equal(A.col, B.col)
        assert np.array_equal(A.val.view(np.int64), B.val.view(np.int64)), name


def test_csr1_errors(tmp_path):
    p = tmp_path / "bad.csr"
    p.write_bytes(b"CSR2" + b"\0" * 16)
    with pytest.raises(SpgemmError) as e:
        csr.load_bin(str(p))
    assert e.value.status == _capi.SPG_ERR_IO
    p.write_bytes(b"CSR1" + np.array([10, 0], np.int32).tobytes() + np.array([5], np.int64).tobytes())
    with pytest.raises(SpgemmError):
        csr.load_bin(str(p))
    with pytest.raises(SpgemmError):
        csr.load_bin(str(tmp_path / "missing.csr"))


def test_host_validation_rejects_malformed():
    good = csr.laplace2d(4)
    good.validate()
    cases = []
    unsorted = csr.laplace2d(4)
    unsorted.col[[1, 2]] = unsorted.col[[2, 1]]
    cases.append(unsorted)
    dup = csr.laplace2d(4)
    dup.col[2] = dup.col[1]
    cases.append(dup)
    oob = csr.laplace2d(4)
    oob.col[-1] = 16
    cases.append(oob)
    nonmono = csr.laplace2d(4)
    nonmono.rowptr[3], nonmono.rowptr[4] = nonmono.rowptr[4], nonmono.rowptr[3]
    cases.append(nonmono)
    for A in cases:
        with pytest.raises(SpgemmError) as e:
            A.validate()
        assert e.value.status == _capi.SPG_ERR_INVALID_CSR


def test_benchmark_generator_sizes():
    """Counts quoted for the benchmark configurations: the 5-point Laplacian on
    64² (nnz 20,224; products 100,104) and the 27-point stencil on 96³
    (nnz 23,393,656; A·A products 622,835,864)."""
    A = csr.laplace2d(64)
    assert (A.n, A.nnz) == (4096, 20224)
    assert csr.products(A, "AA") == 100104 == csr.products(A, "AAt")
    B = csr.stencil27(96, seed=2)
    assert (B.n, B.nnz) == (884736, 23393656)
    assert csr.products(B, "AA") == 622835864
    assert B.val.min() >= -1.0 and B.val.max() < 1.0
    B2 = csr.stencil27(8, seed=2)
    B3 = csr.stencil27(8, seed=2)
    assert np.array_equal(B2.val, B3.val)


def test_rmat_properties():
    R = csr.rmat(12, 16, seed=3)
    R.validate()
    assert R.n == 4096
    assert R.nnz < 16 * 4096  # duplicates merged
    assert R.val.min() >= 0.0 and R.val.max() < 1.0
    rows = np.repeat(np.arange(R.n), np.diff(R.rowptr))
    assert (rows == R.col).sum() > 0  # self-loops kept
    deg = np.diff(R.rowptr)
    assert deg[:64].mean() > 4 * deg.mean()  # mass concentrates on low indices (a = 0.57)


def test_er_and_banded_shapes():
    E = csr.erdos_renyi(3000, 12.0, seed=9)
    E.validate()
    assert abs(E.nnz / 3000 - 12.0) < 0.5
    Bd = csr.banded(3000, 16, 0.3, seed=9)
    Bd.validate()
    rows = np.repeat(np.arange(Bd.n), np.diff(Bd.rowptr))
    assert np.abs(rows - Bd.col).max() <= 16
    assert (rows == Bd.col).sum() == 3000


def declared_prototypes():
    """name -> number of parameters, from the header's prototypes."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(spg_[a-z0-9_]+)\s*\(([^;{}]*?)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_argument_counts_match_the_header():
    protos = declared_prototypes()
    assert set(protos) == set(declared_functions())
    wrong = {n: (k, len(_capi.SIGNATURES[n][1])) for n, k in protos.items()
             if len(_capi.SIGNATURES[n][1]) != k}
    assert not wrong, wrong


STRUCTS = {"spg_csr_dev": "SpgCsrDev", "spg_csr_out": "SpgCsrOut", "spg_config": "SpgConfig",
           "spg_eng_result": "SpgEngResult", "spg_plan_info": "SpgPlanInfo",
           "spg_descriptors": "SpgDescriptors", "spg_server_config": "SpgServerConfig",
           "spg_request_info": "SpgRequestInfo", "spg_server_stats": "SpgServerStats",
           "spg_host_csr": "SpgHostCsr"}


def c_field_name(field):
    """The C name of a mirrored field: Python keywords carry a trailing '_'."""
    import keyword
    return field[:-1] if field.endswith("_") and keyword.iskeyword(field[:-1]) else field


def test_binding_structs_have_the_c_layout(tmp_path):
    """Size and every field offset of each ctypes mirror equal the C struct's,
    as gcc lays it out from the header."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"',
             "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        cls = getattr(_capi, pyname)
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            cfield = c_field_name(field)
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {cfield}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        cname, what, value = line.split()
        cls = getattr(_capi, STRUCTS[cname])
        got = ctypes.sizeof(cls) if what == "size" else getattr(cls, what).offset
        assert got == int(value), (cname, what, got, value)
    # every C field is mirrored (the C program only names mirrored fields, so
    # a C field missing from the mirror shows up as a size difference above)


def test_cli_errors_before_the_device(golden_dir, tmp_path):
    """The CLI's argument and input errors: one line on stderr, exit 1, found
    before any device work (so they hold on a machine without a GPU)."""
    import subprocess
    cli = _capi.CLI_PATH
    lap = os.path.join(golden_dir, "laplace2d_64.csr")
    p = subprocess.run([cli], capture_output=True, text=True)
    assert p.returncode == 1 and p.stderr.startswith("usage:")
    p = subprocess.run([cli, "t", lap, "AtA"], capture_output=True, text=True)
    assert p.returncode == 1 and "task must be AA, AAt or AAtS" in p.stderr and not p.stdout
    p = subprocess.run([cli, "t", str(tmp_path / "missing.csr"), "AA"], capture_output=True,
                       text=True)
    assert p.returncode == 1 and p.stderr.startswith("spgemm_b200: read:") and not p.stdout


def test_no_gpu_means_errors_not_a_cpu_fallback():
    """Without a usable CUDA device every product entry point fails loudly —
    a status from the C ABI, an exception from Python — and nothing is
    computed on the host instead."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from appt_spgemm_b200.engine import Engine
    L = _capi.lib()
    ctx = ctypes.c_void_p()
    assert L.spg_create(ctypes.byref(ctx), None) == _capi.SPG_ERR_CUDA
    assert not ctx.value
    r = _capi.SpgEngResult()
    assert L.spg_run_ours(b"AA", None, None, None, 0, 0, 1, ctypes.byref(r)) == _capi.SPG_ERR_CUDA
    assert b"cuda" in L.spg_last_error_string().lower()
    with pytest.raises(RuntimeError):
        Engine("cuda:0")


def test_batch_mix_follows_its_recipe():
    """The batched workload's generator: n log-uniform in [1k, 64k), banded and
    Erdős–Rényi matrices alternating, their parameters in range, values in
    [−1, 1), valid CSR, and the same seed gives the same matrices."""
    mats, params = csr.batch_mix(64, seed=4)
    assert len(mats) == len(params) == 64
    for b, (A, p) in enumerate(zip(mats, params)):
        A.validate()
        assert A.n == p["n"] and 1000 <= A.n < 64000
        assert p["kind"] == ("banded" if b % 2 == 0 else "er")
        if p["kind"] == "banded":
            assert 3 <= p["bw"] <= 64
            rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
            assert np.abs(rows - A.col).max() <= p["bw"]
            assert (rows == A.col).sum() == A.n  # diagonal always present
        else:
            assert 4.0 <= p["lambda"] < 32.0
        assert A.val.min() >= -1.0 and A.val.max() < 1.0
    ns = np.array([p["n"] for p in params])
    assert ns.min() < 4000 and ns.max() > 16000  # spread over the log range
    again, _ = csr.batch_mix(8, seed=4)
    for A, B in zip(mats[:8], again):
        assert np.array_equal(A.col, B.col) and np.array_equal(A.val, B.val)
