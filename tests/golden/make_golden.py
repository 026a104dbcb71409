"""Generate the golden fixtures from the reference's own Python code.

Run in a container where the reference tree is mounted (read-only), giving its
root in the required variable REFERENCE_ROOT:

    REFERENCE_ROOT=<reference tree> python tests/golden/make_golden.py

For a set of small matrices built by this project's generators it records,
using the reference's functions unmodified:
  - the CSR1 file written by write_bin (src/export_bin.py:20-29), committed as
    <name>.csr so the engine's reader/writer are checked byte for byte;
  - checksum(A@A) and checksum(A@A.T) (src/export_bin.py:31-35, :46-47): the
    scipy product's nnz (numeric semantics: exact zeros pruned) and Σv, Σ|v|,
    Σv² — the reference's correctness convention for this path;
  - the structural nnz (scipy product of the 0/1 patterns, nothing cancels);
  - the product counts est_outputs (bench/run_baseline.py:38-44).
The fixtures (golden.json + *.csr) need no reference tree at test time.
"""
import importlib.util
import json
import os
import pathlib
import sys
from unittest import mock

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("REFERENCE_ROOT")
if not REF or not os.path.isdir(REF):
    sys.exit("make_golden.py: set REFERENCE_ROOT to the reference tree's root")
sys.path.insert(0, REPO)

from appt_spgemm_b200 import csr  # noqa: E402


def load_ref_module(rel):
    """Import a reference script by path; its module-level mkdir calls (which
    would write into the read-only tree) are turned into no-ops."""
    path = os.path.join(REF, rel)
    spec = importlib.util.spec_from_file_location("ref_" + rel.replace("/", "_")[:-3], path)
    mod = importlib.util.module_from_spec(spec)
    with mock.patch.object(pathlib.Path, "mkdir", lambda *a, **k: None):
        spec.loader.exec_module(mod)
    return mod


def cases():
    yield "laplace2d_64", csr.laplace2d(64)
    yield "stencil27_6", csr.stencil27(6, seed=2)
    yield "uniform_300x7", csr.uniform(300, 7, seed=11)
    yield "banded_500_bw8", csr.banded(500, 8, 0.3, seed=12)
    yield "er_400_l6", csr.erdos_renyi(400, 6.0, seed=13)
    yield "rmat_s9_ef8", csr.rmat(9, 8, seed=14)
    # empty rows and columns, one dense row, one dense column
    n = 64
    rows, cols = [], []
    for j in range(0, n, 1):
        rows.append(5); cols.append(j)
        rows.append(j); cols.append(40)
    rows += [9, 9, 63]; cols += [0, 63, 63]
    M = sp.coo_matrix((np.linspace(-1.5, 2.0, len(rows)), (rows, cols)), shape=(n, n)).tocsr()
    M.sum_duplicates(); M.sort_indices()
    yield "edge_dense_row_col", csr.CsrHost(n, M.indptr.astype(np.int32),
                                            M.indices.astype(np.int32), M.data.copy())


def main():
    export_bin = load_ref_module("src/export_bin.py")
    run_baseline = load_ref_module("bench/run_baseline.py")
    out = {"generated_by": "tests/golden/make_golden.py",
           "reference_functions": ["src/export_bin.py:write_bin", "src/export_bin.py:checksum",
                                   "bench/run_baseline.py:est_outputs"],
           "cases": {}}
    for name, A in cases():
        S = A.to_scipy()
        export_bin.write_bin(S, os.path.join(HERE, name + ".csr"))
        P = S.copy()
        P.data[:] = 1.0
        entry = {"n": A.n, "nnz": A.nnz}
        est_aa, est_aat = run_baseline.est_outputs(S)
        entry["products"] = {"AA": int(est_aa), "AAt": int(est_aat)}
        for task, prod, pat in (("AA", S @ S, P @ P), ("AAt", S @ S.T, P @ P.T)):
            nnz, s, a, q = export_bin.checksum(prod)
            entry[task] = {"nnz_scipy": int(nnz), "nnz_structural": int(pat.nnz),
                           "sum": s, "abssum": a, "sq": q}
        out["cases"][name] = entry
        print(name, entry["AA"]["nnz_structural"], entry["AAt"]["nnz_structural"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
