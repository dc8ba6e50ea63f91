"""Regenerate the golden fixtures in this directory from the reference itself.

Every fixture's C was computed by the reference's own kernels
(fukien/contention-aware-spgemm built from its sources into oracle/_ref with
oracle/Makefile), for all three of its accumulators (hash, hsersc, hybacc),
which must agree once each row is sorted by column.  Inputs come from the
project's seeded generators, so the fixtures pin the whole chain: inputs,
reference output, and the oracle restatement checked against them in
tests/test_oracle.py.

The MatrixMarket fixture pins the loader: `loader_sym.mtx` read by the
reference's raw2csr (src/mm/mm_utils.c:451-692).

The driver fixtures pin the process boundary: `rmat_ones/` holds a small
PaRMAT-style edge list and the two files the reference's rmat_ones
(src/rmat_ones.c) writes from it; `driver_<algo>_g500_12_8.log` is the
stdout of the reference's ams_<algo>spgemm driver (built with IN_VERIFY) on
the dataset `bin/cas_gen g500 12 8` writes, whose VERIFYRESULT triple and
line layout the GPU drivers must reproduce.

Run from the repository root, where oracle/_ref has been built:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "contention-aware-spgemm_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import shutil  # noqa: E402
import subprocess  # noqa: E402
import tempfile  # noqa: E402

import casgemm  # noqa: E402
import oracle  # noqa: E402
from matrices import from_coo, with_int_values  # noqa: E402


def cases():
    rng = np.random.default_rng(11)
    out = {}
    A = casgemm.gen_g500(8, 8, 8)
    out["g500_s8_ef8"] = (A, A.transpose())
    A = casgemm.gen_er(8, 16, 9)
    out["er_s8_ef16"] = (A, A.transpose())
    A = with_int_values(casgemm.gen_g500(9, 4, 10), 77)
    out["g500_s9_ef4_int"] = (A, A.transpose())
    Z = casgemm.gen_zipf(600, 3000, 200, 5000, 12, col_q=20.0)
    out["zipf_600x3000"] = (Z, Z.transpose())
    n = 400
    r = np.concatenate([np.zeros(n, np.int64), np.arange(n), rng.integers(0, n, 600)])
    c = np.concatenate([np.arange(n), np.zeros(n, np.int64), rng.integers(0, n, 600)])
    key = np.unique(r * n + c)
    D = from_coo(n, n, key // n, key % n)
    out["dense_row_hot_col"] = (D, D.transpose())
    U = from_coo(200, 40, rng.integers(0, 200, 1500), rng.integers(0, 40, 1500))
    out["duplicates_ncol40"] = (U, U.transpose())
    G = from_coo(150, 220, rng.integers(0, 150, 900), rng.integers(0, 220, 900),
                 rng.integers(1, 9, 900).astype(np.float64))
    H = from_coo(220, 500, rng.integers(0, 220, 1800), rng.integers(0, 500, 1800),
                 rng.integers(-3, 4, 1800).astype(np.float64))
    out["general_AB_int"] = (G, H)
    return out


def main():
    for name, (A, B) in cases().items():
        res = {}
        for algo in ("hash", "hsersc", "hybacc"):
            r = oracle.ref_spgemm(A, B, algo, small=True)
            assert r is not None, f"{name}: input below one morsel of the small build"
            res[algo] = r
        base = res["hybacc"]
        for algo, r in res.items():
            for i in range(3):
                assert np.array_equal(r[i], base[i]), f"{name}: reference {algo} disagrees with hybacc"
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            a_shape=np.array([A.num_row, A.num_col]), a_rp=A.row_ptrs, a_cols=A.cols, a_vals=A.vals,
            b_shape=np.array([B.num_row, B.num_col]), b_rp=B.row_ptrs, b_cols=B.cols, b_vals=B.vals,
            c_rp=base[0], c_cols=base[1].astype(np.int32), c_vals=base[2],
            flop=np.array([casgemm.intprod(A, B)]))
        print(f"{name}: nnz(A)={A.nnz} nnz(C)={len(base[1])}")
    # MatrixMarket loader: symmetric file with an explicit zero, a duplicate,
    # a diagonal entry, a two-column (pattern) line and a non-unit value
    mtx = os.path.join(HERE, "loader_sym.mtx")
    with open(mtx, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n% comment line\n")
        f.write("5 5 8\n1 1 2.5\n2 1 1.0\n3 2 0.0\n4 3 7.0\n4 3 7.0\n5 5\n5 1 -1.0\n3 3 1.0\n")
    nr, nc, rp, cols, vals = oracle.ref_load_mtx(mtx)
    np.savez_compressed(os.path.join(HERE, "loader_sym.npz"), shape=np.array([nr, nc]), rp=rp, cols=cols, vals=vals)
    print(f"loader_sym: {nr}x{nc} nnz={len(cols)}")


def driver_fixtures():
    ref = os.path.join(ROOT, "oracle", "_ref")
    gen = os.path.join(ROOT, "contention-aware-spgemm_b200", "bin", "cas_gen")
    with tempfile.TemporaryDirectory() as tmp:
        ds = os.path.join(tmp, "dataset")
        os.makedirs(ds)
        # edge list: each undirected edge of a seeded R-MAT once, 0-based
        A = casgemm.gen_g500(4, 2, 5)
        rows = np.repeat(np.arange(A.num_row), np.diff(A.row_ptrs))
        keep = rows < A.cols
        edges = "".join(f"{u}\t{v}\n" for u, v in zip(rows[keep], A.cols[keep]))
        open(os.path.join(ds, "g500_4_2.txt"), "w").write(edges)
        subprocess.run([os.path.join(ref, "rmat_ones"), "g500_4_2"], cwd=tmp, check=True, capture_output=True)
        out = os.path.join(HERE, "rmat_ones")
        os.makedirs(out, exist_ok=True)
        for suffix in (".txt", ".org.mtx", ".trs.mtx"):
            shutil.copy(os.path.join(ds, "g500_4_2" + suffix), os.path.join(out, "g500_4_2" + suffix))
        subprocess.run([gen, "g500", "12", "8"], cwd=tmp, check=True, capture_output=True,
                       env=dict(os.environ, CAS_DATASET_DIR=ds))
        for algo in ("hash", "hsersc", "hybacc"):
            p = subprocess.run([os.path.join(ref, f"ams_{algo}spgemm"), "g500_12_8"], cwd=tmp, check=True,
                               capture_output=True, text=True)
            open(os.path.join(HERE, f"driver_{algo}_g500_12_8.log"), "w").write(p.stdout)
            print(f"driver_{algo}: {sum(1 for x in p.stdout.splitlines() if x.startswith('VERIFYRESULT'))} verify lines")


if __name__ == "__main__":
    main()
    driver_fixtures()
