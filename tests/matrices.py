"""Seeded test matrices (small enough for the CPU oracle to finish in seconds)."""
import numpy as np

import casgemm
from casgemm import Csr


def from_coo(nr, nc, rows, cols, vals=None, dtype=np.float64) -> Csr:
    """CSR with entries sorted by (row, col); duplicates kept, as the reference loader does."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    if vals is None:
        vals = np.ones(len(rows), dtype)
    vals = np.asarray(vals, dtype)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rp = np.zeros(nr + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp)
    return Csr(nr, nc, rp, cols.astype(np.int32), vals)


def with_int_values(A: Csr, seed: int) -> Csr:
    return Csr(A.num_row, A.num_col, A.row_ptrs, A.cols, casgemm.int_values(A.nnz, seed))


def cases():
    """(name, A, B) pairs covering the shapes the reference's drivers meet and the edge cases."""
    out = []
    for s, ef in [(6, 2), (8, 4), (10, 8), (12, 8), (12, 16)]:
        A = casgemm.gen_g500(s, ef, 100 + s)
        out.append((f"g500_s{s}_ef{ef}", A, A.transpose()))
    for s, ef in [(10, 4), (12, 32), (13, 32)]:
        A = casgemm.gen_er(s, ef, 200 + s)
        out.append((f"er_s{s}_ef{ef}", A, A.transpose()))
    Z = casgemm.gen_zipf(4000, 20000, 800, 40000, 7, col_q=50.0)
    out.append(("zipf_4000x20000", Z, Z.transpose()))
    rng = np.random.default_rng(5)
    # empty matrix
    E = from_coo(50, 40, [], [])
    out.append(("empty", E, E.transpose()))
    # one dense row and one dense column (hot column): heavy rows on both sides
    n = 3000
    r = np.concatenate([np.zeros(n, np.int64), np.arange(n), rng.integers(0, n, 4000)])
    c = np.concatenate([np.arange(n), np.zeros(n, np.int64), rng.integers(0, n, 4000)])
    key = np.unique(r * n + c)
    D = from_coo(n, n, key // n, key % n)
    out.append(("dense_row_hot_col", D, D.transpose()))
    # duplicates inside rows (kept by the loader, both contribute)
    rr = rng.integers(0, 300, 3000)
    cc = rng.integers(0, 50, 3000)
    U = from_coo(300, 50, rr, cc)
    out.append(("duplicates_ncol50", U, U.transpose()))
    # rectangular general A*B with B independent of A, ragged rows
    G = from_coo(700, 900, rng.integers(0, 700, 9000), rng.integers(0, 900, 9000), rng.integers(1, 9, 9000).astype(np.float64))
    H = from_coo(900, 5000, rng.integers(0, 900, 20000), rng.integers(0, 5000, 20000), rng.normal(size=20000))
    out.append(("general_AB", G, H))
    return out
