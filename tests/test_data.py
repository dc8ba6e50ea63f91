"""CPU: the data layer — seeded generators, CSR helpers, MatrixMarket I/O."""
import os

import numpy as np
import pytest

import casgemm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _check_graph(A, n, n_edges):
    assert A.num_row == A.num_col == n
    assert A.nnz == 2 * n_edges
    S = A.to_scipy()
    assert (S != S.T).nnz == 0, "not symmetric"
    assert S.diagonal().sum() == 0, "self-loops"
    for i in range(0, n, max(1, n // 64)):
        row = A.cols[A.row_ptrs[i]:A.row_ptrs[i + 1]]
        assert np.all(np.diff(row) > 0), "row not strictly increasing (duplicate or unsorted)"


@pytest.mark.parametrize("scale,ef", [(8, 2), (10, 8), (12, 16)])
def test_g500_rmat(scale, ef):
    A = casgemm.gen_g500(scale, ef, 17)
    _check_graph(A, 1 << scale, ef << scale)
    deg = np.diff(A.row_ptrs)
    assert deg.max() > 8 * deg.mean(), "R-MAT skew missing"
    B = casgemm.gen_g500(scale, ef, 17)
    assert np.array_equal(A.row_ptrs, B.row_ptrs) and np.array_equal(A.cols, B.cols)
    C = casgemm.gen_g500(scale, ef, 18)
    assert not np.array_equal(A.cols[: min(len(A.cols), len(C.cols))], C.cols[: min(len(A.cols), len(C.cols))])


def test_er_rmat_is_balanced():
    A = casgemm.gen_er(12, 32, 21)
    _check_graph(A, 1 << 12, 32 << 12)
    deg = np.diff(A.row_ptrs)
    assert deg.max() < 3 * deg.mean()


def test_generator_independent_of_thread_count():
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import casgemm, hashlib; A = casgemm.gen_g500(11, 8, 5); "
            "print(hashlib.sha1(A.cols.tobytes()).hexdigest())" % os.path.dirname(casgemm.__file__))
    outs = set()
    for t in ("1", "3"):
        env = dict(os.environ, OMP_NUM_THREADS=t)
        outs.add(subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                                check=True).stdout.strip())
    assert len(outs) == 1


def test_zipf_bipartite():
    nr, nc, amax, target = 3000, 20000, 600, 30000
    Z = casgemm.gen_zipf(nr, nc, amax, target, 9, col_q=50.0)
    assert Z.num_row == nr and Z.num_col == nc
    deg = np.diff(Z.row_ptrs)
    assert abs(Z.nnz - target) <= nr  # rounding of the rank law
    assert deg.max() == amax and deg.min() >= 1
    for i in range(0, nr, 97):
        row = Z.cols[Z.row_ptrs[i]:Z.row_ptrs[i + 1]]
        assert np.all(np.diff(row) > 0)
    colcount = np.bincount(Z.cols, minlength=nc)
    assert colcount[:100].sum() > colcount[-100:].sum() * 5, "column popularity not skewed"


def test_transpose_and_intprod():
    Z = casgemm.gen_zipf(500, 900, 120, 4000, 3, col_q=5.0)
    T = Z.transpose()
    assert (T.to_scipy() != Z.to_scipy().T).nnz == 0
    cnt = np.diff(T.row_ptrs)[Z.cols].sum()
    assert casgemm.intprod(Z, T) == cnt


def test_int_values_range_and_seed():
    v = casgemm.int_values(10000, 4)
    assert v.dtype == np.int32 and v.min() == 1 and v.max() == 8
    assert np.array_equal(v, casgemm.int_values(10000, 4))


def test_mtx_loader_matches_reference_loader():
    """cas_mtx_read against the reference's raw2csr on the same file (golden)."""
    z = np.load(os.path.join(GOLDEN, "loader_sym.npz"))
    M = casgemm.mtx_read(os.path.join(GOLDEN, "loader_sym.mtx"))
    assert [M.num_row, M.num_col] == list(z["shape"])
    np.testing.assert_array_equal(M.row_ptrs, z["rp"])
    np.testing.assert_array_equal(M.cols.astype(np.int64), z["cols"])
    np.testing.assert_array_equal(M.vals, z["vals"])


def test_mtx_roundtrip(tmp_path):
    A = casgemm.gen_g500(9, 4, 2)
    p = str(tmp_path / "a.org.mtx")
    casgemm.mtx_write(p, A, symmetric=True)
    B = casgemm.mtx_read(p)
    np.testing.assert_array_equal(A.row_ptrs, B.row_ptrs)
    np.testing.assert_array_equal(A.cols, B.cols)
    assert np.all(B.vals == 1.0)
    Z = casgemm.gen_zipf(300, 700, 60, 2000, 4, col_q=5.0)
    q = str(tmp_path / "z.trs.mtx")
    casgemm.mtx_write(q, Z.transpose(), symmetric=False)
    T = casgemm.mtx_read(q)
    assert (T.to_scipy() != Z.to_scipy().T).nnz == 0


def test_binary_csr_cache_roundtrip(tmp_path):
    Z = casgemm.gen_zipf(400, 900, 80, 3000, 6, col_q=5.0)
    p = str(tmp_path / "z.csr")
    casgemm.csr_write_bin(p, Z)
    R = casgemm.csr_read_bin(p)
    assert (R.num_row, R.num_col) == (Z.num_row, Z.num_col)
    np.testing.assert_array_equal(R.row_ptrs, Z.row_ptrs)
    np.testing.assert_array_equal(R.cols, Z.cols)
    np.testing.assert_array_equal(R.vals, Z.vals)
    open(p, "r+b").write(b"XX")  # a damaged header is refused, not misread
    with pytest.raises(ValueError):
        casgemm.csr_read_bin(p)
