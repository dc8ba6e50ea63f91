"""CPU: the oracle restatement, pinned against the reference.

* the committed golden fixtures (C computed by the reference's own kernels,
  tests/golden/make_golden.py) for all three accumulators;
* the reference itself, live, where oracle/_ref has been built;
* scipy for real-valued inputs, and the pieces of the restatement
  (radix sort, hash symbolic, morsel packing) on their own.
"""
import glob
import os

import numpy as np
import pytest

import casgemm
import oracle
from matrices import from_coo

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz")) if not p.endswith("loader_sym.npz"))


def load_fixture(path):
    z = np.load(path)
    A = casgemm.Csr(int(z["a_shape"][0]), int(z["a_shape"][1]), z["a_rp"], z["a_cols"], z["a_vals"])
    B = casgemm.Csr(int(z["b_shape"][0]), int(z["b_shape"][1]), z["b_rp"], z["b_cols"], z["b_vals"])
    return A, B, (z["c_rp"], z["c_cols"].astype(np.int64), z["c_vals"]), int(z["flop"][0])


def test_fixtures_present():
    assert len(FIXTURES) >= 7


@pytest.mark.parametrize("algo", ["hash", "hsersc", "hybacc"])
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_matches_golden(path, algo):
    A, B, C, flop = load_fixture(path)
    rp, cols, vals, f = oracle.oracle_spgemm(A, B, algo)
    assert f == flop
    np.testing.assert_array_equal(rp, C[0])
    np.testing.assert_array_equal(cols, C[1])
    np.testing.assert_array_equal(vals, C[2])


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("algo", ["hash", "hsersc", "hybacc"])
def test_oracle_matches_reference_live(algo):
    mats = [casgemm.gen_g500(11, 8, 3), casgemm.gen_er(10, 16, 4), casgemm.gen_zipf(2000, 9000, 500, 20000, 5, col_q=30.0)]
    for A in mats:
        B = A.transpose()
        ref = oracle.ref_spgemm(A, B, algo, small=True)
        got = oracle.oracle_spgemm(A, B, algo)
        for i in range(3):
            np.testing.assert_array_equal(got[i], ref[i])


def test_hash_rows_unsorted_but_same_set():
    """The hash accumulator emits slot order (src/ams/ams_utils.c:301-309); sorted it equals ESC's rows."""
    A = casgemm.gen_g500(9, 8, 21)
    B = A.transpose()
    h = oracle.oracle_spgemm(A, B, "hash", sort=False)
    e = oracle.oracle_spgemm(A, B, "hsersc", sort=False)
    unsorted_rows = sum(np.any(np.diff(h[1][h[0][i]:h[0][i + 1]]) < 0) for i in range(A.num_row))
    assert unsorted_rows > 0
    hs = oracle.sort_rows(*h[:3])
    np.testing.assert_array_equal(hs[1], e[1])
    np.testing.assert_array_equal(hs[2], e[2])


def test_oracle_matches_scipy_real_values():
    rng = np.random.default_rng(3)
    G = from_coo(300, 400, rng.integers(0, 300, 3000), rng.integers(0, 400, 3000), rng.normal(size=3000))
    H = from_coo(400, 250, rng.integers(0, 400, 3000), rng.integers(0, 250, 3000), rng.normal(size=3000))
    C = (G.to_scipy() @ H.to_scipy()).tocsr()
    C.sort_indices()
    for algo in ("hash", "hsersc", "hybacc"):
        rp, cols, vals, _ = oracle.oracle_spgemm(G, H, algo)
        # structural nonzeros: scipy may drop exact cancellations, the reference keeps them
        S = casgemm.Csr(300, 250, rp, cols, vals).to_scipy()
        np.testing.assert_allclose((S - C).toarray(), 0.0, atol=1e-12)
        assert len(cols) >= C.nnz


def test_radix_sort_restatement_is_stable():
    import ctypes
    lib = oracle.oracle_lib()
    rng = np.random.default_rng(0)
    keys = rng.integers(0, 70000, 5000).astype(np.int64)
    vals = np.arange(5000, dtype=np.float64)
    k, v = keys.copy(), vals.copy()
    ak, av = np.empty_like(k), np.empty_like(v)
    lib.orc_radix_sort_kv(k.ctypes.data, v.ctypes.data, ak.ctypes.data, av.ctypes.data, len(k))
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(k, keys[order])
    np.testing.assert_array_equal(v, vals[order])


def test_hash_symbolic_counts():
    import ctypes
    lib = oracle.oracle_lib()
    A = casgemm.gen_zipf(800, 3000, 300, 8000, 9, col_q=10.0)
    B = A.transpose()
    a, ka = oracle.to_orc(A.row_ptrs, A.cols, A.vals, A.num_col)
    b, kb = oracle.to_orc(B.row_ptrs, B.cols, B.vals, B.num_col)
    flp = np.zeros(A.num_row, np.int64)
    nz = np.zeros(A.num_row, np.int64)
    lib.orc_flp_populate(ctypes.byref(a), ctypes.byref(b), flp.ctypes.data)
    lib.orc_hash_symb(ctypes.byref(a), ctypes.byref(b), flp.ctypes.data, nz.ctypes.data)
    S = A.to_scipy()
    C = (S @ B.to_scipy()).tocsr()
    np.testing.assert_array_equal(nz, np.diff(C.indptr))
    assert flp.sum() == casgemm.intprod(A, B)


def test_pack_morsels_properties():
    """Morsels of pack_ams_pack (src/ams/ams_utils.c:1410-1596)."""
    import ctypes
    lib = oracle.oracle_lib()
    A = casgemm.gen_g500(10, 8, 5)
    B = A.transpose()
    cnt = np.concatenate([[0], np.cumsum(np.diff(B.row_ptrs)[A.cols])])
    row_flp = (cnt[A.row_ptrs[1:]] - cnt[A.row_ptrs[:-1]]).astype(np.int64)
    ps_flp = np.concatenate([[0], np.cumsum(row_flp)]).astype(np.int64)
    ps_w = A.row_ptrs.astype(np.int64)
    morsel = 256
    total = int(ps_w[-1]) // morsel
    bounds = np.zeros(total + 1, np.int64)
    cf = np.zeros(total, np.float64)
    mx = np.zeros(total, np.int64)
    order = np.zeros(total, np.int64)
    lh, ht = ctypes.c_int64(), ctypes.c_int64()
    t = lib.orc_pack_morsels(A.num_row, ps_w.ctypes.data, row_flp.ctypes.data, ps_flp.ctypes.data, morsel, 0.85,
                             bounds.ctypes.data, cf.ctypes.data, mx.ctypes.data, order.ctypes.data,
                             ctypes.byref(lh), ctypes.byref(ht))
    assert t == total
    assert bounds[0] == 0 and bounds[-1] == A.num_row and np.all(np.diff(bounds) >= 0)
    nonempty = np.diff(bounds) > 0
    assert lh.value == int((~nonempty).sum())
    keyed = sorted(range(total), key=lambda j: (cf[j], j))
    np.testing.assert_array_equal(order, keyed)
    for j in np.nonzero(nonempty)[0][:50]:
        s, e = bounds[j], bounds[j + 1]
        assert mx[j] == row_flp[s:e].max()
        assert cf[j] == pytest.approx((ps_flp[e] - ps_flp[s]) / (ps_w[e] - ps_w[s]))
