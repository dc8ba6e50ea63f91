"""GPU: B = A^T made on the device (cas_csr_transpose).

The reference reads B from <dataset>.trs.mtx, which its trpl_transpose
(src/mm/mm_utils.c:742-754) writes from the same triples as A sorted by
(row, column).  The device transpose must equal the host's stable
counting-sort transpose (casgemm.transpose) entry for entry: row pointers,
columns and values, with duplicate (row, column) entries in A's order.
Cases: uniform and skewed R-MAT graphs, a rectangular Zipf matrix with hot
columns, a column with 50,000 entries (several tiles and radix passes in the
long-row sort), duplicates with distinct integer values, an empty matrix,
and a device input whose column leaves the matrix.
"""
import numpy as np
import pytest

import casgemm
from matrices import from_coo, with_int_values

pytestmark = pytest.mark.gpu


def same(got, want):
    assert got.num_row == want.num_row and got.num_col == want.num_col
    np.testing.assert_array_equal(got.row_ptrs, want.row_ptrs)
    np.testing.assert_array_equal(got.cols, want.cols)
    np.testing.assert_array_equal(got.vals, want.vals)


def _giant_column():
    rng = np.random.default_rng(4)
    n_rows, n_cols = 60000, 5000
    r = np.concatenate([np.arange(50000), rng.integers(0, n_rows, 90000)])
    c = np.concatenate([np.zeros(50000, np.int64), rng.integers(1, n_cols, 90000)])
    key = np.unique(r * n_cols + c)
    return from_coo(n_rows, n_cols, key // n_cols, key % n_cols, rng.normal(size=len(key)))


def _duplicates():
    rng = np.random.default_rng(6)
    r = rng.integers(0, 400, 6000)
    c = rng.integers(0, 60, 6000)
    return from_coo(400, 60, r, c, rng.integers(1, 9, 6000).astype(np.int32), dtype=np.int32)


CASES = {
    "er_s13_ef32": lambda: casgemm.gen_er(13, 32, 3),
    "g500_s15_ef16": lambda: casgemm.gen_g500(15, 16, 5),
    "zipf_20000x60000": lambda: casgemm.gen_zipf(20000, 60000, 4000, 200000, 9, col_q=20.0),
    "giant_column": _giant_column,
    "duplicates_int": _duplicates,
    "g500_int": lambda: with_int_values(casgemm.gen_g500(12, 8, 2), 3),
    "empty": lambda: from_coo(30, 70, [], []),
}


class _DevView:
    """A zero-copy view of a device array for torch (__cuda_array_interface__)."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False), "version": 3}


def _fetch(ptr, count, dtype):
    import torch
    if count == 0:
        return np.zeros(0, dtype)
    t = torch.as_tensor(_DevView(ptr, count, np.dtype(dtype).str), device="cuda")
    return t.cpu().numpy().copy()


def _device_to_host(cb):
    vt = np.float64 if cb.val_type == casgemm.VAL_F64 else np.int32
    return casgemm.Csr(cb.num_row, cb.num_col, _fetch(cb.row_ptrs, cb.num_row + 1, np.int64),
                       _fetch(cb.cols, cb.num_nnz, np.int32), _fetch(cb.rats, cb.num_nnz, vt))


@pytest.mark.parametrize("name", sorted(CASES))
def test_transpose_equals_host(ctx, name):
    A = CASES[name]()
    want = casgemm.transpose(A)
    same(ctx.transpose(A), want)             # host input, host output
    if A.nnz:                                # device input, device output
        dB = ctx.transpose_device(casgemm.DeviceCsr.upload(A))
        try:
            got = _device_to_host(dB)
        finally:
            ctx.free(dB)
        same(got, want)


def test_transpose_rejects_columns_out_of_range(ctx):
    import torch
    A = casgemm.gen_g500(8, 4, 1)
    cols = A.cols.copy()
    cols[3] = A.num_col + 5
    t = [torch.from_numpy(x).cuda() for x in (A.row_ptrs, cols, A.vals)]
    dA = casgemm.DeviceCsr(A.num_row, A.num_col, A.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), keep=t)
    with pytest.raises(casgemm.CasError):
        ctx.transpose_device(dA)


def test_product_with_device_transpose(ctx):
    """C = A * B with B = A^T made on the device equals C with the host's B."""
    A = casgemm.gen_g500(13, 8, 21)
    want = ctx.spgemm(A, casgemm.transpose(A), "hybacc")
    got = ctx.spgemm(A, ctx.transpose(A), "hybacc")
    np.testing.assert_array_equal(got.csr.row_ptrs, want.csr.row_ptrs)
    np.testing.assert_array_equal(got.csr.cols, want.csr.cols)
    np.testing.assert_array_equal(got.csr.vals, want.csr.vals)
