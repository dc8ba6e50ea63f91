"""GPU parity at the sizes of the benchmark configurations.

The small parity cases (test_parity_gpu.py) compare whole outputs with the
oracle.  Here the products are the configurations the benchmark runs, and the
check is against the reference's own kernels (fukien/contention-aware-spgemm
built from its sources into oracle/_ref), rows sorted:

* G500 R-MAT scale 17, edge factor 8 (seed 17): the whole C, bit for bit, for
  all three accumulators (row pointers, columns, values).  About 5.1e8
  output entries; the reference runs the whole product in seconds.
* Uniform (ER) R-MAT scale 21, edge factor 32 (seed 21): C has 8.6e9 entries
  (103 GB), more than the host can hold in the reference's layout.  Rows of C
  are independent, so the reference runs on three row blocks (start, middle,
  end) of about 1e8 products each, and each block's row digests (the
  cas_csr_digest row form, computed by the oracle after sorting the rows) must
  equal the GPU product's row digests of the same rows.
* Zipf bipartite 850,000 x 2,000,000 (12 M nonzeros, column offset 1000,
  seed 3): the same three-block check, with B its explicit transpose.
"""
import numpy as np
import pytest

import casgemm
import oracle

pytestmark = pytest.mark.gpu

BLOCK_PRODUCTS = 100_000_000


def _need_ref():
    if not oracle.ref_available("hybacc", small=False):
        pytest.skip("oracle/_ref not built")


def _device_csr(M):
    import torch
    t = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (M.row_ptrs, M.cols, M.vals)]
    return casgemm.DeviceCsr(M.num_row, M.num_col, M.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                             M.val_type, keep=t)


def _blocks(ps, block_products):
    """Three row blocks [r0, r1) at the start, middle and end of the product prefix."""
    m = len(ps) - 1
    total = int(ps[-1])
    out = []
    for start in (0, total // 2, max(0, total - block_products)):
        r0 = min(int(np.searchsorted(ps, start, side="left")), m - 1)
        r1 = int(np.searchsorted(ps, int(ps[r0]) + block_products, side="left"))
        out.append((r0, max(r0 + 1, min(r1, m))))
    return out


def _check_blocks(ctx, A, B):
    dA, dB = _device_csr(A), _device_csr(B)
    cc, _ = ctx.spgemm_device(dA, dB, "hybacc")
    try:
        _, gpu_rows = ctx.digest(cc, rows=True)
        nnz_gpu = cc.num_nnz
    finally:
        ctx.free(cc)
    ps = casgemm.row_products_prefix(A, B)
    assert ctx.stats()["flop"] == int(ps[-1])
    assert nnz_gpu == ctx.stats()["nnz_c"]
    for r0, r1 in _blocks(ps, BLOCK_PRODUCTS):
        res = oracle.ref_row_digests(casgemm.slice_rows(A, r0, r1), B, "hybacc", small=True)
        assert res is not None
        rp, rows, _, _ = res
        assert int(rp[-1]) > 0
        bad = np.nonzero(rows != gpu_rows[r0:r1])[0]
        assert len(bad) == 0, f"rows [{r0},{r1}): {len(bad)} row digests differ, first row {r0 + int(bad[0])}"


def test_g500_s17_ef8_whole_product_bit_for_bit(ctx):
    _need_ref()
    A = casgemm.gen_g500(17, 8, 17)
    ref = oracle.ref_spgemm(A, A, "hybacc", small=False)
    assert ref is not None
    rp, cols, vals = ref[0], ref[1], ref[2]
    assert len(cols) > 5e8
    for algo in ("hybacc", "hash", "hsersc"):
        out = ctx.spgemm(A, A, algo)
        assert np.array_equal(out.csr.row_ptrs, rp), algo
        assert np.array_equal(out.csr.cols, cols), algo
        assert np.array_equal(out.csr.vals, vals), algo
        assert out.stats["flop"] == casgemm.intprod(A, A)
        del out


def test_er_s21_ef32_row_blocks_match_reference(ctx):
    _need_ref()
    A = casgemm.gen_er(21, 32, 21)
    _check_blocks(ctx, A, A)


def test_zipf_850k_row_blocks_match_reference(ctx):
    _need_ref()
    A = casgemm.gen_zipf(850000, 2000000, 50000, 12000000, 3, col_q=1000.0)
    _check_blocks(ctx, A, A.transpose())
