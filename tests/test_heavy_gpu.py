"""GPU: the heaviest dense rows split across thread blocks.

Dense rows of 2^17 products or more are cut into parts by A-entry ranges of
about equal products; the parts add into C by atomics after one block per
row has written its columns (cas_tuning.heavy_split).  The output must equal
the oracle's bit for bit, and the product with the split off: an R-MAT graph
with 15 such rows, the same with integer values, and a 700,000 x 400,000
Zipf matrix whose heavy rows span two 512 Ki-column slices.
"""
import numpy as np
import pytest

import casgemm
import oracle
from matrices import with_int_values

pytestmark = pytest.mark.gpu


def _cases():
    g = casgemm.gen_g500(14, 16, 7)
    z = casgemm.gen_zipf(700000, 400000, 30000, 1500000, 6, col_q=1000.0)
    return {"g500_s14_ef16": (g, g.transpose()), "g500_s14_ef16_int": (with_int_values(g, 5),
                                                                        with_int_values(g, 5).transpose()),
            "zipf_700k_two_slices": (z, z.transpose())}


@pytest.mark.parametrize("name", ["g500_s14_ef16", "g500_s14_ef16_int", "zipf_700k_two_slices"])
def test_split_rows_match_oracle(ctx, name):
    A, B = _cases()[name]
    P = np.diff(casgemm.row_products_prefix(A, B))
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    nz = np.diff(ref[0])
    heavy = int(((P >= 1 << 17) & (nz > 4096)).sum())  # dense rows (over 4096 columns) of 2^17 products or more
    assert heavy > 0
    saved = ctx.get_tuning()
    try:
        ctx.set_tuning(heavy_split=1)
        on = ctx.spgemm(A, B, "hybacc")
        ctx.set_tuning(heavy_split=0)
        off = ctx.spgemm(A, B, "hybacc")
    finally:
        ctx.set_tuning(**saved)
    assert on.stats["split_rows"] == heavy and off.stats["split_rows"] == 0
    for out in (on, off):
        np.testing.assert_array_equal(out.csr.row_ptrs, ref[0])
        np.testing.assert_array_equal(out.csr.cols.astype(np.int64), ref[1])
        np.testing.assert_array_equal(out.csr.vals.astype(np.float64), ref[2])
