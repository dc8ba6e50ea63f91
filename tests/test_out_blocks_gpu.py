"""GPU: a C returned in host memory computed in row blocks (cas_tuning.out_blocks).

Each block runs the four phases as a product of its own and is copied out
while the next one is computed; the blocks' rows land at their places in
one host CSR.  Checked bit for bit against the oracle (small cases, every
accumulator, empty blocks and rows, fused and dense rows, int32
values) and against the same product in one block (a C large enough for the
context to register its host arrays, so the copies go by DMA straight into
them; and the size rule's own choice of blocks).
"""
import numpy as np
import pytest

import casgemm
import oracle
from matrices import from_coo, with_int_values

pytestmark = pytest.mark.gpu


def same(out, ref):
    np.testing.assert_array_equal(out.csr.row_ptrs, ref[0])
    np.testing.assert_array_equal(out.csr.cols.astype(np.int64), ref[1])
    np.testing.assert_array_equal(out.csr.vals.astype(np.float64), ref[2])


def same_csr(a, b):
    np.testing.assert_array_equal(a.row_ptrs, b.row_ptrs)
    np.testing.assert_array_equal(a.cols, b.cols)
    np.testing.assert_array_equal(a.vals, b.vals)


def with_tuning(ctx, fn, **kw):
    saved = ctx.get_tuning()
    ctx.set_tuning(**kw)
    try:
        return fn()
    finally:
        ctx.set_tuning(**saved)


def _skewed_rows(seed=4):
    """Rows 0-299 and 900-999 of A empty, row 500 holding 1800 of its
    entries and the rest 3 each: the blocks (cut at equal A entries) between
    row 500's neighbours are empty and the last holds no entries."""
    rng = np.random.default_rng(seed)
    r, c = [], []
    for i in range(300, 900):
        k = 1800 if i == 500 else 3
        r.append(np.full(k, i))
        c.append(rng.choice(4000, k, replace=False))
    A = from_coo(1000, 4000, np.concatenate(r), np.concatenate(c), rng.integers(1, 4, sum(map(len, r))).astype(float))
    br = np.repeat(np.arange(4000), 12)
    bc = np.concatenate([rng.choice(30000, 12, replace=False) for _ in range(4000)])
    B = from_coo(4000, 30000, br, bc, rng.integers(1, 4, len(br)).astype(np.float64))
    return A, B


def _dense_rows(seed=6):
    """Rows of a few thousand distinct columns (the dense path) among short ones."""
    rng = np.random.default_rng(seed)
    n_rows, n_mid, ncol = 300, 2000, 20000
    r = np.repeat(np.arange(n_rows), 40)
    c = np.concatenate([rng.choice(n_mid, 40, replace=False) for _ in range(n_rows)])
    A = from_coo(n_rows, n_mid, r, c, rng.integers(1, 4, len(r)).astype(np.float64))
    br = np.repeat(np.arange(n_mid), 150)
    bc = np.concatenate([rng.choice(ncol, 150, replace=False) for _ in range(n_mid)])
    B = from_coo(n_mid, ncol, br, bc, rng.integers(1, 4, len(br)).astype(np.float64))
    return A, B


def _cases():
    er = casgemm.gen_er(12, 32, 7)
    g500 = casgemm.gen_g500(12, 16, 5)
    pa, pb = _skewed_rows()
    da, db = _dense_rows()
    return [("er_s12_ef32", er, er.transpose()), ("g500_s12_ef16", g500, g500.transpose()),
            ("skewed_rows", pa, pb), ("dense_rows", da, db),
            ("g500_int", with_int_values(g500, 9), with_int_values(g500, 9).transpose())]


@pytest.mark.parametrize("blocks", [2, 7])
@pytest.mark.parametrize("accum", ["hybacc", "hash", "hsersc"])
@pytest.mark.parametrize("case", range(5), ids=["er_s12_ef32", "g500_s12_ef16", "skewed_rows", "dense_rows",
                                                  "g500_int"])
def test_row_blocks_match_oracle(ctx, case, accum, blocks):
    name, A, B = _cases()[case]
    ref = oracle.oracle_spgemm(A, B, accum)
    out = with_tuning(ctx, lambda: ctx.spgemm(A, B, accum), out_blocks=blocks)
    same(out, ref)
    assert 1 < out.stats["out_blocks"] <= blocks
    assert out.stats["flop"] == ref[3] and out.stats["nnz_c"] == len(ref[1])
    one = with_tuning(ctx, lambda: ctx.spgemm(A, B, accum), out_blocks=1)
    assert one.stats["out_blocks"] == 1
    for k in ("flop", "nnz_c", "fused_rows", "esc_overflow_rows"):
        assert out.stats[k] == one.stats[k], k
    assert sum(out.stats["numc_bins"].values()) == sum(one.stats["numc_bins"].values())


def test_row_blocks_into_registered_host_arrays(ctx):
    """C of about 0.8 GB: the first call's host arrays are registered when
    they come back, so the second call copies its blocks into them by DMA."""
    E = casgemm.gen_er(16, 16, 11)
    B = E.transpose()
    one = with_tuning(ctx, lambda: ctx.spgemm(E, B), out_blocks=1)
    for _ in range(2):
        out = with_tuning(ctx, lambda: ctx.spgemm(E, B), out_blocks=12)
        same_csr(out.csr, one.csr)
        assert out.stats["out_blocks"] == 12
    assert out.stats["d2h_direct_bytes"] >= 12.0 * out.stats["nnz_c"]
    assert out.stats["d2h_bytes"] >= out.stats["d2h_direct_bytes"]


def test_size_rule_picks_blocks(ctx):
    """out_blocks 0 (default): one block under 1 GiB of C (about 12 bytes an
    entry), else one per 2 GiB and at least 2 (here C is about 1.8 GB)."""
    E = casgemm.gen_er(16, 24, 12)
    B = E.transpose()
    auto = with_tuning(ctx, lambda: ctx.spgemm(E, B), out_blocks=0)
    one = with_tuning(ctx, lambda: ctx.spgemm(E, B), out_blocks=1)
    same_csr(auto.csr, one.csr)
    assert auto.stats["out_blocks"] >= 2
    small = casgemm.gen_er(10, 8, 3)
    assert with_tuning(ctx, lambda: ctx.spgemm(small, small.transpose()), out_blocks=0).stats["out_blocks"] == 1


def test_device_output_is_one_block(ctx):
    import torch
    E = casgemm.gen_er(12, 16, 2)
    dA = casgemm.DeviceCsr.upload(E)
    dB = casgemm.DeviceCsr.upload(E.transpose())
    C, _ = with_tuning(ctx, lambda: ctx.spgemm_device(dA, dB), out_blocks=5)
    try:
        assert ctx.stats()["out_blocks"] == 1
    finally:
        ctx.free(C)
        torch.cuda.synchronize()


def test_out_blocks_range(ctx):
    with pytest.raises(casgemm.CasError):
        ctx.set_tuning(out_blocks=-1)
    with pytest.raises(casgemm.CasError):
        ctx.set_tuning(out_blocks=65)
