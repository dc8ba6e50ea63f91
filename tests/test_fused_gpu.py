"""GPU: the fused ESC rows (no symbolic pass, offsets by look-back).

Rows of 2049..5120 products are counted, sorted and placed by one kernel in
row order, in its index form (column and product index in shared memory) or
its column-and-value form.  Checked bit for bit against the oracle and against the same
product with fusion off: uniform rows (nearly all fused), rows whose
buckets overflow (deferred to the radix-sort kernel after an in-kernel
count), int32 values, rows split over several A chunks, device output.
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


def hot_column_matrix(seed=3, ncol=3000, per_row=160, hot=1):
    """Rows whose products crowd one bucket: per_row A entries whose B rows
    all hold columns 0..hot-1 (so per_row * hot keys in the first bucket),
    plus other columns below ncol, 20 per B row."""
    rng = np.random.default_rng(seed)
    n_rows, n_mid = 40, 400
    r, c = [], []
    for i in range(n_rows):
        ks = rng.choice(n_mid, per_row, replace=False)
        r += [i] * per_row
        c += list(ks)
    A = from_coo(n_rows, n_mid, np.array(r), np.array(c))
    br, bc = [], []
    for k in range(n_mid):
        cols = np.concatenate([np.arange(hot), rng.choice(np.arange(hot, ncol), 20 - hot, replace=False)])
        br += [k] * 20
        bc += list(cols)
    B = from_coo(n_mid, ncol, np.array(br), np.array(bc))
    return A, B


@pytest.mark.parametrize("algo", ["hybacc", "hsersc"])
def test_er_rows_fused(ctx, algo):
    A = casgemm.gen_er(13, 32, 7)
    B = A.transpose()
    ref = oracle.oracle_spgemm(A, B, algo)
    out = ctx.spgemm(A, B, algo)
    assert out.stats["fused_rows"] > A.num_row // 2
    same(out, ref)
    ctx.set_fusion(False)
    try:
        off = ctx.spgemm(A, B, algo)
    finally:
        ctx.set_fusion(True)
    assert off.stats["fused_rows"] == 0
    same(off, ref)


def test_overflowing_fused_rows_are_deferred(ctx):
    # columns spread over 4M: the hot column's bucket spans 2048 columns, too
    # wide to sum densely, so each row is counted in-kernel and deferred
    A, B = hot_column_matrix(ncol=1 << 22)
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    out = ctx.spgemm(A, B, "hybacc")
    assert out.stats["fused_rows"] == A.num_row
    assert out.stats["esc_overflow_rows"] == A.num_row
    same(out, ref)


@pytest.mark.parametrize("fuse,form", [(True, 0), (False, 0), (True, 1)])
def test_huge_narrow_buckets_summed_densely(ctx, fuse, form):
    # columns below 3000: the hot columns' bucket spans 2 columns, summed by
    # the whole block in place, no row deferred.  The index form takes rows
    # of one staged chunk (at most 128 A entries): 120 entries, 2 hot columns
    A, B = hot_column_matrix() if form == 0 else hot_column_matrix(per_row=120, hot=2)
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    saved = ctx.get_tuning()
    ctx.set_tuning(fusion=int(fuse), esc_form=form)
    try:
        out = ctx.spgemm(A, B, "hybacc")
    finally:
        ctx.set_tuning(**saved)
    if fuse:
        assert out.stats["fused_rows"] == A.num_row
    assert out.stats["esc_overflow_rows"] == 0
    same(out, ref)


def test_index_form_defers_two_huge_buckets(ctx):
    # hot columns 0, 1 and 2048, 2049 over 4096 columns (buckets of 2
    # columns): two buckets of 240 products each
    rng = np.random.default_rng(5)
    A, B = hot_column_matrix(per_row=120, hot=1, ncol=4096)
    hot = [0, 1, 2048, 2049]
    br, bc = np.repeat(np.arange(B.num_row), 20), []
    for k in range(B.num_row):
        bc.append(np.concatenate([hot, rng.choice(np.setdiff1d(np.arange(4096), hot), 16, replace=False)]))
    B = from_coo(B.num_row, 4096, br, np.concatenate(bc))
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    out = ctx.spgemm(A, B, "hybacc")
    assert out.stats["fused_rows"] == A.num_row
    assert out.stats["esc_overflow_rows"] == A.num_row
    same(out, ref)


def test_fused_int_values(ctx):
    A = with_int_values(casgemm.gen_g500(12, 16, 5), 9)
    B = A.transpose()
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    out = ctx.spgemm(A, B, "hybacc")
    assert out.stats["fused_rows"] > 0
    assert out.csr.vals.dtype == np.int64
    same(out, ref)


def test_fused_rows_over_several_a_chunks(ctx):
    """A rows of 200 entries (the kernel stages 128 at a time), 15 per B row."""
    rng = np.random.default_rng(8)
    r = np.repeat(np.arange(30), 200)
    c = np.concatenate([rng.choice(1000, 200, replace=False) for _ in range(30)])
    A = from_coo(30, 1000, r, c, rng.integers(1, 5, len(r)).astype(np.float64))
    br = np.repeat(np.arange(1000), 15)
    bc = np.concatenate([rng.choice(5000, 15, replace=False) for _ in range(1000)])
    B = from_coo(1000, 5000, br, bc, rng.integers(1, 5, len(br)).astype(np.float64))
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    saved = ctx.get_tuning()
    try:
        for form, deferred in ((1, 30), (0, 0)):  # the index form takes one staged chunk
            ctx.set_tuning(esc_form=form)
            out = ctx.spgemm(A, B, "hybacc")
            assert out.stats["fused_rows"] == 30
            assert out.stats["esc_overflow_rows"] == deferred
            same(out, ref)
    finally:
        ctx.set_tuning(**saved)


def test_fused_device_output_digest(ctx):
    import torch
    dev = torch.device("cuda", 0)
    A = casgemm.gen_er(12, 32, 11)
    B = A.transpose()

    def to_dev(M):
        t = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (M.row_ptrs, M.cols, M.vals)]
        return casgemm.DeviceCsr(M.num_row, M.num_col, M.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                                 M.val_type, keep=t)

    cc, _ = ctx.spgemm_device(to_dev(A), to_dev(B), "hybacc")
    try:
        d = ctx.digest(cc)
        nnz = cc.num_nnz
    finally:
        ctx.free(cc)
    rp, cols, vals, _ = oracle.oracle_spgemm(A, B, "hybacc")
    assert nnz == len(cols)
    assert d == oracle.csr_digest(rp, cols, vals)[0]


def test_profiling_leaves_no_cuda_error(ctx):
    """Timing queries for bins that never ran must not leave an error behind
    (the next CUDA call of another library would report it)."""
    import torch
    A = casgemm.gen_er(12, 32, 3)
    ctx.set_profiling(True)
    try:
        out = ctx.spgemm(A, A.transpose(), "hybacc")
    finally:
        ctx.set_profiling(False)
    assert out.stats["fused_rows"] > 0 and out.stats["fused_ms"] > 0
    torch.zeros(4, device="cuda").sum().item()  # raises if an error is pending


def test_tuning_routes_rows_but_not_results(ctx):
    """cas_set_tuning moves rows between kernels; C stays bit-identical."""
    A = casgemm.gen_g500(12, 16, 4)
    B = A.transpose()
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    saved = ctx.get_tuning()
    seen = set()
    try:
        for kw in ({"esc_max_products": 1024}, {"hash_max_nnz": 256}, {"fused_min_products": 512},
                   {"acc_thres": 5.0}, {"fusion": 0}, {"esc_form": 0}, {"esc_form": 0, "fused_min_products": 512},
                   {"bin_order": 0}, {"heavy_split": 0}):
            ctx.set_tuning(**saved)
            ctx.set_tuning(**kw)
            out = ctx.spgemm(A, B, "hybacc")
            same(out, ref)
            seen.add(tuple(sorted((k, v) for k, v in out.stats["numc_bins"].items() if v)))
        with pytest.raises(casgemm.CasError):
            ctx.set_tuning(esc_max_products=9000)
    finally:
        ctx.set_tuning(**saved)
    assert len(seen) >= 3, "the knobs change the routing"


def test_autotuner_caches_per_class(ctx, tmp_path):
    import torch
    dev = torch.device("cuda", 0)

    def to_dev(M):
        t = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (M.row_ptrs, M.cols, M.vals)]
        return casgemm.DeviceCsr(M.num_row, M.num_col, M.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                                 M.val_type, keep=t)

    A = casgemm.gen_er(11, 32, 2)
    key = casgemm.Autotuner.key(A, A)
    path = str(tmp_path / "tune.json")
    tuner = casgemm.Autotuner(ctx, path)
    before = ctx.get_tuning()
    cfg = tuner.tune(key, to_dev(A), to_dev(A), trials=1)
    assert ctx.get_tuning() == before  # tuning leaves the context as it was
    assert cfg["seconds"] > 0 and cfg["seconds"] <= cfg["default_seconds"]
    again = casgemm.Autotuner(ctx, path)
    assert again.apply(key)
    try:
        out = ctx.spgemm(A, A.transpose(), "hybacc")
        same(out, oracle.oracle_spgemm(A, A.transpose(), "hybacc"))
    finally:
        ctx.set_tuning(**before)


@pytest.mark.parametrize("per_b", [100, 180])
def test_index_form_many_shared_columns(ctx, per_b):
    """Rows of 3000 (fused) or 5400 (ESC bin) products of which half fall
    on 300 common columns: hundreds of columns with several products each,
    which the index form zeroes in C and adds into with global atomics."""
    rng = np.random.default_rng(11)
    n_rows, n_mid, ncol = 64, 600, 5000
    r = np.repeat(np.arange(n_rows), 30)
    c = np.concatenate([rng.choice(n_mid, 30, replace=False) for _ in range(n_rows)])
    A = from_coo(n_rows, n_mid, r, c, rng.integers(1, 4, len(r)).astype(np.float64))
    common = rng.choice(ncol, 300, replace=False)
    br = np.repeat(np.arange(n_mid), per_b)
    bc = np.concatenate([rng.choice(common, per_b, replace=False) if k % 2 else
                         rng.choice(ncol, per_b, replace=False) for k in range(n_mid)])
    B = from_coo(n_mid, ncol, br, bc, rng.integers(1, 4, len(br)).astype(np.float64))
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    saved = ctx.get_tuning()
    try:
        for form in (1, 0):
            ctx.set_tuning(esc_form=form)
            out = ctx.spgemm(A, B, "hybacc")
            assert out.stats["esc_overflow_rows"] == 0
            same(out, ref)
    finally:
        ctx.set_tuning(**saved)


def _hot_long_rows(seed=8, ncol=3000, per_row=80, blen=40, hot=2):
    """Fused rows (80 A entries of B rows with 40 columns each: 3200
    products) whose B rows all hold the hot columns 0..hot-1, so one bucket
    gets 160 products over 2 columns (summed densely), while the B rows are
    long enough for the value pass to walk them a warp per row."""
    rng = np.random.default_rng(seed)
    n_rows, n_mid = 30, 300
    r = np.repeat(np.arange(n_rows), per_row)
    c = np.concatenate([rng.choice(n_mid, per_row, replace=False) for _ in range(n_rows)])
    A = from_coo(n_rows, n_mid, r, c)
    bc = [np.concatenate([np.arange(hot), rng.choice(np.arange(hot, ncol), blen - hot, replace=False)])
          for _ in range(n_mid)]
    B = from_coo(n_mid, ncol, np.repeat(np.arange(n_mid), blen), np.concatenate(bc))
    return A, B


def _register_form_cases():
    er = casgemm.gen_er(13, 32, 7)
    er_wide = casgemm.gen_er(12, 40, 3)   # rows of 5121..6144 products: the 6144 bin
    g500 = casgemm.gen_g500(12, 16, 5)   # short B rows: the product-order value pass
    hotA, hotB = hot_column_matrix(per_row=120, hot=2)
    longA, longB = _hot_long_rows()
    return [("er_s13_ef32", er, er.transpose()), ("er_s12_ef40", er_wide, er_wide.transpose()),
            ("g500_s12_ef16", g500, g500.transpose()), ("hot_columns", hotA, hotB),
            ("g500_int", with_int_values(g500, 9), with_int_values(g500, 9).transpose()),
            ("hot_long_rows", longA, longB)]


@pytest.mark.parametrize("fuse", [True, False])
@pytest.mark.parametrize("case", range(6), ids=["er_s13_ef32", "er_s12_ef40", "g500_s12_ef16", "hot_columns",
                                                  "g500_int", "hot_long_rows"])
def test_register_form_matches_oracle(ctx, case, fuse):
    """esc_form 2: the index form with each thread's keys held in registers
    between the histogram and the scatter, (for long B rows) a warp per B
    row in the value pass, and values staged in shared memory at their
    places and copied out in order; fused rows and the 4800 / 6144 ESC
    bins, with a bucket of hub columns summed densely among them."""
    name, A, B = _register_form_cases()[case]
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    saved = ctx.get_tuning()
    ctx.set_tuning(fusion=int(fuse), esc_form=2)
    try:
        out = ctx.spgemm(A, B, "hybacc")
        again = ctx.spgemm(A, B, "hsersc")
    finally:
        ctx.set_tuning(**saved)
    same(out, ref)
    same(again, oracle.oracle_spgemm(A, B, "hsersc"))
    if fuse and name.startswith("er_s13"):
        assert out.stats["fused_rows"] > A.num_row // 2
