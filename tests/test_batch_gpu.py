"""Batches of independent products (cas_batch_run: waves, per call, concurrent workers) and product digests.

Every job's digest, nnz(C), products and row digests must equal the oracle's
for the same job run alone (its C through oracle/csr_digest), in every mode:
the block-diagonal waves, one call per job, and calls per job on several
worker threads and streams.  Small budgets split jobs
across waves; int32 values accumulate exactly in int64.
"""
import numpy as np
import pytest

import casgemm
import oracle
from matrices import from_coo

pytestmark = pytest.mark.gpu


def oracle_job(A, B):
    rp, cols, vals, flop = oracle.oracle_spgemm(A, B, "hybacc")
    if A.vals.dtype == np.int32:
        # int32 inputs: the library's output values are int64 (exact), the
        # oracle's fp64 sums of the same integers
        assert np.all(vals == np.round(vals))
        vals = vals.astype(np.int64)
    d, rows = oracle.csr_digest(rp, cols, vals)
    return {"flop": flop, "nnz_c": len(cols), "digest": d, "rows": rows}


def small_batch(n, seed, int_vals=True):
    spec = casgemm.batch_spec(n, seed, scales=(5, 11), edge_factors=(2, 4, 8, 16))
    return [casgemm.batch_job(s, ef, gs, int_vals) for s, ef, gs in spec]


def check(out, jobs):
    for j, (A, B) in enumerate(jobs):
        want = oracle_job(A, B)
        got = out[j]
        assert got["status"] == 0, j
        assert got["flop"] == want["flop"], j
        assert got["nnz_c"] == want["nnz_c"], j
        assert got["digest"] == want["digest"], j
        if "row_digests" in got:
            np.testing.assert_array_equal(got["row_digests"], want["rows"])


def test_digest_matches_oracle(ctx):
    A = casgemm.gen_g500(10, 8, 3)
    B = A.transpose()
    import torch
    dev = torch.device("cuda", 0)

    def to_dev(M):
        t = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (M.row_ptrs, M.cols, M.vals)]
        return casgemm.DeviceCsr(M.num_row, M.num_col, M.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                                 M.val_type, keep=t)

    cc, _ = ctx.spgemm_device(to_dev(A), to_dev(B), "hybacc")
    try:
        d, rows = ctx.digest(cc, rows=True)
    finally:
        ctx.free(cc)
    want = oracle_job(A, B)
    assert d == want["digest"]
    np.testing.assert_array_equal(rows, want["rows"])


@pytest.mark.parametrize("mode", ["waves", "per_call", "concurrent"])
def test_batch_int_values(ctx, mode):
    jobs = small_batch(24, 7)
    out, st = ctx.batch_run(jobs, "hybacc", mode, row_digests=True)
    check(out, jobs)
    assert st["jobs_ok"] == 24
    assert st["waves"] == (1 if mode == "waves" else 24)


def test_batch_waves_split_jobs(ctx):
    jobs = small_batch(12, 9)
    # a budget far below one job's output: many waves, jobs cut across them
    out, st = ctx.batch_run(jobs, "hybacc", "waves", wave_budget=2e5, row_digests=True)
    assert st["waves"] > 12
    check(out, jobs)


@pytest.mark.parametrize("accum", ["hash", "hsersc"])
def test_batch_f64_accumulators(ctx, accum):
    jobs = small_batch(10, 11, int_vals=False)
    out, _ = ctx.batch_run(jobs, accum, "waves")
    check(out, jobs)


def test_batch_general_and_empty_jobs(ctx):
    rng = np.random.default_rng(5)
    G = from_coo(150, 220, rng.integers(0, 150, 900), rng.integers(0, 220, 900),
                 rng.integers(1, 9, 900).astype(np.float64))
    H = from_coo(220, 500, rng.integers(0, 220, 1800), rng.integers(0, 500, 1800),
                 rng.integers(-3, 4, 1800).astype(np.float64))
    E = from_coo(40, 30, np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0))
    F = from_coo(30, 60, rng.integers(0, 30, 100), rng.integers(0, 60, 100), np.ones(100))
    jobs = [(G, H), (E, F), (F.transpose(), E.transpose()), (G, H)]
    for mode in ("waves", "per_call", "concurrent"):
        out, _ = ctx.batch_run(jobs, "hybacc", mode)
        check(out, jobs)


def test_batch_rejects_bad_column(ctx):
    A = casgemm.gen_g500(6, 4, 1)
    bad = casgemm.Csr(A.num_row, A.num_col, A.row_ptrs, A.cols.copy(), A.vals)
    bad.cols[5] = A.num_col + 3
    with pytest.raises(casgemm.CasError) as e:
        ctx.batch_run([(A, A.transpose()), (bad, A.transpose())], "hybacc", "waves")
    assert e.value.status == 1


def test_batch_concurrent_reports_the_failing_job(ctx):
    A = casgemm.gen_g500(6, 4, 1)
    bad = casgemm.Csr(A.num_row, A.num_col, A.row_ptrs, A.cols.copy(), A.vals)
    bad.cols[5] = A.num_col + 3
    with pytest.raises(casgemm.CasError) as e:
        ctx.batch_run([(A, A.transpose()), (bad, A.transpose()), (A, A.transpose())], "hybacc", "concurrent")
    assert e.value.status == 1 and "job 1" in str(e.value)
    # the context and its workers still run batches
    jobs = small_batch(6, 3)
    out, st = ctx.batch_run(jobs, "hybacc", "concurrent")
    check(out, jobs)
    assert st["jobs_ok"] == 6
