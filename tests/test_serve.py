"""The serving loop (cas_serve_*): admission, budget, chunking, overlap.

CPU (dry run: the scheduler without device work, a request "runs" for a
time proportional to its bound): requests are admitted in arrival order,
never more than `slots` at once, never more reserved bytes than the budget;
a request larger than the budget runs in row chunks; later arrivals start
while earlier ones run.

GPU: every result in a concurrent mix equals the oracle's for the same
request run alone (digest, nnz, products, and the full C where kept),
including a chunked request; a large request does not hold up small ones
admitted after it.
"""
import time

import numpy as np
import pytest

import casgemm
import oracle
from conftest import has_gpu


def bound_of(A, B):
    P = np.diff(casgemm.row_products_prefix(A, B))
    vb = 12.0
    return (12.0 * np.minimum(P, B.num_col).sum() + 40.0 * A.num_row + vb * A.nnz
            + 16.0 + 8.0 * (B.num_row + 1) + vb * B.nnz)


def requests(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if i % 2 == 0:
            A = casgemm.gen_g500(int(rng.integers(7, 11)), int(rng.choice([4, 8, 16])), int(rng.integers(1 << 30)))
        else:
            nr = int(rng.integers(300, 2000))
            A = casgemm.gen_zipf(nr, 4 * nr, min(200, 2 * nr), 12 * nr, int(rng.integers(1 << 30)), col_q=20.0)
        out.append((A, A.transpose()))
    return out


def test_dry_run_admission_order_and_limits():
    reqs = requests(16, 1)
    budget = 3 * max(bound_of(A, B) for A, B in reqs)
    with casgemm.Server(slots=3, mem_budget=budget, dry_run=True, dry_run_ns_per_byte=2.0) as srv:
        ids = [srv.submit(A, B) for A, B in reqs]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert all(r["status"] == 0 for r in res)
    admits = [r["t_admit"] for r in res]
    assert admits == sorted(admits), "admission is in arrival order"
    assert 2 <= st["max_inflight"] <= 3
    assert st["max_inflight_bytes"] <= budget
    for r, (A, B) in zip(res, reqs):
        assert r["bound"] == pytest.approx(bound_of(A, B), rel=1e-9)
        assert r["flop"] == casgemm.intprod(A, B)


def test_dry_run_continuous_admission():
    """A small request that arrives while a long one runs starts before it ends."""
    big = casgemm.gen_g500(11, 16, 3)
    small = casgemm.gen_g500(6, 4, 4)
    with casgemm.Server(slots=2, mem_budget=1e12, dry_run=True, dry_run_ns_per_byte=20.0) as srv:
        b = srv.submit(big, big.transpose())
        time.sleep(0.01)
        s = srv.submit(small, small.transpose())
        rs, rb = srv.wait(s), srv.wait(b)
    assert rs["t_admit"] < rb["t_done"] and rs["t_done"] < rb["t_done"]


def test_dry_run_chunking_and_rejection():
    A = casgemm.gen_g500(9, 8, 5)
    B = A.transpose()
    whole = bound_of(A, B)
    fixed = 16.0 + 8.0 * (B.num_row + 1) + 12.0 * B.nnz
    with casgemm.Server(slots=2, mem_budget=fixed + (whole - fixed) / 5, dry_run=True) as srv:
        r = srv.wait(srv.submit(A, B))
        assert r["status"] == 0 and r["chunks"] >= 5 and r["bound"] <= fixed + (whole - fixed) / 5
        assert srv.stats()["chunked"] == 1
    with casgemm.Server(slots=1, mem_budget=fixed / 2, dry_run=True) as srv:
        r = srv.wait(srv.submit(A, B))
        assert r["status"] == 7  # CAS_ERR_REJECTED: B's copy alone is over the budget


def test_submit_rejects_bad_requests():
    A = casgemm.gen_g500(6, 4, 1)
    with casgemm.Server(slots=1, dry_run=True) as srv:
        with pytest.raises(casgemm.CasError):
            srv.submit(A, casgemm.gen_g500(7, 4, 1))  # shapes do not chain
        with pytest.raises(casgemm.CasError):
            srv.poll(12345)


def alone(A, B):
    rp, cols, vals, flop = oracle.oracle_spgemm(A, B, "hybacc")
    return rp, cols, vals, flop, oracle.csr_digest(rp, cols, vals)[0]


@pytest.mark.gpu
def test_mix_equals_alone():
    if not has_gpu():
        pytest.skip("no CUDA device")
    reqs = requests(14, 2)
    with casgemm.Server(slots=4, keep_output=True) as srv:
        ids = [srv.submit(A, B) for A, B in reqs]
        res = [srv.wait(i, 120.0) for i in ids]
        st = srv.stats()
    assert st["max_inflight"] >= 2, "requests overlapped on the device"
    for r, (A, B) in zip(res, reqs):
        rp, cols, vals, flop, d = alone(A, B)
        assert r["status"] == 0
        assert r["flop"] == flop and r["nnz_c"] == len(cols) and r["digest"] == d
        np.testing.assert_array_equal(r["C"].row_ptrs, rp)
        np.testing.assert_array_equal(r["C"].cols.astype(np.int64), cols)
        np.testing.assert_array_equal(r["C"].vals, vals)


@pytest.mark.gpu
def test_chunked_request_equals_alone():
    if not has_gpu():
        pytest.skip("no CUDA device")
    A = casgemm.gen_g500(11, 8, 9)
    B = A.transpose()
    fixed = 16.0 + 8.0 * (B.num_row + 1) + 12.0 * B.nnz
    with casgemm.Server(slots=2, mem_budget=fixed + (bound_of(A, B) - fixed) / 7, keep_output=True) as srv:
        r = srv.wait(srv.submit(A, B), 120.0)
    rp, cols, vals, flop, d = alone(A, B)
    assert r["status"] == 0 and r["chunks"] >= 7
    assert r["digest"] == d and r["nnz_c"] == len(cols) and r["flop"] == flop
    np.testing.assert_array_equal(r["C"].row_ptrs, rp)
    np.testing.assert_array_equal(r["C"].vals, vals)


@pytest.mark.gpu
def test_small_requests_pass_a_large_one():
    if not has_gpu():
        pytest.skip("no CUDA device")
    # the large request runs for tens of milliseconds; the small ones are
    # submitted right behind it and must be admitted into the free slots
    # while it runs (continuous batching), not after it drains
    big = casgemm.gen_g500(17, 16, 3)
    bigT = big.transpose()
    smalls = [casgemm.gen_g500(8, 4, 10 + i) for i in range(6)]
    with casgemm.Server(slots=3) as srv:
        b = srv.submit(big, bigT)
        ids = [srv.submit(S, S.transpose()) for S in smalls]
        rs = [srv.wait(i, 120.0) for i in ids]
        rb = srv.wait(b, 300.0)
    assert rb["status"] == 0 and all(r["status"] == 0 for r in rs)
    assert all(r["t_admit"] < rb["t_done"] for r in rs)
    assert sum(r["t_done"] < rb["t_done"] for r in rs) >= 1


@pytest.mark.gpu
def test_resident_operands_equal_alone():
    """Operands uploaded once and kept on the device: several requests name
    the same resident matrices, mixed with host requests; each result equals
    the same product alone.  A chunked resident request (row pointers rebased
    on the device) equals its product too."""
    if not has_gpu():
        pytest.skip("no CUDA device")
    reqs = requests(6, 3)
    dev = [(casgemm.DeviceCsr.upload(A), casgemm.DeviceCsr.upload(B)) for A, B in reqs]
    order = [0, 1, 2, 0, 3, 1, 4, 5, 0, 2]
    with casgemm.Server(slots=3, keep_output=True) as srv:
        ids = [srv.submit(*dev[k]) for k in order] + [srv.submit(*reqs[1])]
        res = [srv.wait(i, 120.0) for i in ids]
    for r, k in zip(res, order + [1]):
        A, B = reqs[k]
        rp, cols, vals, flop, d = alone(A, B)
        assert r["status"] == 0
        assert r["flop"] == flop and r["nnz_c"] == len(cols) and r["digest"] == d
        np.testing.assert_array_equal(r["C"].row_ptrs, rp)
        np.testing.assert_array_equal(r["C"].vals, vals)
    A = casgemm.gen_g500(11, 8, 9)
    B = A.transpose()
    dA, dB = casgemm.DeviceCsr.upload(A), casgemm.DeviceCsr.upload(B)
    budget = 16.0 + (bound_of(A, B) - 16.0 - 8.0 * (B.num_row + 1) - 12.0 * B.nnz) / 6
    with casgemm.Server(slots=2, mem_budget=budget, keep_output=True) as srv:
        r = srv.wait(srv.submit(dA, dB), 120.0)
    rp, cols, vals, flop, d = alone(A, B)
    assert r["status"] == 0 and r["chunks"] >= 5
    assert r["digest"] == d and r["nnz_c"] == len(cols) and r["flop"] == flop
    np.testing.assert_array_equal(r["C"].row_ptrs, rp)
    np.testing.assert_array_equal(r["C"].cols.astype(np.int64), cols)
    np.testing.assert_array_equal(r["C"].vals, vals)


@pytest.mark.gpu
def test_resident_operands_checked_at_submission():
    """A resident request whose columns leave B is refused at submission."""
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    A = casgemm.gen_g500(8, 4, 1)
    B = A.transpose()
    bad_cols = A.cols.copy()
    bad_cols[5] = B.num_row + 7
    t = [torch.from_numpy(x).cuda() for x in (A.row_ptrs, bad_cols, A.vals)]
    dA = casgemm.DeviceCsr(A.num_row, A.num_col, A.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), keep=t)
    with casgemm.Server(slots=1) as srv:
        with pytest.raises(casgemm.CasError):
            srv.submit(dA, casgemm.DeviceCsr.upload(B))
