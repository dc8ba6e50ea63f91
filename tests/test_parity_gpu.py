"""GPU parity: casgemm (CUDA, through the C ABI) against the CPU oracle.

Integer-valued products must match bit for bit (row pointers, sorted column
indices, values).  The one case with real-valued inputs is compared with
rtol 1e-12: fp64 sums in a different order round differently.
"""
import numpy as np
import pytest

import casgemm
import oracle
from matrices import cases, with_int_values

pytestmark = pytest.mark.gpu

CASES = cases()
IDS = [c[0] for c in CASES]


def check(res: casgemm.Csr, ref, exact: bool, name: str):
    rp, cols, vals = ref[0], ref[1], ref[2]
    assert np.array_equal(res.row_ptrs, rp), f"{name}: row pointers differ"
    assert np.array_equal(res.cols.astype(np.int64), cols), f"{name}: columns differ"
    if exact:
        assert np.array_equal(res.vals.astype(np.float64), vals), f"{name}: values differ"
    else:
        np.testing.assert_allclose(res.vals, vals, rtol=1e-12, atol=1e-12 * max(1.0, float(np.abs(vals).max())))


@pytest.mark.parametrize("algo", ["hash", "hsersc", "hybacc"])
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_f64(ctx, case, algo):
    name, A, B = case
    ref = oracle.oracle_spgemm(A, B, algo)
    out = ctx.spgemm(A, B, algo)
    exact = name != "general_AB"
    check(out.csr, ref, exact, name)
    assert out.stats["flop"] == ref[3]
    assert out.stats["nnz_c"] == len(ref[1])


@pytest.mark.parametrize("algo", ["hash", "hybacc"])
@pytest.mark.parametrize("case", CASES[:8], ids=IDS[:8])
def test_int32_values(ctx, case, algo):
    """int32 values 1..8 in, int64 sums out (the batched configuration's arithmetic)."""
    name, A, _ = case
    Ai = with_int_values(A, 41)
    Bi = Ai.transpose()
    ref = oracle.oracle_spgemm(Ai, Bi, algo)
    out = ctx.spgemm(Ai, Bi, algo)
    assert out.csr.vals.dtype == np.int64
    check(out.csr, ref, True, name)


def test_reference_layout_int64_columns(ctx):
    """A csr_t-shaped input (int64 columns, src/inc/store.h:49-56) and int64 output columns."""
    A = casgemm.gen_g500(10, 8, 3)
    T = A.transpose()
    A64 = casgemm.Csr(A.num_row, A.num_col, A.row_ptrs, A.cols.astype(np.int64), A.vals)
    B64 = casgemm.Csr(T.num_row, T.num_col, T.row_ptrs, T.cols.astype(np.int64), T.vals)
    out = ctx.spgemm(A64, B64, "hybacc", col_bytes=8)
    ref = oracle.oracle_spgemm(A, T, "hybacc")
    assert out.csr.cols.dtype == np.int64
    check(out.csr, ref, True, "int64 columns")


@pytest.mark.parametrize("algo", ["hash", "hybacc"])
def test_same_host_matrix_as_both_inputs(ctx, algo):
    """C = A*A with one host CSR passed as A and as B (a symmetric A, so A*A^T):
    one device copy serves both, and C equals the oracle's A*A^T."""
    A = casgemm.gen_er(12, 16, 4)
    ref = oracle.oracle_spgemm(A, A.transpose(), algo)
    out = ctx.spgemm(A, A, algo)
    check(out.csr, ref, True, "A as both inputs")
    assert out.stats["h2d_bytes"] == 8 * (A.num_row + 1) + 12 * A.nnz
    two = ctx.spgemm(A, A.transpose(), algo)
    assert two.stats["h2d_bytes"] == 2 * out.stats["h2d_bytes"]


def test_runtime_phases(ctx):
    A = casgemm.gen_g500(12, 8, 9)
    out = ctx.spgemm(A, A.transpose(), "hybacc")
    rt = out.runtime
    assert all(rt[k] >= 0 for k in rt)
    assert abs(rt["total_time"] - (rt["init_time"] + rt["symb_time"] + rt["mgmt_time"] + rt["numc_time"])) < 1e-9


def test_host_output_dma_into_kept_blocks(ctx):
    """The host blocks of a returned C go back to the context on cas_csr_free,
    which registers the large ones with CUDA; the next output of about the
    same size lands in them by DMA directly, with the same result."""
    A = casgemm.gen_er(14, 32, 9)
    B = A.transpose()
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    first = ctx.spgemm(A, B, "hybacc")
    second = ctx.spgemm(A, B, "hybacc")
    assert second.stats["d2h_direct_bytes"] >= 8 * second.csr.nnz  # the values at least
    for out in (first, second):
        np.testing.assert_array_equal(out.csr.row_ptrs, ref[0])
        np.testing.assert_array_equal(out.csr.cols.astype(np.int64), ref[1])
        np.testing.assert_array_equal(out.csr.vals, ref[2])
    # reference layout (int64 columns): the columns are widened through staging
    third = ctx.spgemm(A, B, "hybacc", col_bytes=8)
    np.testing.assert_array_equal(third.csr.cols, ref[1])
    np.testing.assert_array_equal(third.csr.vals, ref[2])


def _raw_host_product(ctx, ca, cb):
    """cas_spgemm into host memory through the C ABI; the caller frees C."""
    import ctypes
    cc = casgemm.CasCsr()
    cc.on_device, cc.col_bytes = 0, 4
    st = ctx.lib.cas_spgemm(ctx.h, casgemm.ACCUM["hybacc"], ctypes.byref(ca), ctypes.byref(cb), ctypes.byref(cc),
                            None)
    assert st == 0, ctx.lib.cas_last_error(ctx.h).decode()
    return cc


def _host_arrays(cc):
    import ctypes
    m, nnz = cc.num_row, cc.num_nnz
    rp = np.ctypeslib.as_array(ctypes.cast(cc.row_ptrs, ctypes.POINTER(ctypes.c_int64)), (m + 1,)).copy()
    cols = np.ctypeslib.as_array(ctypes.cast(cc.cols, ctypes.POINTER(ctypes.c_int32)), (nnz,)).astype(np.int64)
    vals = np.ctypeslib.as_array(ctypes.cast(cc.rats, ctypes.POINTER(ctypes.c_double)), (nnz,)).copy()
    return rp, cols, vals


def test_registered_block_freed_without_its_context():
    """A C whose host blocks the context has registered with CUDA may be freed
    with no context (cas_csr_free(NULL, C)): the blocks are unregistered and
    dropped from the producing context's cache first, so its next output goes
    to fresh blocks (no direct DMA) and is still exact; after a free through
    the context, outputs land in registered blocks again."""
    import ctypes
    from conftest import has_gpu
    if not has_gpu():
        pytest.skip("no CUDA device")
    ctx = casgemm.Context(0)  # a context of its own: its block cache starts empty
    A = casgemm.gen_er(14, 32, 9)
    B = A.transpose()
    ref = oracle.oracle_spgemm(A, B, "hybacc")
    ca, cb = A.as_cas(), B.as_cas()
    c1 = _raw_host_product(ctx, ca, cb)
    ctx.lib.cas_csr_free(ctx.h, ctypes.byref(c1))           # into the cache, registered
    c2 = _raw_host_product(ctx, ca, cb)                      # lands in the registered blocks
    assert ctx.stats()["d2h_direct_bytes"] >= 8 * c2.num_nnz
    got = _host_arrays(c2)
    assert ctx.lib.cas_csr_free(None, ctypes.byref(c2)) == 0  # no context: released from ctx's records
    for x, y in zip(got, ref[:3]):
        np.testing.assert_array_equal(x, y)
    c3 = _raw_host_product(ctx, ca, cb)
    assert ctx.stats()["d2h_direct_bytes"] == 0              # fresh blocks, nothing registered
    for x, y in zip(_host_arrays(c3), ref[:3]):
        np.testing.assert_array_equal(x, y)
    ctx.lib.cas_csr_free(ctx.h, ctypes.byref(c3))
    c4 = _raw_host_product(ctx, ca, cb)
    assert ctx.stats()["d2h_direct_bytes"] >= 8 * c4.num_nnz
    for x, y in zip(_host_arrays(c4), ref[:3]):
        np.testing.assert_array_equal(x, y)
    ctx.lib.cas_csr_free(ctx.h, ctypes.byref(c4))
    ctx.close()
