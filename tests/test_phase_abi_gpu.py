"""The phase-function ABI, called the way a caller that keeps the reference's
phase structure calls it (the drivers' hybaccspgemm(),
src/ams_hybaccspgemm.c:36-215):

    flp_populate -> scan -> hash_symb -> scan -> allocate C -> *_numc

through cas_flp_populate, cas_scan, cas_hash_symb and cas_{hash,hsersc,
hybacc}_numc on device CSRs, each output compared with the oracle's
restatement of the same phase (orc_flp_populate, orc_scan, orc_hash_symb,
orc_spgemm) bit for bit.  One case has rows of more than 4096 distinct
columns, so the numeric call runs the dense kernel without bitmaps kept from
a symbolic pass of its own.
"""
import ctypes

import numpy as np
import pytest

import casgemm
import oracle
from matrices import from_coo

pytestmark = pytest.mark.gpu


def _dev(M):
    import torch
    t = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (M.row_ptrs, M.cols, M.vals)]
    return casgemm.DeviceCsr(M.num_row, M.num_col, M.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                             M.val_type, keep=t)


def _oracle_phases(A, B):
    lib = oracle.oracle_lib()
    a, ka = oracle.to_orc(A.row_ptrs, A.cols, A.vals, A.num_col)
    b, kb = oracle.to_orc(B.row_ptrs, B.cols, B.vals, B.num_col)
    m = A.num_row
    flp = np.zeros(max(m, 1), np.int64)
    nz = np.zeros(max(m, 1), np.int64)
    lib.orc_flp_populate(ctypes.byref(a), ctypes.byref(b), flp.ctypes.data)
    lib.orc_hash_symb(ctypes.byref(a), ctypes.byref(b), flp.ctypes.data, nz.ctypes.data)
    del ka, kb
    return flp[:m], nz[:m]


def _heavy_rows_case():
    """Rows 0 and 1 reach every column; the other rows are sparse and random."""
    n = 9000
    rng = np.random.default_rng(11)
    r = np.concatenate([np.zeros(n, np.int64), np.ones(n // 2, np.int64) , rng.integers(2, n, 30000)])
    c = np.concatenate([np.arange(n), np.arange(0, n, 2), rng.integers(0, n, 30000)])
    key = np.unique(r * n + c)
    A = from_coo(n, n, key // n, key % n)
    return A, A.transpose()


CASES = {
    "g500_s12_ef8": lambda: (lambda A: (A, A.transpose()))(casgemm.gen_g500(12, 8, 12)),
    "er_s13_ef32": lambda: (lambda A: (A, A.transpose()))(casgemm.gen_er(13, 32, 13)),
    "heavy_rows": _heavy_rows_case,
}


@pytest.mark.parametrize("algo", ["hash", "hsersc", "hybacc"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_phase_sequence_matches_oracle(ctx, name, algo):
    import torch
    A, B = CASES[name]()
    m = A.num_row
    dA, dB = _dev(A), _dev(B)
    lib = ctx.lib
    flp_ref, nz_ref = _oracle_phases(A, B)

    d_flp = torch.zeros(m, dtype=torch.int64, device="cuda")
    assert lib.cas_flp_populate(ctx.h, ctypes.byref(dA.c), ctypes.byref(dB.c), d_flp.data_ptr()) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_flp.cpu().numpy(), flp_ref)

    d_ps = torch.zeros(m + 1, dtype=torch.int64, device="cuda")
    assert lib.cas_scan(ctx.h, d_ps.data_ptr(), d_flp.data_ptr(), m + 1) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_ps.cpu().numpy(), np.concatenate([[0], np.cumsum(flp_ref)]))

    d_nz = torch.zeros(m, dtype=torch.int64, device="cuda")
    assert lib.cas_hash_symb(ctx.h, ctypes.byref(dA.c), ctypes.byref(dB.c), d_flp.data_ptr(), d_nz.data_ptr()) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_nz.cpu().numpy(), nz_ref)

    d_rp = torch.zeros(m + 1, dtype=torch.int64, device="cuda")
    assert lib.cas_scan(ctx.h, d_rp.data_ptr(), d_nz.data_ptr(), m + 1) == 0
    torch.cuda.synchronize()
    nnz = int(d_rp[-1])
    d_col = torch.full((max(nnz, 1),), -1, dtype=torch.int32, device="cuda")
    d_val = torch.full((max(nnz, 1),), -1.0, dtype=torch.float64, device="cuda")
    C = casgemm.CasCsr(m, B.num_col, nnz, d_rp.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), 4,
                       casgemm.VAL_F64, 1, 0)
    fn = {"hash": lib.cas_hash_numc, "hsersc": lib.cas_hsersc_numc, "hybacc": lib.cas_hybacc_numc}[algo]
    assert fn(ctx.h, ctypes.byref(dA.c), ctypes.byref(dB.c), d_flp.data_ptr(), ctypes.byref(C)) == 0, \
        lib.cas_last_error(ctx.h).decode()
    torch.cuda.synchronize()
    rp, cols, vals, flop = oracle.oracle_spgemm(A, B, algo)
    np.testing.assert_array_equal(d_rp.cpu().numpy(), rp)
    np.testing.assert_array_equal(d_col[:nnz].cpu().numpy().astype(np.int64), cols)
    np.testing.assert_array_equal(d_val[:nnz].cpu().numpy(), vals)
    if name == "heavy_rows":
        assert int(nz_ref.max()) > 4096  # the dense kernel ran on these rows
    # the phase entry points do not need d_row_flp
    d_nz2 = torch.zeros(m, dtype=torch.int64, device="cuda")
    assert lib.cas_hash_symb(ctx.h, ctypes.byref(dA.c), ctypes.byref(dB.c), None, d_nz2.data_ptr()) == 0
    torch.cuda.synchronize()
    assert torch.equal(d_nz, d_nz2)
