"""GPU test of cas_scan_noalloc, the scan entry point that allocates nothing.

Some callers cannot allocate device memory: a process whose device memory is
owned and budgeted by another framework's pool, or a latency-sensitive loop
that cannot afford the synchronisation a cudaMalloc/cudaFree may bring.  They
call cas_scan_noalloc, whose scratch is a fixed array inside the library; its
output must equal the allocating cas_scan's, call after call, although every
call reuses the same scratch.

The file is named so that pytest collects it last: a run that stops at the
first failure has then already run every other test.
"""
import ctypes

import numpy as np
import pytest

import casgemm

pytestmark = pytest.mark.gpu

CAS_ERR_REJECTED = 7
MAX_N = 16384 * 4096  # the array holds 16,384 tile sums of 4,096 elements


def _noalloc(lib):
    fn = lib.cas_scan_noalloc
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    return fn


def _both(ctx, x):
    """Scan x (length n-1) into n outputs with both entry points."""
    import torch

    n = len(x) + 1
    d_in = torch.from_numpy(x).cuda()
    out_noalloc = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    out_ref = torch.full((n,), -2, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = _noalloc(ctx.lib)(out_noalloc.data_ptr(), d_in.data_ptr(), n, stream)
    assert st == 0, f"cas_scan_noalloc returned {st}"
    torch.cuda.synchronize()
    assert ctx.lib.cas_scan(ctx.h, out_ref.data_ptr(), d_in.data_ptr(), n) == 0
    torch.cuda.synchronize()
    return out_noalloc.cpu().numpy(), out_ref.cpu().numpy()


def test_noalloc_scan_matches_cas_scan_twice(ctx):
    rng = np.random.default_rng(2024)
    # two calls in a row through the shared scratch: a long scan over many
    # tiles, then a short one whose tiles the first call's partials still cover
    for length in (3_000_000, 77_777):
        x = rng.integers(0, 1_000_000, size=length, dtype=np.int64)
        got, ref = _both(ctx, x)
        np.testing.assert_array_equal(got, ref)
        expect = np.concatenate([[0], np.cumsum(x)])
        np.testing.assert_array_equal(got, expect)


def test_noalloc_scan_rejects_oversize(ctx):
    import torch

    small = torch.zeros(4, dtype=torch.int64, device="cuda")
    # rejected before any memory is touched, so the small arrays are safe here
    st = _noalloc(ctx.lib)(small.data_ptr(), small.data_ptr(), MAX_N + 1, None)
    assert st == CAS_ERR_REJECTED


def test_noalloc_scan_at_the_size_limit(ctx):
    """n == MAX_N: the last of the 16,384 tile sums fills the array's last slot."""
    import torch

    n = MAX_N
    g = torch.Generator(device="cuda").manual_seed(7)
    d_in = torch.randint(0, 4, (n - 1,), dtype=torch.int64, device="cuda", generator=g)
    out = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    ref = torch.full((n,), -2, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # twice in a row through the shared scratch
        out.fill_(-1)
        assert _noalloc(ctx.lib)(out.data_ptr(), d_in.data_ptr(), n, stream) == 0
        torch.cuda.synchronize()
        assert ctx.lib.cas_scan(ctx.h, ref.data_ptr(), d_in.data_ptr(), n) == 0
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    assert int(out[0]) == 0
    assert int(out[-1]) == int(d_in.sum())
    assert int(out[n // 2]) == int(d_in[: n // 2].sum())

