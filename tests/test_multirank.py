"""CPU, two ranks over gloo: the multi-GPU form of the product.

Rows of C are independent, so the N-rank form gives each rank a contiguous
shard of A's rows with about 1/N of the products (casgemm.row_shard) and B
whole; nothing is exchanged while computing.  Here every rank computes its
shard with the CPU oracle (the GPU path is the same call on a device), the
ranks all-gather their shards, and the assembled rows must equal the
single-rank product exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    for p in (os.path.join(ROOT, "contention-aware-spgemm_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import casgemm
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = casgemm.gen_g500(10, 8, 31)
        B = A.transpose()
        r0, r1 = casgemm.row_shard(casgemm.row_products_prefix(A, B), rank, world)
        rp, cols, vals, flop = oracle.oracle_spgemm(casgemm.slice_rows(A, r0, r1), B, "hybacc")
        shards = [None] * world
        dist.all_gather_object(shards, (r0, r1, rp, cols, vals, flop))
        if rank == 0:
            out.put(shards)
    finally:
        dist.destroy_process_group()


def test_two_rank_row_shards_reassemble():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "contention-aware-spgemm_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import casgemm
    import oracle

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    shards = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards.sort(key=lambda s: s[0])
    assert shards[0][0] == 0 and shards[0][1] == shards[1][0] and shards[1][1] == 1 << 10
    flops = [s[5] for s in shards]
    assert min(flops) > 0.3 * sum(flops)  # balanced by products, not rows
    A = casgemm.gen_g500(10, 8, 31)
    rp, cols, vals, flop = oracle.oracle_spgemm(A, A.transpose(), "hybacc")
    assert sum(flops) == flop
    got_rp = np.concatenate([[0], np.cumsum(np.concatenate([np.diff(s[2]) for s in shards]))])
    np.testing.assert_array_equal(got_rp, rp)
    np.testing.assert_array_equal(np.concatenate([s[3] for s in shards]), cols)
    np.testing.assert_array_equal(np.concatenate([s[4] for s in shards]), vals)


def _assemble_worker(rank, world, port, out):
    import sys
    for p in (os.path.join(ROOT, "contention-aware-spgemm_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import datetime
    import torch
    import casgemm
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        A = casgemm.gen_g500(10, 8, 31)
        B = A.transpose()
        if world == 3 and rank == 1:
            r0 = r1 = casgemm.row_shard(casgemm.row_products_prefix(A, B), 0, 2)[1]  # an empty shard
        elif world == 3:
            r0, r1 = casgemm.row_shard(casgemm.row_products_prefix(A, B), rank // 2, 2)
        else:
            r0, r1 = casgemm.row_shard(casgemm.row_products_prefix(A, B), rank, world)
        rp, cols, vals, _ = oracle.oracle_spgemm(casgemm.slice_rows(A, r0, r1), B, "hybacc")
        got = casgemm.gather_shards(torch.from_numpy(rp), torch.from_numpy(cols), torch.from_numpy(vals), r0, r1,
                                    A.num_row)
        if rank == 0:
            out.put(tuple(t.numpy() for t in got))
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_shards_assembled_on_the_root(world):
    """C assembled on rank 0 from every rank's row shard (an all-gather of the
    shard sizes, then point-to-point transfers of columns, values and row
    pointers) equals the single-rank product; with 3 ranks one shard is
    empty."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "contention-aware-spgemm_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import casgemm
    import oracle

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_assemble_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    rp, cols, vals = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    A = casgemm.gen_g500(10, 8, 31)
    want = oracle.oracle_spgemm(A, A.transpose(), "hybacc")
    np.testing.assert_array_equal(rp, want[0])
    np.testing.assert_array_equal(cols, want[1])
    np.testing.assert_array_equal(vals, want[2])

