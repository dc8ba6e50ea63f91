"""CPU: the numpy digest restatement against its definition, entry by entry."""
import numpy as np

import oracle

M = (1 << 64) - 1


def mix64(z):
    z = (z + 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return z ^ (z >> 31)


def digest_loops(rp, cols, vals):
    total, rows = 0, []
    for r in range(len(rp) - 1):
        h = 0
        for k, e in enumerate(range(rp[r], rp[r + 1])):
            v = vals[e]
            bits = int(np.float64(v).view(np.uint64)) if isinstance(v, (float, np.floating)) else int(v) & M
            h = (h + (mix64((int(cols[e]) * 0x9E3779B97F4A7C15 + k) & M) ^ mix64((bits + 0x632BE59BD9B4E019) & M))) & M
        rows.append(h)
        total = (total + mix64((h + r) & M)) & M
    return total, rows


def test_digest_restatement():
    rng = np.random.default_rng(1)
    rp = np.concatenate([[0], np.cumsum(rng.integers(0, 7, 40))]).astype(np.int64)
    cols = rng.integers(0, 1 << 20, rp[-1]).astype(np.int32)
    for vals in (rng.normal(size=rp[-1]), rng.integers(-9, 1 << 40, rp[-1]).astype(np.int64)):
        d, rows = oracle.csr_digest(rp, cols, vals)
        d2, rows2 = digest_loops(rp, cols, vals)
        assert d == d2
        assert [int(x) for x in rows] == rows2


def test_digest_sees_order_and_values():
    rp = np.array([0, 3, 5], np.int64)
    cols = np.array([1, 4, 9, 0, 2], np.int32)
    vals = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    d = oracle.csr_digest(rp, cols, vals)[0]
    assert d != oracle.csr_digest(rp, cols[[1, 0, 2, 3, 4]], vals[[1, 0, 2, 3, 4]])[0]
    v2 = vals.copy()
    v2[4] = 6.0
    assert d != oracle.csr_digest(rp, cols, v2)[0]
    assert d != oracle.csr_digest(np.array([0, 2, 5], np.int64), cols, vals)[0]
