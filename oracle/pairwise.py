"""numpy's float32 pairwise summation order, restated (TEST ORACLE).

numpy reduces a contiguous float32 array by recursive halving at multiples
of 8 down to blocks of <= 128 values; a block of 8 or more is summed in 8
interleaved float32 accumulators combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7))
plus a sequential tail; a block under 8 is summed sequentially from 0.
(numpy/_core/src/umath/loops_utils.h.src, ``pairwise_sum``; numpy 2.3.)
solve_adr's stop rule takes ``C[j][m].mean()`` with this order, so the CUDA
path replays it (adr.cu, means_*); this module is what the tests check the
replay against.
"""

import numpy as np


def _block(a):
    n = a.shape[0]
    f = np.float32
    if n < 8:
        r = f(0.0)
        for v in a:
            r = f(r + v)
        return r
    m8 = n - (n % 8)
    r = a[:8].astype(np.float32).copy()
    for i in range(8, m8, 8):
        r = (r + a[i:i + 8]).astype(np.float32)
    res = f(f(f(r[0] + r[1]) + f(r[2] + r[3])) + f(f(r[4] + r[5]) + f(r[6] + r[7])))
    for v in a[m8:]:
        res = f(res + v)
    return res


def pairwise_sum(a):
    """float32 sum of the 1-D array `a` in numpy's order."""
    a = np.ascontiguousarray(a, np.float32)
    n = a.shape[0]
    if n <= 128:
        return _block(a)
    n2 = n // 2
    n2 -= n2 % 8
    return np.float32(pairwise_sum(a[:n2]) + pairwise_sum(a[n2:]))


def pairwise_mean(a):
    """float32 mean the way ndarray.mean() computes it for float32 input."""
    a = np.ascontiguousarray(a, np.float32)
    return np.float32(pairwise_sum(a) / np.float32(a.shape[0]))


def tree(n):
    """The leaves (start, length) of the summation tree over n values."""
    out = []

    def rec(s, k):
        if k <= 128:
            out.append((s, k))
            return
        k2 = k // 2
        k2 -= k2 % 8
        rec(s, k2)
        rec(s + k2, k - k2)

    if n > 0:
        rec(0, n)
    return out
