"""Host-side arithmetic of bench.py that needs no GPU: the share of the
reference formulation's streamed entries that the lower-triangle k-truss
support product streams, against a direct count."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _direct_share(rp, col):
    n = len(rp) - 1
    streamed = full = 0
    for i in range(n):
        ci = col[rp[i]:rp[i + 1]]
        low = ci[ci < i]
        if len(low) == 0:
            continue
        last = low.max()
        for k in ci:
            ck = col[rp[k]:rp[k + 1]]
            streamed += int((ck <= last).sum())
            full += len(ck)
    return streamed / max(1, full)


def test_ktruss_streamed_share_matches_direct_count():
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(0)
    for n, p in [(60, 0.15), (200, 0.03), (5, 0.0), (40, 0.9)]:
        M = rng.random((n, n)) < p
        M = np.triu(M, 1)
        M = M | M.T
        rp = np.concatenate([[0], np.cumsum(M.sum(1))]).astype(np.int64)
        col = np.concatenate([np.flatnonzero(M[i]) for i in range(n)] + [np.zeros(0, dtype=np.int64)])
        assert abs(bench.ktruss_streamed_share(rp, col) - _direct_share(rp, col)) < 1e-12
