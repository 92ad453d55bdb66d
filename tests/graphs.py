"""Small hand-made graphs with closed-form answers, and CSR helpers for tests."""
import itertools

import numpy as np

from graphkokkos_b200.api import Csr


def from_edges(n, edges, directed=False):
    """Symmetric (unless directed) CSR from an edge list, sorted and deduplicated."""
    rows, cols = [], []
    for u, v in edges:
        if u == v:
            continue
        rows.append(u)
        cols.append(v)
        if not directed:
            rows.append(v)
            cols.append(u)
    if rows:
        key = np.unique(np.asarray(rows, dtype=np.int64) * n + np.asarray(cols, dtype=np.int64))
        r, c = key // n, key % n
    else:
        r = c = np.zeros(0, dtype=np.int64)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    return Csr(n, n, rp, c.astype(np.int32), None, int(len(c)))


def complete(n):
    return from_edges(n, list(itertools.combinations(range(n), 2)))


def wheel(n_rim):
    hub = n_rim
    e = [(i, (i + 1) % n_rim) for i in range(n_rim)] + [(i, hub) for i in range(n_rim)]
    return from_edges(n_rim + 1, e)


def star(n_leaves):
    return from_edges(n_leaves + 1, [(0, i) for i in range(1, n_leaves + 1)])


def path(n):
    return from_edges(n, [(i, i + 1) for i in range(n - 1)])


def disjoint_triangles(k):
    e = []
    for t in range(k):
        b = 3 * t
        e += [(b, b + 1), (b + 1, b + 2), (b, b + 2)]
    return from_edges(3 * k, e)


def empty(n):
    return Csr(n, n, np.zeros(n + 1, dtype=np.int64), np.zeros(0, dtype=np.int32), None, 0)


def random_csr(m, n, density, seed, values=False, max_val=5):
    rng = np.random.default_rng(seed)
    mask = rng.random((m, n)) < density
    r, c = np.nonzero(mask)
    rp = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=m), out=rp[1:])
    val = rng.integers(-max_val, max_val + 1, size=len(c)).astype(np.int32) if values else None
    return Csr(m, n, rp, c.astype(np.int32), val, int(len(c)))


def dense_of(csr):
    d = np.zeros((csr.m, csr.n), dtype=np.int64)
    rp = np.asarray(csr.rowptr)
    col = np.asarray(csr.col)
    val = np.ones(len(col), dtype=np.int64) if csr.val is None else np.asarray(csr.val, dtype=np.int64)
    for i in range(csr.m):
        d[i, col[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
    return d


def brandes_f64(csr, sources):
    """Textbook Brandes (BFS, unweighted, unnormalised, one direction)."""
    n = csr.m
    rp = np.asarray(csr.rowptr)
    col = np.asarray(csr.col)
    bc = np.zeros(n)
    for s in sources:
        sigma = np.zeros(n)
        dist = -np.ones(n, dtype=np.int64)
        sigma[s] = 1.0
        dist[s] = 0
        order = [s]
        q = [s]
        while q:
            nq = []
            for v in q:
                for w in col[rp[v]:rp[v + 1]]:
                    if dist[w] < 0:
                        dist[w] = dist[v] + 1
                        nq.append(w)
                    if dist[w] == dist[v] + 1:
                        sigma[w] += sigma[v]
            order += nq
            q = nq
        delta = np.zeros(n)
        for v in reversed(order):
            for w in col[rp[v]:rp[v + 1]]:
                if dist[w] == dist[v] + 1:
                    delta[v] += sigma[v] / sigma[w] * (1 + delta[w])
            if v != s:
                bc[v] += delta[v]
    return bc


def bc_mismatches(got, want, rtol=1e-12):
    """Vertices whose FP64 BC score is not within rtol relative of the oracle's;
    an oracle score of exactly 0 must be exactly 0 (no absolute tolerance)."""
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape, (got.shape, want.shape)
    zero = want == 0.0
    bad = np.where(zero, got != 0.0, ~(np.abs(got - want) <= rtol * np.abs(want)))
    return np.flatnonzero(bad)


def assert_bc_close(got, want, rtol=1e-12):
    bad = bc_mismatches(got, want, rtol)
    if len(bad):
        got = np.asarray(got, dtype=np.float64)
        want = np.asarray(want, dtype=np.float64)
        show = ", ".join(f"v{v}: {got[v]!r} vs {want[v]!r}" for v in bad[:5])
        raise AssertionError(f"{len(bad)} of {len(want)} BC scores outside rtol {rtol} (atol 0): {show}")
