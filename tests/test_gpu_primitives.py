"""The alternate-BC operators of the reference (include/matrix_la.h:182-328)
on the GPU against the CPU restatement, bit for bit: add_nointersect, the
dense masked eWiseMult, fuseEWiseMultAdd and mxmm_spd (FP64 with the
reference's fused multiply-adds).  The restatement itself is pinned against
the reference in test_oracle.py."""
import numpy as np
import pytest

from tests import graphs as G
from tests.test_oracle import disjoint_pair

pytestmark = pytest.mark.gpu


def dev(x):
    import torch
    if isinstance(x, np.ndarray):
        return torch.as_tensor(x).cuda()
    return x.to("cuda")


def host(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_add_nointersect(gk, orc, cuda, seed):
    A, B = disjoint_pair(300, 120, seed, density=0.1)
    want = orc.add_nointersect(A, B)
    for a, b in ((A, B), (dev(A), dev(B))):
        C = gk.add_nointersect(a, b)
        for w, g in zip(want, (C.rowptr, C.col, C.val)):
            np.testing.assert_array_equal(host(g), w)
    # rows ending with B entries, B-only and empty rows, pattern-only operands
    rng = np.random.default_rng(seed)
    mask = rng.random((200, 90)) < 0.08
    side = rng.random((200, 90)) < 0.5
    r, c = np.nonzero(mask & side)
    rp = np.zeros(201, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=200), out=rp[1:])
    Ap = G.Csr(200, 90, rp, c.astype(np.int32), None, len(c))
    r, c = np.nonzero(mask & ~side)
    rp = np.zeros(201, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=200), out=rp[1:])
    Bp = G.Csr(200, 90, rp, c.astype(np.int32), None, len(c))
    want = orc.add_nointersect(Ap, Bp)
    C = gk.add_nointersect(dev(Ap), dev(Bp))
    for w, g in zip(want, (C.rowptr, C.col, C.val)):
        np.testing.assert_array_equal(host(g), w)
    E = G.empty(7)
    C = gk.add_nointersect(E, E)
    assert C.nnz == 0 and list(host(C.rowptr)) == [0] * 8


def test_dense_ewise_mult_masked_and_fuse(gk, orc, cuda):
    rng = np.random.default_rng(5)
    m, n = 300, 257
    A, B, C = (rng.standard_normal((m, n)) for _ in range(3))
    M = G.random_csr(m, n, 0.05, seed=6)
    want = orc.dense_ewise_mult_masked(A, B, M)
    np.testing.assert_array_equal(gk.dense_ewise_mult_masked(A, B, M), want)
    np.testing.assert_array_equal(host(gk.dense_ewise_mult_masked(dev(A), dev(B), dev(M))), want)
    want = orc.fuse_ewise_mult_add(A, B, C)
    Ch = C.copy()
    gk.dense_fuse_ewise_mult_add(A, B, Ch)
    np.testing.assert_array_equal(Ch, want)
    Cd = dev(C)
    gk.dense_fuse_ewise_mult_add(dev(A), dev(B), Cd)
    np.testing.assert_array_equal(host(Cd), want)


@pytest.mark.parametrize("seed", [7, 8])
def test_mxmm_spd(gk, orc, cuda, seed):
    rng = np.random.default_rng(seed)
    m, k, n = 400, 350, 96
    S = G.random_csr(m, k, 0.03, seed=seed, values=True)
    D = rng.standard_normal((k, n))
    M = G.random_csr(m, n, 0.1, seed=seed + 1)
    sval = rng.standard_normal(S.nnz)
    # A's values: A_val when given, else A's int32 values, else 1 (pattern only)
    ints = np.asarray(S.val, dtype=np.float64)
    for av, want_av in ((sval, sval), (None, ints)):
        want = orc.mxmm_spd(S, D, M, want_av)
        np.testing.assert_array_equal(gk.mxmm_spd(S, D, M, A_val=av), want)
        np.testing.assert_array_equal(host(gk.mxmm_spd(dev(S), dev(D), dev(M), A_val=None if av is None else dev(av))),
                                      want)
    P = G.Csr(S.m, S.n, S.rowptr, S.col, None, S.nnz)
    np.testing.assert_array_equal(gk.mxmm_spd(P, D, M), orc.mxmm_spd(P, D, M))
    # the product written over B (square case, as the reference's W = A·W)
    Sq = G.random_csr(n, n, 0.05, seed=seed + 2, values=True)
    Mq = G.random_csr(n, n, 0.2, seed=seed + 3)
    W = rng.standard_normal((n, n))
    want = orc.mxmm_spd(Sq, W, Mq, np.asarray(Sq.val, dtype=np.float64))
    Wd = dev(W)
    gk.mxmm_spd(dev(Sq), Wd, dev(Mq), out=Wd)
    np.testing.assert_array_equal(host(Wd), want)
    Wh = W.copy()
    gk.mxmm_spd(Sq, Wh, Mq, out=Wh)
    np.testing.assert_array_equal(Wh, want)
