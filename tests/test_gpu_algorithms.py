"""Parity of the CUDA k-truss and batched betweenness centrality with the
oracle: k-truss edge sets bit-exact, FP64 BC within 1e-12 relative."""
import json
import os

import numpy as np
import pytest

from tests import graphs as G

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
BC_RTOL = 1e-12


def dev(csr):
    return csr.to("cuda")


@pytest.mark.parametrize("scale,seed,k", [(9, 5, 3), (10, 7, 4), (11, 7, 5), (12, 2, 6), (12, 2, 9)])
def test_ktruss_matches_oracle(gk, orc, cuda, scale, seed, k):
    A = gk.gen_rmat(scale, 16, seed=seed)
    rp, col, iters, _ = orc.ktruss(A, k)
    T, it = gk.ktruss(dev(A), k)
    assert it == iters
    assert T.nnz == len(col)
    np.testing.assert_array_equal(T.rowptr.cpu().numpy(), rp)
    np.testing.assert_array_equal(T.col.cpu().numpy(), col)


def test_ktruss_host_buffers_and_closed_forms(gk, orc, cuda):
    T, it = gk.ktruss(G.complete(6), 6)
    assert T.nnz == 30 and it == 1
    T, it = gk.ktruss(G.wheel(10), 4)
    assert T.nnz == 0
    A = G.from_edges(5, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (3, 4)])
    T, it = gk.ktruss(A, 3)
    assert T.nnz == 12 and it == 2
    with pytest.raises(gk.GkError):
        gk.ktruss(A, 2)


def test_ktruss_golden(gk, cuda):
    g = json.load(open(os.path.join(GOLDEN, "ktruss.json")))
    for case in g["cases"]:
        A = gk.gen_rmat(case["scale"], case["edge_factor"], seed=case["seed"], device="cuda")
        T, it = gk.ktruss(A, case["k"])
        assert it == case["iterations"]
        assert T.nnz == case["nnz"]
        rp = T.rowptr.cpu().numpy()
        col = T.col.cpu().numpy()
        rows = np.repeat(np.arange(A.m, dtype=np.int64), np.diff(rp))
        h = int(np.bitwise_xor.reduce((col.astype(np.int64) * 2654435761 + rows) & 0xFFFFFFFF)) if len(col) else 0
        assert h == case["xor_hash"]


def test_ktruss_fixed_point(gk, cuda):
    A = gk.gen_rmat(12, 16, seed=3, device="cuda")
    T, _ = gk.ktruss(A, 5)
    T2, it2 = gk.ktruss(T, 5)
    assert it2 == 1 and T2.nnz == T.nnz


def test_ktruss_nonsymmetric_input(gk, orc, cuda):
    """A non-symmetric matrix takes the full-mask support S<C> = C·C (the
    lower-triangle shortcut needs S = S^T) and still matches the oracle."""
    for seed in (5, 6):
        A = G.random_csr(400, 400, 0.06, seed=seed)
        # no self-loops, as the k-truss input requires
        rp, col = np.asarray(A.rowptr), np.asarray(A.col)
        rows = np.repeat(np.arange(A.m), np.diff(rp))
        keep = col != rows
        nrp = np.zeros(A.m + 1, dtype=np.int64)
        np.cumsum(np.bincount(rows[keep], minlength=A.m), out=nrp[1:])
        B = gk.Csr(A.m, A.m, nrp, col[keep].astype(np.int32), None, int(keep.sum()))
        want_rp, want_col, want_it, _ = orc.ktruss(B, 3)
        T, it = gk.ktruss(dev(B), 3)
        assert it == want_it and T.nnz == len(want_col)
        np.testing.assert_array_equal(T.rowptr.cpu().numpy(), want_rp)
        np.testing.assert_array_equal(T.col.cpu().numpy(), want_col)


def test_ktruss_graph_loop_matches_host_loop(gk, cuda):
    """The pass loop runs as one CUDA graph (conditional while node); with
    profiling on the host drives the same passes.  Both, and both schedulers,
    give the same edge set and pass count."""
    lib = gk.load()
    A = gk.gen_rmat(13, 16, seed=4, device="cuda")
    T, it = gk.ktruss(A, 5)
    from graphkokkos_b200 import sched
    sched.load_model()
    TL, itL = gk.ktruss(A, 5, sched="learned")
    lib.gk_prof_enable(1)
    try:
        TH, itH = gk.ktruss(A, 5)
    finally:
        lib.gk_prof_enable(0)
    assert it == itL == itH and it > 2
    for X in (TL, TH):
        assert X.nnz == T.nnz
        assert np.array_equal(X.rowptr.cpu().numpy(), T.rowptr.cpu().numpy())
        assert np.array_equal(X.col.cpu().numpy(), T.col.cpu().numpy())


# ---------------------------------------------------------------------------
# betweenness centrality
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("scale,nsrc,seed", [(9, 40, 1), (10, 64, 2), (11, 100, 3), (12, 512, 4), (10, 1, 5)])
def test_bc_matches_oracle(gk, orc, cuda, scale, nsrc, seed):
    A = gk.gen_rmat(scale, 16, seed=seed)
    rng = np.random.default_rng(seed)
    src = rng.choice(A.m, size=nsrc, replace=False)
    want = orc.bc_f64(A, src)
    got = gk.bc_batch(dev(A), src).cpu().numpy()
    G.assert_bc_close(got, want, BC_RTOL)


def test_bc_more_than_one_chunk(gk, orc, cuda):
    A = gk.gen_rmat(10, 8, seed=9)
    src = np.random.default_rng(1).choice(A.m, size=700, replace=False)
    G.assert_bc_close(gk.bc_batch(dev(A), src).cpu().numpy(), orc.bc_f64(A, src), BC_RTOL)


def test_bc_closed_forms_and_host_buffers(gk, cuda):
    bc = gk.bc_batch(G.path(5), range(5))
    G.assert_bc_close(bc, [0, 6, 8, 6, 0])
    bc = gk.bc_batch(G.star(6), range(7))
    assert bc[0] == pytest.approx(30.0) and np.all(bc[1:] == 0)


def test_bc_transpose_paths(gk, orc, cuda):
    """An undirected pattern with sorted rows is used as its own transpose; the
    same graph with each row's columns reversed (unsorted) or with unit values
    goes through the radix-sort transpose.  All three give the oracle's scores."""
    import torch
    A = gk.gen_rmat(11, 16, seed=13)
    src = np.random.default_rng(13).choice(A.m, size=96, replace=False)
    want = orc.bc_f64(A, src)
    rp = np.asarray(A.rowptr, dtype=np.int64)
    col = np.asarray(A.col)[:A.nnz]
    rev = np.concatenate([col[rp[i]:rp[i + 1]][::-1] for i in range(A.m)]).astype(np.int32)
    unsorted = gk.Csr(A.m, A.n, torch.from_numpy(rp.copy()), torch.from_numpy(rev), None, A.nnz)
    valued = gk.Csr(A.m, A.n, torch.from_numpy(rp.copy()), torch.from_numpy(col.astype(np.int32)),
                    torch.ones(A.nnz, dtype=torch.int32), A.nnz)
    for X in (A, unsorted, valued):
        G.assert_bc_close(gk.bc_batch(dev(X), src).cpu().numpy(), want, BC_RTOL)


def test_bc_directed(gk, orc, cuda):
    A = G.random_csr(300, 300, 0.02, seed=11)
    src = np.arange(0, 300, 7)
    np.testing.assert_allclose(gk.bc_batch(dev(A), src).cpu().numpy(), G.brandes_f64(A, src), BC_RTOL)


def test_bc_heavy_vertices(gk, orc, cuda):
    # hub of degree > 512 goes to the CTA-per-vertex kernels
    A = G.from_edges(2000, [(0, i) for i in range(1, 2000)] + [(i, i + 1) for i in range(1, 1999, 3)])
    src = np.arange(0, 2000, 17)
    G.assert_bc_close(gk.bc_batch(dev(A), src).cpu().numpy(), orc.bc_f64(A, src), BC_RTOL)


@pytest.mark.parametrize("shape", [0, 1, -1])
def test_bc_forward_shapes_match_oracle(gk, orc, cuda, shape):
    """Every forward level as pull (0), as push (1), or by the plain rule (-1),
    driven from the host with per-level timing: same FP64 result."""
    from graphkokkos_b200 import sched
    cases = [(gk.gen_rmat(11, 16, seed=3), 200, 1),
             (G.from_edges(2000, [(0, i) for i in range(1, 2000)] + [(i, i + 1) for i in range(1, 1999, 3)]), 90, 2),
             (G.random_csr(300, 300, 0.02, seed=11), 40, 3)]
    for A, nsrc, seed in cases:
        src = np.random.default_rng(seed).choice(A.m, size=nsrc, replace=False)
        ms, feat, bc = sched.bc_tune(dev(A), src, shape)
        assert len(ms) >= 1 and np.all(ms > 0) and feat.shape == (len(ms), 8)
        want = orc.bc_f64(A, src) if A.m != 300 else G.brandes_f64(A, src)
        G.assert_bc_close(bc.cpu().numpy(), want, BC_RTOL)


def test_bc_graph_loop_matches_host_loop(gk, cuda):
    """The level loops run as CUDA graphs; with profiling on the host drives
    the same levels.  Plain and learned shape choices agree too."""
    from graphkokkos_b200 import sched
    lib = gk.load()
    A = gk.gen_rmat(13, 16, seed=6, device="cuda")
    src = np.random.default_rng(6).choice(A.m, size=300, replace=False)
    ref = gk.bc_batch(A, src).cpu().numpy()
    lib.gk_prof_enable(2)
    try:
        host = gk.bc_batch(A, src).cpu().numpy()
    finally:
        lib.gk_prof_enable(0)
    G.assert_bc_close(host, ref, BC_RTOL)
    if os.path.exists(sched.BC_MODEL_PATH):
        sched.load_bc_model()
        learned = gk.bc_batch(A, src, sched="learned").cpu().numpy()
        G.assert_bc_close(learned, ref, BC_RTOL)


def test_bc_golden(gk, cuda):
    g = json.load(open(os.path.join(GOLDEN, "bc.json")))
    for case in g["cases"]:
        A = gk.gen_rmat(case["scale"], case["edge_factor"], seed=case["seed"], device="cuda")
        got = gk.bc_batch(A, case["sources"]).cpu().numpy()
        np.testing.assert_allclose(got, np.asarray(case["bc_ref_float"]), rtol=2e-4, atol=1e-2)


def test_bc_errors(gk, cuda):
    A = dev(G.path(5))
    with pytest.raises(gk.GkError):
        gk.bc_batch(A, [0, 0])
    with pytest.raises(gk.GkError):
        gk.bc_batch(A, [7])
