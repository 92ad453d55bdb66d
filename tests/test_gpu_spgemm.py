"""Parity of the CUDA masked SpGEMM path with the oracle (bit-exact integers).

Every kernel variant is checked on its own (gk_*_variant entry points force
all rows onto one variant) as well as under the scheduler, on seeded RMAT /
Erdos-Renyi graphs, random plus-times products with values, hand-made graphs
and edge cases.  All calls go through the C ABI."""
import json
import os

import numpy as np
import pytest

from tests import graphs as G

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
NV = 24


def dev(csr):
    return csr.to("cuda")


@pytest.mark.parametrize("scale,seed", [(8, 1), (10, 2), (12, 3), (14, 1)])
def test_tc_rmat_every_variant(gk, orc, cuda, scale, seed):
    A = gk.gen_rmat(scale, 16, seed=seed)
    L = gk.lower_host(A)
    want = orc.tc_lower(L)
    Ld = dev(L)
    assert gk.tc_count(Ld) == want
    for v in range(NV):
        assert gk.tc_count_variant(Ld, v) == want, f"variant {v}"


def test_tc_golden_config1(gk, cuda):
    g = json.load(open(os.path.join(GOLDEN, "tc.json")))
    case = [c for c in g["cases"] if c["scale"] == 14][0]
    A = gk.gen_rmat(14, 16, seed=case["seed"], device="cuda")
    assert A.nnz == case["nnz_sym"]
    L = gk.extract_lower(A)
    assert L.nnz == case["nnz_lower"]
    assert gk.tc_count(L) == case["triangles"]
    assert gk.tc_count(L, sched="plain") == case["triangles"]


def test_tc_host_buffers(gk, orc, cuda):
    A = gk.gen_rmat(11, 16, seed=4)
    L = gk.lower_host(A)
    assert gk.tc_count(L) == orc.tc_lower(L)


@pytest.mark.parametrize("maker", [lambda: G.complete(7), lambda: G.wheel(9), lambda: G.star(20),
                                   lambda: G.path(30), lambda: G.disjoint_triangles(6), lambda: G.empty(5),
                                   lambda: G.complete(300)])
def test_tc_small_graphs(gk, orc, cuda, maker):
    L = gk.lower_host(maker())
    want = orc.tc_lower(L)
    Ld = dev(L)
    assert gk.tc_count(Ld) == want
    for v in range(NV):
        assert gk.tc_count_variant(Ld, v) == want


def test_tc_er(gk, orc, cuda):
    A = gk.gen_er(20000, 300000, seed=3)
    L = gk.lower_host(A)
    assert gk.tc_count(dev(L)) == orc.tc_lower(L)


def test_tc_rmat18(gk, orc, cuda):
    A = gk.gen_rmat(18, 16, seed=1, device="cuda")
    L = gk.extract_lower(A)
    want = orc.tc_lower(L.numpy())
    assert gk.tc_count(L) == want
    for v in (0, 3, 5, 8, 9, 12):
        assert gk.tc_count_variant(L, v) == want


def test_tc_concurrent_variant_streams(gk, orc, cuda):
    """GK_CONCURRENT_VARIANTS=1 forks every variant kernel onto its own side
    stream (the library reads the setting once per process, so the check runs
    in a child process): same counts under both schedulers."""
    import subprocess
    import sys
    A = gk.gen_rmat(16, 16, seed=2)
    want = orc.tc_lower(gk.lower_host(A))
    code = ("import graphkokkos_b200 as gk; from graphkokkos_b200 import sched; sched.load_model(); "
            "L = gk.extract_lower(gk.gen_rmat(16, 16, seed=2, device='cuda')); "
            "print(gk.tc_count(L, sched='plain'), gk.tc_count(L, sched='learned'))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, GK_CONCURRENT_VARIANTS="1"))
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.split() == [str(want), str(want)]


def test_tc_row_sums(gk, orc, cuda):
    A = gk.gen_rmat(12, 16, seed=8)
    L = gk.lower_host(A)
    got = gk.tc_row_sums(dev(L)).cpu().numpy().astype(np.uint64)
    np.testing.assert_array_equal(got, orc.tc_row_sums(L))


def test_tc_batched(gk, orc, cuda):
    graphs = []
    for i in range(24):
        if i % 2:
            A = gk.gen_er(500 + 97 * i, 4000 + 300 * i, seed=100 + i)
        else:
            A = gk.gen_rmat(6 + i % 7, 16, seed=100 + i)
        graphs.append(gk.lower_host(A))
    want = np.array([orc.tc_lower(L) for L in graphs], dtype=np.uint64)
    got_host = gk.tc_count_batched(graphs)
    np.testing.assert_array_equal(got_host, want)
    got_dev = gk.tc_count_batched([dev(L) for L in graphs])
    np.testing.assert_array_equal(got_dev, want)


@pytest.mark.parametrize("sched", ["plain", "learned"])
def test_tc_batched_host_groups(gk, orc, cuda, monkeypatch, sched):
    """Host graphs are copied and counted in groups (the copies of the next
    group overlap the count of this one); a small group size forces many groups,
    some of them holding only edgeless graphs."""
    if sched == "learned":
        from graphkokkos_b200 import sched as S
        S.load_model()
    graphs = []
    for i in range(30):
        if i in (3, 4, 5, 17):
            graphs.append(gk.lower_host(G.empty(7 + i)))
        elif i % 3 == 0:
            graphs.append(gk.lower_host(gk.gen_er(300 + 41 * i, 2500 + 200 * i, seed=500 + i)))
        else:
            graphs.append(gk.lower_host(gk.gen_rmat(5 + i % 6, 16, seed=500 + i)))
    want = np.array([orc.tc_lower(L) for L in graphs], dtype=np.uint64)
    for stage_min in ("1", "3000", "40000"):
        monkeypatch.setenv("GK_BATCH_STAGE_MIN", stage_min)
        np.testing.assert_array_equal(gk.tc_count_batched(graphs, sched=sched), want)
    # host and device graphs mixed in one batch
    mixed = [dev(L) if i % 4 == 1 else L for i, L in enumerate(graphs)]
    np.testing.assert_array_equal(gk.tc_count_batched(mixed, sched=sched), want)


# ---------------------------------------------------------------------------
# general masked SpGEMM with values (plus-times)
# ---------------------------------------------------------------------------
CASES = [
    # (m, k, n, density A, density B, density M)
    (40, 30, 50, 0.2, 0.2, 0.3),
    (300, 200, 250, 0.02, 0.05, 0.04),
    (128, 128, 128, 0.5, 0.5, 0.6),       # long mask rows: chunking in the small variants
    (600, 400, 3000, 0.01, 0.3, 0.2),     # mask rows of ~600 across a wide column range
    (1, 5, 7, 1.0, 1.0, 1.0),
]


@pytest.mark.parametrize("case", CASES)
def test_mxmm_values_every_variant(gk, orc, cuda, case):
    m, k, n, da, db, dm = case
    A = G.random_csr(m, k, da, 1, values=True)
    B = G.random_csr(k, n, db, 2, values=True)
    M = G.random_csr(m, n, dm, 3)
    want = orc.mxmm(A, B, M)
    Ad, Bd, Md = dev(A), dev(B), dev(M)
    for v in range(NV):
        got = gk.mxmm_masked_variant(Ad, Bd, Md, v).cpu().numpy()
        np.testing.assert_array_equal(got, want, err_msg=f"variant {v}")
    for accum in ("auto", "msa", "mca", "hash"):
        got = gk.mxmm_masked(Ad, Bd, Md, accum=accum).cpu().numpy()
        np.testing.assert_array_equal(got, want, err_msg=accum)
    # host buffers through the same entry point
    np.testing.assert_array_equal(gk.mxmm_masked(A, B, M), want)


def test_mxmm_plus_pair(gk, orc, cuda):
    A = G.random_csr(200, 150, 0.05, 4, values=True)
    B = G.random_csr(150, 180, 0.05, 5, values=True)
    M = G.random_csr(200, 180, 0.1, 6)
    import copy
    Ap, Bp = copy.copy(A), copy.copy(B)
    Ap.val = None
    Bp.val = None
    want = orc.mxmm(Ap, Bp, M)
    got = gk.mxmm_masked(dev(A), dev(B), dev(M), semiring="plus_pair").cpu().numpy()
    np.testing.assert_array_equal(got, want)


def test_mxmm_edge_cases(gk, orc, cuda):
    # empty A rows, empty mask rows, empty B, zero-size shapes
    A = G.random_csr(50, 40, 0.05, 7, values=True)
    B = G.empty(40)
    B = type(B)(40, 60, np.zeros(41, dtype=np.int64), np.zeros(0, dtype=np.int32), None, 0)
    M = G.random_csr(50, 60, 0.2, 8)
    got = gk.mxmm_masked(dev(A), dev(B), dev(M)).cpu().numpy()
    assert np.all(got == 0) and len(got) == M.nnz
    Z = G.empty(0)
    assert len(gk.mxmm_masked(Z, Z, Z)) == 0
    with pytest.raises(gk.GkError) as e:
        gk.mxmm_masked(dev(A), dev(A), dev(M))
    assert e.value.code == 1


def test_mxmm_square_graph(gk, orc, cuda):
    A = gk.gen_rmat(11, 16, seed=21)
    want = orc.mxmm(A, A, A)
    Ad = dev(A)
    for v in range(NV):
        np.testing.assert_array_equal(gk.mxmm_masked_variant(Ad, Ad, Ad, v, semiring="plus_pair").cpu().numpy(),
                                      want, err_msg=f"variant {v}")


# ---------------------------------------------------------------------------
# graph ingest on the device
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("scale,seed", [(6, 1), (10, 7), (14, 2), (16, 3)])
def test_device_rmat_equals_host(gk, cuda, scale, seed):
    H = gk.gen_rmat(scale, 16, seed=seed)
    D = gk.gen_rmat(scale, 16, seed=seed, device="cuda")
    assert D.nnz == H.nnz
    np.testing.assert_array_equal(D.rowptr.cpu().numpy(), H.rowptr)
    np.testing.assert_array_equal(D.col.cpu().numpy(), H.col)


def test_device_er_equals_host(gk, cuda):
    H = gk.gen_er(12345, 100000, seed=77)
    D = gk.gen_er(12345, 100000, seed=77, device="cuda")
    np.testing.assert_array_equal(D.rowptr.cpu().numpy(), H.rowptr)
    np.testing.assert_array_equal(D.col.cpu().numpy(), H.col)


def test_device_transforms(gk, orc, cuda):
    A = gk.gen_rmat(12, 8, seed=5)
    L = gk.extract_lower(dev(A))
    orp, ocol = orc.extract_lower(A)
    np.testing.assert_array_equal(L.rowptr.cpu().numpy(), orp)
    np.testing.assert_array_equal(L.col.cpu().numpy(), ocol)
    R = G.random_csr(300, 500, 0.02, 9, values=True)
    T = gk.transpose(dev(R), with_values=True)
    trp, tcol, tval = orc.transpose(R)
    np.testing.assert_array_equal(T.rowptr.cpu().numpy(), trp)
    np.testing.assert_array_equal(T.col.cpu().numpy(), tcol)
    np.testing.assert_array_equal(T.val.cpu().numpy(), tval)
    Th = gk.transpose(R, with_values=True)  # host buffers
    np.testing.assert_array_equal(Th.col, tcol)


def _lower_with_diagonal(n, density, seed):
    """A square L holding entries at and below the diagonal, random values."""
    R = G.random_csr(n, n, density, seed, values=True)
    rp, col, val = np.asarray(R.rowptr), np.asarray(R.col), np.asarray(R.val)
    rows = np.repeat(np.arange(n), np.diff(rp))
    keep = col <= rows
    rows, col, val = rows[keep], col[keep], val[keep]
    nrp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=nrp[1:])
    return G.Csr(n, n, nrp, col.astype(np.int32), val.astype(np.int32), int(len(col)))


def test_device_symm_and_adjacency(gk, orc, cuda):
    """build_symm_from_lower and build_adjacency_matrix on the GPU against the
    reference's own (include/matrix.h:643-696): patterns bit-exact, the
    transpose's entry first on equal columns, values carried."""
    A = gk.gen_rmat(12, 8, seed=5)
    Lh = gk.lower_host(A)
    S = gk.build_symm_from_lower(dev(Lh))
    np.testing.assert_array_equal(S.rowptr.cpu().numpy(), A.rowptr)
    np.testing.assert_array_equal(S.col.cpu().numpy(), A.col)
    for L in (Lh, _lower_with_diagonal(300, 0.05, 4)):
        want_rp, want_col = orc.ref_build_symm(L) if orc.ref_available() else (None, None)
        for X in (dev(L), L):  # device and host buffers
            S = gk.build_symm_from_lower(X, with_values=True)
            rp = S.rowptr.cpu().numpy() if hasattr(S.rowptr, "cpu") else S.rowptr
            col = S.col.cpu().numpy() if hasattr(S.col, "cpu") else S.col
            val = S.val.cpu().numpy() if hasattr(S.val, "cpu") else S.val
            if want_rp is not None:
                np.testing.assert_array_equal(rp, want_rp)
                np.testing.assert_array_equal(col, want_col)
            # values: an entry below the diagonal is L's, above it L^T's; on the
            # diagonal the transpose's copy comes first, then L's (equal values)
            dense = G.dense_of(L)
            rows = np.repeat(np.arange(L.m), np.diff(rp))
            want_val = np.where(col <= rows, dense[rows, col], dense[col, rows])
            np.testing.assert_array_equal(val, want_val)
    Gv = G.random_csr(200, 300, 0.03, 8, values=True)
    for X in (dev(Gv), Gv):
        Adj = gk.build_adjacency_matrix(X)
        np.testing.assert_array_equal(np.asarray(Adj.rowptr.cpu() if hasattr(Adj.rowptr, "cpu") else Adj.rowptr),
                                      Gv.rowptr)
        np.testing.assert_array_equal(np.asarray(Adj.col.cpu() if hasattr(Adj.col, "cpu") else Adj.col), Gv.col)
        assert np.all(np.asarray(Adj.val.cpu() if hasattr(Adj.val, "cpu") else Adj.val) == 1)


def test_learned_without_model_is_an_error(gk, cuda):
    if gk.load().gk_sched_has_model():
        pytest.skip("a model is loaded in this process")
    L = dev(gk.lower_host(G.complete(5)))
    with pytest.raises(gk.GkError) as e:
        gk.tc_count(L, sched="learned")
    assert e.value.code == 1


@pytest.mark.parametrize("scale,seed", [(9, 1), (11, 3), (13, 2)])
def test_tc_vertex_and_lu_match_reference(gk, orc, cuda, scale, seed):
    """Per-vertex triangle counts (C<A> = A·A row sums / 2) and the L·U count
    against the reference's own triangle_counting_vertex / _masked_lu."""
    A = gk.gen_rmat(scale, 16, seed=seed)
    want_v = orc.ref_tc_vertex(A) if scale < 13 else orc.tc_vertex(A)
    got_v = gk.tc_vertex(dev(A)).cpu().numpy()
    np.testing.assert_array_equal(got_v, want_v)
    np.testing.assert_array_equal(gk.tc_vertex(A), want_v)  # host arrays
    want = orc.ref_tc_lu(A) if scale < 13 else orc.tc_lower(gk.lower_host(A))
    assert gk.tc_count_lu(dev(A)) == want == gk.tc_count(gk.lower_host(A))
    from graphkokkos_b200 import sched
    sched.load_model()
    assert gk.tc_count_lu(dev(A), sched="learned") == want


def test_cmask_matches_reference(gk, orc, cuda):
    """C<!M> = A·B against the reference's own mxmm_msa_cmask (values,
    explicit zeros, sorted rows), rectangular shapes, both semirings, host and
    device arrays."""
    for seed in range(3):
        A = G.random_csr(90, 70, 0.08, seed=seed, values=True)
        B = G.random_csr(70, 110, 0.08, seed=seed + 10, values=True)
        M = G.random_csr(90, 110, 0.15, seed=seed + 20)
        want = orc.ref_mxmm_cmask(A, B, M) if orc.ref_available() else orc.mxmm_cmask(A, B, M)
        for X in (gk.mxmm_cmask(A, B, M), gk.mxmm_cmask(dev(A), dev(B), dev(M))):
            got = [np.asarray(x.cpu() if hasattr(x, "cpu") else x) for x in (X.rowptr, X.col, X.val)]
            for g, w in zip(got, want):
                np.testing.assert_array_equal(g, w)
        P = gk.mxmm_cmask(A, B, M, semiring="plus_pair")
        pr, pc, pv = orc.mxmm_cmask(G.random_csr(90, 70, 0.08, seed=seed), G.random_csr(70, 110, 0.08, seed=seed + 10), M)
        np.testing.assert_array_equal(P.rowptr, pr)
        np.testing.assert_array_equal(P.val, pv)


def test_cmask_two_hop_non_edges(gk, orc, cuda):
    """C<!A> = A·A on RMAT graphs (pairs two hops apart that are not edges,
    with their path counts), larger than one product batch at scale 14."""
    for scale, seed in [(10, 1), (14, 2)]:
        A = gk.gen_rmat(scale, 16, seed=seed)
        rp, col, val = orc.mxmm_cmask(A, A, A)
        X = gk.mxmm_cmask(dev(A), dev(A), dev(A))
        np.testing.assert_array_equal(X.rowptr.cpu().numpy(), rp)
        np.testing.assert_array_equal(X.col.cpu().numpy(), col)
        np.testing.assert_array_equal(X.val.cpu().numpy(), val)
