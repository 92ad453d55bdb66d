"""Pins the oracle (CPU restatement, oracle/gk_oracle.cpp) to the reference.

Three kinds of evidence, as the reference ships no test vectors:
  * the reference's own code, compiled unmodified against the Kokkos-API shim
    (oracle/_ref), run on the same seeded inputs (skipped where it was not
    built);
  * golden fixtures generated from that build (tests/golden/, made by
    tests/golden/make_golden.py);
  * closed-form answers on hand-made graphs and independent second methods.
"""
import json
import os

import numpy as np
import pytest

from tests import graphs as G

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def need_ref(orc):
    if not orc.ref_available():
        pytest.skip("reference oracle not built (reference sources absent)")


# ---------------------------------------------------------------------------
# closed forms
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n,tri", [(3, 1), (4, 4), (5, 10), (8, 56)])
def test_tc_complete(gk, orc, n, tri):
    L = gk.lower_host(G.complete(n))
    assert orc.tc_lower(L) == tri
    assert orc.tc_merge(L) == tri


def test_tc_shapes(gk, orc):
    assert orc.tc_lower(gk.lower_host(G.wheel(7))) == 7
    assert orc.tc_lower(gk.lower_host(G.star(9))) == 0
    assert orc.tc_lower(gk.lower_host(G.path(10))) == 0
    assert orc.tc_lower(gk.lower_host(G.disjoint_triangles(5))) == 5
    assert orc.tc_lower(gk.lower_host(G.empty(6))) == 0


def test_ktruss_closed_forms(orc):
    # K5 is a 5-truss (every edge in 3 triangles); a wheel's rim edges have support 1
    rp, col, iters, _ = orc.ktruss(G.complete(5), 5)
    assert len(col) == 20 and iters == 1
    rp, col, iters, _ = orc.ktruss(G.wheel(8), 4)
    assert len(col) == 0
    # K4 plus a pendant edge: the pendant has support 0 and is removed for k=3
    A = G.from_edges(5, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (3, 4)])
    rp, col, iters, _ = orc.ktruss(A, 3)
    assert len(col) == 12 and iters == 2


def test_bc_closed_forms(orc):
    # path 0-1-2-3-4, all sources: bc(v) = 2 * (#pairs separated by v)
    P = G.path(5)
    bc = orc.bc_f64(P, range(5))
    np.testing.assert_allclose(bc, [0, 6, 8, 6, 0])
    # star with 6 leaves, all sources: hub = 6*5
    bc = orc.bc_f64(G.star(6), range(7))
    assert bc[0] == pytest.approx(30.0)
    assert np.all(bc[1:] == 0)


def test_bc_matches_brandes(gk, orc):
    A = gk.gen_rmat(9, 8, seed=11)
    rng = np.random.default_rng(3)
    src = rng.choice(A.m, size=40, replace=False)
    ours = orc.bc_f64(A, src)
    ref = G.brandes_f64(A, src)
    np.testing.assert_allclose(ours, ref, rtol=1e-12, atol=1e-9)


def test_bc_directed_matches_brandes(orc):
    A = G.random_csr(60, 60, 0.06, seed=5)
    src = np.arange(0, 60, 3)
    np.testing.assert_allclose(orc.bc_f64(A, src), G.brandes_f64(A, src), rtol=1e-12, atol=1e-9)


def test_mxmm_dense(orc):
    for seed in range(4):
        A = G.random_csr(37, 23, 0.2, seed, values=True)
        B = G.random_csr(23, 41, 0.25, seed + 10, values=True)
        M = G.random_csr(37, 41, 0.3, seed + 20)
        c = orc.mxmm(A, B, M)
        full = G.dense_of(A) @ G.dense_of(B)
        rp, col = M.rowptr, M.col
        want = np.concatenate([full[i, col[rp[i]:rp[i + 1]]] for i in range(M.m)])
        np.testing.assert_array_equal(c, want.astype(np.int32))


def test_transforms(gk, orc):
    A = gk.gen_rmat(8, 8, seed=4)
    orp, ocol = orc.extract_lower(A)
    L = gk.lower_host(A)
    np.testing.assert_array_equal(orp, L.rowptr)
    np.testing.assert_array_equal(ocol, L.col)
    trp, tcol, _ = orc.transpose(A)
    np.testing.assert_array_equal(trp, A.rowptr)  # symmetric
    np.testing.assert_array_equal(tcol, A.col)


# ---------------------------------------------------------------------------
# against the reference's own code
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("scale,seed", [(8, 1), (10, 2), (12, 3)])
def test_tc_vs_reference(gk, orc, scale, seed):
    need_ref(orc)
    A = gk.gen_rmat(scale, 16, seed=seed)
    L = gk.lower_host(A)
    got = orc.tc_lower(L)
    for accum in ("msa", "mca"):
        assert orc.ref_tc(A, accum) == got
    # the sequential MCA agrees too; the sequential MSA (matrix_la.h:696-731)
    # does not reset its value array between rows, so its explicit zeros can
    # carry stale values from earlier rows (a reference defect, not tested)
    assert orc.ref_tc(A, "mca", parallel=False) == got


@pytest.mark.parametrize("scale,seed", [(8, 1), (10, 2), (12, 3)])
def test_tc_vertex_and_lu_vs_reference(gk, orc, scale, seed):
    """triangle_counting_vertex (src/main.cpp:16-39) and _masked_lu (:42-66)
    of the reference (msa and mca) against the restatement."""
    need_ref(orc)
    A = gk.gen_rmat(scale, 16, seed=seed)
    want = orc.tc_vertex(A)
    np.testing.assert_array_equal(orc.ref_tc_vertex(A, accum=0), want)
    np.testing.assert_array_equal(orc.ref_tc_vertex(A, accum=1), want)
    tri = orc.tc_lower(gk.lower_host(A))
    assert int(want.astype(np.int64).sum()) == 3 * tri
    assert orc.ref_tc_lu(A, accum=0) == orc.ref_tc_lu(A, accum=1) == tri


def test_tc_vertex_closed_forms(orc):
    for n in (4, 6, 9):  # every vertex of K_n lies in C(n-1, 2) triangles
        np.testing.assert_array_equal(orc.tc_vertex(G.complete(n)), np.full(n, (n - 1) * (n - 2) // 2))
    np.testing.assert_array_equal(orc.tc_vertex(G.star(6)), np.zeros(7))


def test_mxmm_vs_reference(gk, orc):
    need_ref(orc)
    for seed in range(3):
        A = G.random_csr(120, 90, 0.05, seed, values=True)
        B = G.random_csr(90, 110, 0.06, seed + 1, values=True)
        M = G.random_csr(120, 110, 0.08, seed + 2)
        want = orc.mxmm(A, B, M)
        for accum in ("msa", "mca"):
            np.testing.assert_array_equal(orc.ref_mxmm(A, B, M, accum), want)
        np.testing.assert_array_equal(orc.ref_mxmm(A, B, M, "naive", parallel=False), want)


@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_ktruss_vs_reference(gk, orc, k):
    need_ref(orc)
    A = gk.gen_rmat(10, 16, seed=7)
    rp, col, iters, _ = orc.ktruss(A, k)
    rrp, rcol, riters = orc.ref_ktruss(A, k)
    np.testing.assert_array_equal(rp, rrp)
    np.testing.assert_array_equal(col, rcol)
    assert iters == riters


def test_transforms_vs_reference(gk, orc):
    need_ref(orc)
    A = gk.gen_rmat(9, 8, seed=9)
    rrp, rcol = orc.ref_extract_lower(A)
    orp, ocol = orc.extract_lower(A)
    np.testing.assert_array_equal(rrp, orp)
    np.testing.assert_array_equal(rcol, ocol)
    L = gk.lower_host(A)
    srp, scol = orc.ref_build_symm(L)
    np.testing.assert_array_equal(srp, A.rowptr)
    np.testing.assert_array_equal(scol, A.col)
    D = G.random_csr(50, 70, 0.1, seed=3, values=True)
    a = orc.ref_transpose(D)
    b = orc.transpose(D)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_bc_vs_reference_float(gk, orc):
    """The reference BC is FP32 with int32 path counts; on a graph where no
    count overflows it must agree with the FP64 restatement to float precision.
    Sampled sources are relabelled to 0..b-1 (the reference's only sources)."""
    need_ref(orc)
    A = gk.gen_rmat(10, 8, seed=12)
    rng = np.random.default_rng(4)
    src = rng.choice(A.m, size=64, replace=False)
    ours = orc.bc_f64(A, src)
    R, perm = orc.relabel_sources_first(A, src)
    ref = orc.ref_bc_float(R, len(src))
    ref_orig = ref[perm]
    np.testing.assert_allclose(ref_orig, ours, rtol=2e-4, atol=1e-2)


# ---------------------------------------------------------------------------
# golden fixtures (generated from the reference build; valid without it)
# ---------------------------------------------------------------------------
def _golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_golden_tc(gk, orc):
    g = _golden("tc.json")
    for case in g["cases"]:
        A = gk.gen_rmat(case["scale"], case["edge_factor"], seed=case["seed"])
        assert A.nnz == case["nnz_sym"]
        L = gk.lower_host(A)
        assert L.nnz == case["nnz_lower"]
        assert orc.tc_lower(L) == case["triangles"]


def test_golden_ktruss(gk, orc):
    g = _golden("ktruss.json")
    for case in g["cases"]:
        A = gk.gen_rmat(case["scale"], case["edge_factor"], seed=case["seed"])
        rp, col, iters, _ = orc.ktruss(A, case["k"])
        assert iters == case["iterations"]
        assert len(col) == case["nnz"]
        assert int(np.bitwise_xor.reduce((col.astype(np.int64) * 2654435761 + np.repeat(
            np.arange(A.m), np.diff(rp))) & 0xFFFFFFFF)) == case["xor_hash"]


def test_golden_mxmm(orc):
    g = _golden("mxmm.json")
    for case in g["cases"]:
        A = G.random_csr(*case["A"], values=True)
        B = G.random_csr(*case["B"], values=True)
        M = G.random_csr(*case["M"])
        c = orc.mxmm(A, B, M)
        assert int(c.astype(np.int64).sum()) == case["sum"]
        assert int((c.astype(np.int64) * np.arange(1, len(c) + 1)).sum()) == case["weighted_sum"]


def test_golden_bc(gk, orc):
    g = _golden("bc.json")
    for case in g["cases"]:
        A = gk.gen_rmat(case["scale"], case["edge_factor"], seed=case["seed"])
        src = np.asarray(case["sources"])
        ours = orc.bc_f64(A, src)
        ref = np.asarray(case["bc_ref_float"], dtype=np.float64)
        np.testing.assert_allclose(ours, ref, rtol=2e-4, atol=1e-2)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_cmask_vs_reference(orc, seed):
    """mxmm_msa_cmask (include/matrix_la.h:733-934): the restatement gives the
    reference's C<!M> = A·B entry for entry, values included, on rectangular
    operands and on the two-hop non-edges of a graph (A, A, A)."""
    need_ref(orc)
    A = G.random_csr(90, 70, 0.08, seed=seed, values=True)
    B = G.random_csr(70, 110, 0.08, seed=seed + 10, values=True)
    M = G.random_csr(90, 110, 0.1, seed=seed + 20)
    for a, b, m in ((A, B, M), (M, G.random_csr(110, 90, 0.05, seed=seed), G.random_csr(90, 90, 0.0, seed=1))):
        want = orc.ref_mxmm_cmask(a, b, m)
        got = orc.mxmm_cmask(a, b, m)
        for w, g in zip(want, got):
            np.testing.assert_array_equal(w, g)
    S = G.random_csr(120, 120, 0.05, seed=seed)
    for w, g in zip(orc.ref_mxmm_cmask(S, S, S, parallel=False), orc.mxmm_cmask(S, S, S)):
        np.testing.assert_array_equal(w, g)


# ---------------------------------------------------------------------------
# operators of the alternate BC formulation (include/matrix_la.h:182-328)
# ---------------------------------------------------------------------------
def disjoint_pair(m, n, seed, density=0.15):
    """Sparse A, B (m x n, int values) with disjoint patterns; every row of A
    ends at column n-1, which B never uses, so no row ends with B entries
    (the reference's B-tail copy is then not reached)."""
    rng = np.random.default_rng(seed)
    pick = rng.random((m, n - 1)) < density
    side = rng.random((m, n - 1)) < 0.5
    a = np.zeros((m, n), dtype=bool)
    a[:, : n - 1] = pick & side
    a[:, n - 1] = True
    b = np.zeros((m, n), dtype=bool)
    b[:, : n - 1] = pick & ~side

    def csr(mask):
        r, c = np.nonzero(mask)
        rp = np.zeros(m + 1, dtype=np.int64)
        np.cumsum(np.bincount(r, minlength=m), out=rp[1:])
        return G.Csr(m, n, rp, c.astype(np.int32), rng.integers(-9, 10, len(c)).astype(np.int32), len(c))
    return csr(a), csr(b)


@pytest.mark.parametrize("seed", [1, 2])
def test_add_nointersect_vs_reference(orc, seed):
    need_ref(orc)
    A, B = disjoint_pair(70, 40, seed)
    for w, g in zip(orc.ref_add_nointersect(A, B), orc.add_nointersect(A, B)):
        np.testing.assert_array_equal(w, g)


def test_add_nointersect_closed_form(orc):
    # row 0 ends with B entries (the case the reference mis-copies), row 1 is
    # B only, row 2 A only, row 3 empty
    A = G.Csr(4, 5, np.array([0, 1, 1, 3, 3]), np.array([1, 0, 4], dtype=np.int32),
              np.array([10, 20, 30], dtype=np.int32), 3)
    B = G.Csr(4, 5, np.array([0, 3, 5, 5, 5]), np.array([0, 2, 3, 1, 4], dtype=np.int32),
              np.array([1, 2, 3, 4, 5], dtype=np.int32), 5)
    rp, col, val = orc.add_nointersect(A, B)
    np.testing.assert_array_equal(rp, [0, 4, 6, 8, 8])
    np.testing.assert_array_equal(col, [0, 1, 2, 3, 1, 4, 0, 4])
    np.testing.assert_array_equal(val, [1, 10, 2, 3, 4, 5, 20, 30])


@pytest.mark.parametrize("seed", [3, 4])
def test_dense_operators_vs_reference(orc, seed):
    """The dense masked eWiseMult, fuseEWiseMultAdd and mxmm_spd of the
    reference against the restatement, bit for bit (FP64)."""
    need_ref(orc)
    rng = np.random.default_rng(seed)
    m, k, n = 37, 29, 45
    A = rng.standard_normal((m, n))
    B = rng.standard_normal((m, n))
    C = rng.standard_normal((m, n))
    M = G.random_csr(m, n, 0.2, seed=seed)
    np.testing.assert_array_equal(orc.ref_dense_ewise_mult_masked(A, B, M), orc.dense_ewise_mult_masked(A, B, M))
    np.testing.assert_array_equal(orc.ref_fuse_ewise_mult_add(A, B, C), orc.fuse_ewise_mult_add(A, B, C))
    S = G.random_csr(m, k, 0.25, seed=seed + 1)
    sval = rng.standard_normal(S.nnz)
    D = rng.standard_normal((k, n))
    np.testing.assert_array_equal(orc.ref_mxmm_spd(S, D, M, sval), orc.mxmm_spd(S, D, M, sval))
    np.testing.assert_array_equal(orc.ref_mxmm_spd(S, D, M), orc.mxmm_spd(S, D, M))
    # closed form: a pattern-only A sums B's rows; the mask selects columns
    want = np.zeros((m, n))
    dense_s = G.dense_of(S) != 0
    for i in range(m):
        cols = np.asarray(M.col[M.rowptr[i]:M.rowptr[i + 1]])
        want[i, cols] = D[dense_s[i]].sum(axis=0)[cols]
    np.testing.assert_allclose(orc.mxmm_spd(S, D, M), want, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("scale,seed", [(8, 1), (12, 3), (15, 2)])
def test_oracle_generator_equals_library_builder(gk, orc, scale, seed):
    """The oracle's own restatement of the seeded generators (used by the
    CPU side of the benchmark, which must not load the product library)
    gives the library builder's graphs bit for bit."""
    A = gk.gen_rmat(scale, 16, seed=seed)
    B = orc.gen_rmat(scale, 16, seed)
    np.testing.assert_array_equal(A.rowptr, B.rowptr)
    np.testing.assert_array_equal(A.col, B.col)
    L = gk.lower_host(A)
    Lo = orc.gen_rmat(scale, 16, seed, lower=True)
    np.testing.assert_array_equal(L.rowptr, Lo.rowptr)
    np.testing.assert_array_equal(L.col, Lo.col)
    E = gk.gen_er(3000 + scale, 20000, seed=seed)
    Eo = orc.gen_er(3000 + scale, 20000, seed)
    np.testing.assert_array_equal(E.rowptr, Eo.rowptr)
    np.testing.assert_array_equal(E.col, Eo.col)
