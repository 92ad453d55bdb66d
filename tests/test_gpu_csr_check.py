"""Malformed CSR inputs are refused with GK_ERR_INVALID_CSR before any kernel
indexes through them (spMtx's invariants, include/matrix.h:33-43: row pointers
from 0 to nz, non-decreasing; columns in range; the masked products, triangle
counts and k-truss also need sorted, duplicate-free rows, as the reference's
extract_lower_triangle and MCA merge do, matrix.h:709, matrix_la.h:437-461).
Every malformed input here is built on the host and rejected by the library's
check kernel, which reads only inside the declared arrays."""
import numpy as np
import pytest

from tests import graphs as G

pytestmark = pytest.mark.gpu


def dev(csr):
    import torch
    return type(csr)(csr.m, csr.n, torch.as_tensor(csr.rowptr).cuda(), torch.as_tensor(csr.col).cuda(),
                     None if csr.val is None else torch.as_tensor(csr.val).cuda(), csr.nnz)


def bad_copies(gk, L):
    """(label, matrix, message fragment) for each defect planted in a copy of L."""
    Csr = type(L)
    rp, col = np.array(L.rowptr), np.array(L.col)
    r = int(np.argmax(np.diff(rp) >= 3))  # a row with at least three entries
    out = []
    c = col.copy(); c[rp[r]] = L.n
    out.append(("column = n", Csr(L.m, L.n, rp, c, None, L.nnz), "out of range"))
    c = col.copy(); c[rp[r] + 1] = -1
    out.append(("negative column", Csr(L.m, L.n, rp, c, None, L.nnz), "out of range"))
    c = col.copy(); c[rp[r]], c[rp[r] + 1] = c[rp[r] + 1], c[rp[r]]
    out.append(("unsorted row", Csr(L.m, L.n, rp, c, None, L.nnz), "not strictly increasing"))
    c = col.copy(); c[rp[r] + 1] = c[rp[r]]
    out.append(("duplicate", Csr(L.m, L.n, rp, c, None, L.nnz), "not strictly increasing"))
    p = rp.copy(); p[r + 1], p[r] = p[r], p[r + 1]
    out.append(("decreasing rowptr", Csr(L.m, L.n, p, col, None, L.nnz), "row pointers"))
    p = rp.copy(); p[-1] = L.nnz - 1
    out.append(("rowptr[m] != nnz", Csr(L.m, L.n, p, col, None, L.nnz), "row pointers"))
    p = rp.copy(); p[r + 1] = L.nnz + 5
    out.append(("rowptr past nnz", Csr(L.m, L.n, p, col, None, L.nnz), "row pointers"))
    return out


def test_tc_and_mxmm_refuse_malformed_csr(gk, orc, cuda):
    A = gk.gen_rmat(9, 8, seed=3)
    L = gk.lower_host(A)
    good = orc.tc_lower(L)
    for label, X, msg in bad_copies(gk, L):
        for arg in (X, dev(X)):
            with pytest.raises(gk.GkError, match=msg) as e:
                gk.tc_count(arg)
            assert e.value.code == gk._lib.GK_ERR_INVALID_CSR, label
        with pytest.raises(gk.GkError, match=msg):
            gk.mxmm_masked(L, L, X)  # as the mask
        if "rowptr" in label or "column" in label:
            with pytest.raises(gk.GkError, match=msg):
                gk.mxmm_masked(X, L, L)  # A needs only a valid structure
    assert gk.tc_count(L) == good  # the library still works after the refusals


def test_unsorted_rows_allowed_where_order_does_not_matter(gk, orc, cuda):
    A = G.random_csr(60, 50, 0.1, seed=2, values=True)
    B = G.random_csr(50, 70, 0.1, seed=3, values=True)
    M = G.random_csr(60, 70, 0.2, seed=4)
    want = orc.mxmm(A, B, M)
    # reverse every row of A: the product is the same
    rp = np.asarray(A.rowptr)
    col, val = np.array(A.col), np.array(A.val)
    for i in range(A.m):
        col[rp[i]:rp[i + 1]] = col[rp[i]:rp[i + 1]][::-1].copy()
        val[rp[i]:rp[i + 1]] = val[rp[i]:rp[i + 1]][::-1].copy()
    Ar = type(A)(A.m, A.n, rp, col, val, A.nnz)
    np.testing.assert_array_equal(gk.mxmm_masked(Ar, B, M), want)
    with pytest.raises(gk.GkError, match="not strictly increasing"):
        gk.mxmm_masked(A, Ar.__class__(B.m, B.n, np.asarray(B.rowptr), np.array(B.col)[::-1].copy(),
                                       np.array(B.val), B.nnz), M)


def test_ktruss_bc_batch_refuse_malformed_csr(gk, cuda):
    A = gk.gen_rmat(8, 8, seed=5)
    for label, X, msg in bad_copies(gk, A):
        with pytest.raises(gk.GkError, match=msg):
            gk.ktruss(X, 4)
        if "unsorted" not in label and "duplicate" not in label:
            with pytest.raises(gk.GkError, match=msg):
                gk.bc_batch(X, [0, 1])
    # a graph of the batch whose column leaves its own vertex range is refused
    Ls = [gk.lower_host(gk.gen_rmat(6 + i, 8, seed=40 + i)) for i in range(4)]
    rp, col = np.asarray(Ls[1].rowptr), np.array(Ls[1].col)
    r = int(np.argmax(np.diff(rp) >= 1))
    col[rp[r]] = Ls[1].m + 3  # a vertex of the next graph in the combined matrix
    bad = type(Ls[1])(Ls[1].m, Ls[1].n, rp, col, None, Ls[1].nnz)
    with pytest.raises(gk.GkError, match="out of range"):
        gk.tc_count_batched([Ls[0], bad, Ls[2], Ls[3]])
    p = np.array(Ls[2].rowptr); p[-1] -= 1
    with pytest.raises(gk.GkError, match="row pointers"):
        gk.tc_count_batched([Ls[0], Ls[1], type(Ls[2])(Ls[2].m, Ls[2].n, p, Ls[2].col, None, Ls[2].nnz), Ls[3]])
    p = np.array(Ls[3].rowptr); p[1] = -7
    with pytest.raises(gk.GkError, match="row pointers"):
        gk.tc_count_batched([Ls[0], Ls[1], Ls[2], type(Ls[3])(Ls[3].m, Ls[3].n, p, Ls[3].col, None, Ls[3].nnz)])
