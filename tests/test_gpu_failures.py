"""Error paths without a GPU fault: every scratch allocation of an operator
is made to fail in turn (host-side injection, gk_inject_alloc_failure), the
call must return GK_ERR_OOM, and the next call — injection off — must give
the right answer on the same stream.  Also the invariances the results must
have: triangle counts and BC scores under a relabelling of the vertices."""
import numpy as np
import pytest

from tests import graphs as G

pytestmark = pytest.mark.gpu


def dev(csr):
    return csr.to("cuda")


def relabel(A, perm):
    """A with vertex v renamed perm[v] (sorted rows)."""
    rp = np.asarray(A.rowptr)
    col = np.asarray(A.col)
    rows = np.repeat(np.arange(A.m), np.diff(rp))
    r, c = perm[rows], perm[col]
    order = np.lexsort((c, r))
    r, c = r[order], c[order]
    nrp = np.zeros(A.m + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=A.m), out=nrp[1:])
    return G.Csr(A.m, A.n, nrp, c.astype(np.int32), None, len(c))


def drive_failures(gk, op, check, limit=80):
    """Fails allocation 0, 1, 2, ... of op until it needs fewer than that."""
    lib = gk.load()
    failures = 0
    try:
        for after in range(limit):
            lib.gk_inject_alloc_failure(after)
            try:
                out = op()
            except gk.GkError as e:
                assert e.code == gk._lib.GK_ERR_OOM, str(e)
                failures += 1
                lib.gk_inject_alloc_failure(-1)
                check(op())  # the library is still usable
                continue
            lib.gk_inject_alloc_failure(-1)
            check(out)
            break
        else:
            pytest.fail("the operator kept allocating")
    finally:
        lib.gk_inject_alloc_failure(-1)
    assert failures > 0


def test_allocation_failures_leave_the_library_usable(gk, orc, cuda):
    A = gk.gen_rmat(10, 16, seed=4)
    L = gk.lower_host(A)
    tri = orc.tc_lower(L)
    drive_failures(gk, lambda: gk.tc_count(L), lambda got: got == tri or pytest.fail("tc"))
    drive_failures(gk, lambda: gk.tc_count(dev(L), sched="plain"), lambda got: got == tri or pytest.fail("tc dev"))
    rp, col, iters, _ = orc.ktruss(A, 4)

    def kt_ok(res):
        T, it = res
        assert it == iters and np.array_equal(T.col.cpu().numpy(), col)
    drive_failures(gk, lambda: gk.ktruss(dev(A), 4), kt_ok)
    src = np.arange(24)
    want_bc = orc.bc_f64(A, src)
    drive_failures(gk, lambda: gk.bc_batch(A, src),
                   lambda got: G.assert_bc_close(got, want_bc))
    graphs = [gk.lower_host(gk.gen_rmat(6 + i % 3, 16, seed=70 + i)) for i in range(6)]
    want = np.array([orc.tc_lower(x) for x in graphs], dtype=np.uint64)
    drive_failures(gk, lambda: gk.tc_count_batched(graphs),
                   lambda got: np.testing.assert_array_equal(got, want))
    crp, ccol, cval = orc.mxmm_cmask(A, A, A)
    drive_failures(gk, lambda: gk.mxmm_cmask(A, A, A),
                   lambda C: np.testing.assert_array_equal(np.asarray(C.col), ccol))


@pytest.mark.parametrize("seed", [1, 2])
def test_counts_and_scores_survive_relabelling(gk, orc, cuda, seed):
    A = gk.gen_rmat(11, 16, seed=seed)
    perm = np.random.default_rng(seed).permutation(A.m).astype(np.int64)
    P = relabel(A, perm)
    assert gk.tc_count(gk.lower_host(P)) == gk.tc_count(gk.lower_host(A)) == orc.tc_lower(gk.lower_host(A))
    np.testing.assert_array_equal(gk.tc_vertex(P)[perm], gk.tc_vertex(A))
    src = np.arange(0, A.m, 37)
    bc_a = gk.bc_batch(A, src)
    bc_p = gk.bc_batch(P, perm[src])
    G.assert_bc_close(bc_p[perm], bc_a)
    assert np.all(bc_a >= 0)
