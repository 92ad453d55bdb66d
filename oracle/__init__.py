"""Oracle bindings — TEST INFRASTRUCTURE ONLY.

Loads the CPU restatement (oracle/_build/libgk_oracle.so, built from
oracle/gk_oracle.cpp) and, when it was built, the reference compiled against
the Kokkos-API shim (oracle/_ref/libgk_ref.so).  Only tests/, the smoke check
and bench.py's CPU-baseline leg may import this package; the product never
does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout whose sources the reference oracle compiles in place:
# GK_REFERENCE_DIR, else the checkout's location on the build host.
REFERENCE_DIR = os.environ.get("GK_REFERENCE_DIR", "/root/reference")


def reference_present():
    return os.path.isdir(os.path.join(REFERENCE_DIR, "include"))
PORT_PATH = os.path.join(HERE, "_build", "libgk_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libgk_ref.so")

_port = None
_ref = None


def build(ref=True, adapter=False):
    """Builds the port (always), the reference oracle (when the reference
    sources are present) and, with adapter=True, the reference-side adapter
    of the integration guide (needs libgk_b200.so built first)."""
    targets = ["port"] + (["ref"] if ref else []) + (["adapter"] if adapter else [])
    env = dict(os.environ, GK_REFERENCE_DIR=REFERENCE_DIR if reference_present() else "")
    out = subprocess.run(["make", "-C", HERE] + targets, capture_output=True, text=True, env=env)
    if out.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{out.stdout}\n{out.stderr}")


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_PATH):
            build(ref=False)
        _port = ctypes.CDLL(PORT_PATH)
    return _port


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            raise RuntimeError("reference oracle oracle/_ref/libgk_ref.so was not built")
        _ref = ctypes.CDLL(REF_PATH)
    return _ref


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _host(csr):
    """(m, n, rowptr int64, col int32, val int32|None) as contiguous numpy."""
    rp = np.ascontiguousarray(np.asarray(csr.rowptr if not hasattr(csr.rowptr, "cpu") else csr.rowptr.cpu().numpy(),
                                         dtype=np.int64))
    col = np.ascontiguousarray(np.asarray(csr.col if not hasattr(csr.col, "cpu") else csr.col.cpu().numpy(),
                                          dtype=np.int32))
    val = None
    if csr.val is not None:
        v = csr.val.cpu().numpy() if hasattr(csr.val, "cpu") else csr.val
        val = np.ascontiguousarray(np.asarray(v, dtype=np.int32))
    return csr.m, csr.n, rp, col[: int(rp[-1])], val


I64 = ctypes.c_int64


# ----- port (restatement) -------------------------------------------------------
def tc_lower(L):
    m, _, rp, col, _ = _host(L)
    out = ctypes.c_uint64(0)
    port().orc_tc_lower(I64(m), _p(rp), _p(col), ctypes.byref(out))
    return int(out.value)


def tc_rows(L, row_begin, row_end):
    m, _, rp, col, _ = _host(L)
    out = ctypes.c_uint64(0)
    port().orc_tc_rows(I64(m), _p(rp), _p(col), I64(row_begin), I64(row_end), ctypes.byref(out))
    return int(out.value)


def tc_rows_sample(L, rows, kind="reference"):
    """Bounded CPU sample of triangle counting over the listed rows of L (for
    a representative sample: a sorted uniform random choice of rows).
    kind "reference": the reference's mxmm_msa (oracle/_ref); "port": the
    restatement.  Returns (partial count, sampled nnz, seconds, threads)."""
    m, _, rp, col, _ = _host(L)
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int64))
    out = ctypes.c_int64(0) if kind == "reference" else ctypes.c_uint64(0)
    nz = ctypes.c_int64(0)
    sec = ctypes.c_double(0.0)
    lib = ref() if kind == "reference" else port()
    fn = lib.ref_tc_rows_sample if kind == "reference" else lib.orc_tc_rows_sample
    r = fn(I64(m), _p(rp), _p(col), I64(len(rows)), _p(rows), ctypes.byref(out), ctypes.byref(nz), ctypes.byref(sec))
    if r != 0:
        raise RuntimeError("tc_rows_sample failed")
    threads = ref().ref_get_threads() if kind == "reference" else os.cpu_count()
    return int(out.value), int(nz.value), float(sec.value), int(threads)


def tc_all_rows(L, kind="reference"):
    """tc_rows_sample over every row of L."""
    return tc_rows_sample(L, np.arange(L.m, dtype=np.int64), kind)


def tc_merge(L):
    m, _, rp, col, _ = _host(L)
    out = ctypes.c_uint64(0)
    port().orc_tc_merge(I64(m), _p(rp), _p(col), ctypes.byref(out))
    return int(out.value)


def tc_vertex(A):
    """Triangles through each vertex of a symmetric adjacency (int32)."""
    m, _, rp, col, _ = _host(A)
    out = np.zeros(m, dtype=np.int32)
    port().orc_tc_vertex(I64(m), _p(rp), _p(col), _p(out))
    return out


def tc_row_sums(L):
    m, _, rp, col, _ = _host(L)
    out = np.zeros(m, dtype=np.uint64)
    port().orc_tc_row_sums(I64(m), _p(rp), _p(col), _p(out))
    return out


def mxmm(A, B, M):
    am, an, arp, acol, aval = _host(A)
    bm, bn, brp, bcol, bval = _host(B)
    mm, mn, mrp, mcol, _ = _host(M)
    out = np.zeros(int(mrp[-1]), dtype=np.int32)
    r = port().orc_mxmm_masked(I64(am), I64(an), _p(arp), _p(acol), _p(aval), I64(bm), I64(bn), _p(brp), _p(bcol),
                               _p(bval), I64(mm), I64(mn), _p(mrp), _p(mcol), _p(out))
    if r != 0:
        raise ValueError("oracle mxmm: shape mismatch")
    return out


def _cmask(fn, A, B, M, *extra):
    am, an, arp, acol, aval = _host(A)
    bm, bn, brp, bcol, bval = _host(B)
    mm, mn, mrp, mcol, _ = _host(M)
    rp = np.zeros(am + 1, dtype=np.int64)
    args = (I64(am), I64(an), _p(arp), _p(acol), _p(aval), I64(bm), I64(bn), _p(brp), _p(bcol), _p(bval),
            I64(mm), I64(mn), _p(mrp), _p(mcol))
    if fn(*extra, *args, _p(rp), None, None) != 0:
        raise ValueError("complement-masked product failed")
    col = np.zeros(int(rp[-1]), dtype=np.int32)
    val = np.zeros(int(rp[-1]), dtype=np.int32)
    if fn(*extra, *args, _p(rp), _p(col), _p(val)) != 0:
        raise ValueError("complement-masked product failed")
    return rp, col, val


def mxmm_cmask(A, B, M):
    """C<!M> = A·B (mxmm_msa_cmask semantics): (rowptr, col, val)."""
    return _cmask(port().orc_mxmm_cmask, A, B, M)


def ref_mxmm_cmask(A, B, M, parallel=True):
    """The reference's own mxmm_msa_cmask (matrix_la.h:733-934)."""
    return _cmask(ref().ref_mxmm_cmask, A, B, M, ctypes.c_int(1 if parallel else 0))


def _f64(a):
    return np.ascontiguousarray(np.asarray(a.cpu().numpy() if hasattr(a, "cpu") else a, dtype=np.float64))


def _add_nointersect(fn, extra, A, B):
    m, n, arp, acol, aval = _host(A)
    _, _, brp, bcol, bval = _host(B)
    nnz = int(arp[-1]) + int(brp[-1])
    crp = np.zeros(m + 1, dtype=np.int64)
    ccol = np.zeros(max(nnz, 1), dtype=np.int32)
    cval = np.zeros(max(nnz, 1), dtype=np.int32)
    if fn(*extra, _p(arp), _p(acol), _p(aval), _p(brp), _p(bcol), _p(bval), _p(crp), _p(ccol), _p(cval)) != 0:
        raise ValueError("add_nointersect failed")
    return crp, ccol[:nnz], cval[:nnz]


def add_nointersect(A, B):
    """C = A + B, the true merge (add_nointersect semantics): (rowptr, col, val)."""
    return _add_nointersect(port().orc_add_nointersect, (I64(A.m),), A, B)


def ref_add_nointersect(A, B):
    """The reference's own add_nointersect (matrix_la.h:287-328); valid only
    where every row's last entry comes from A."""
    return _add_nointersect(ref().ref_add_nointersect, (I64(A.m), I64(A.n)), A, B)


def _ewise(fn, A, B, M):
    A, B = _f64(A), _f64(B)
    m, n = A.shape
    _, _, mrp, mcol, _ = _host(M)
    C = np.empty((m, n), dtype=np.float64)
    fn(I64(m), I64(n), _p(A), _p(B), _p(mrp), _p(mcol), _p(C))
    return C


def dense_ewise_mult_masked(A, B, M):
    return _ewise(port().orc_dense_ewise_mult_masked, A, B, M)


def ref_dense_ewise_mult_masked(A, B, M):
    return _ewise(ref().ref_dense_ewise_mult_masked, A, B, M)


def _fuse(fn, A, B, C):
    A, B, C = _f64(A).ravel(), _f64(B).ravel(), _f64(C).ravel().copy()
    fn(I64(C.size), _p(A), _p(B), _p(C))
    return C


def fuse_ewise_mult_add(A, B, C):
    """C + A .* B (a new array)."""
    return _fuse(port().orc_fuse_ewise_mult_add, A, B, C).reshape(np.shape(C))


def ref_fuse_ewise_mult_add(A, B, C):
    return _fuse(ref().ref_fuse_ewise_mult_add, A, B, C).reshape(np.shape(C))


def mxmm_spd(A, B, M, A_val=None):
    """C<M> = A·B with dense B, dense result (mxmm_spd semantics)."""
    m, _, arp, acol, _ = _host(A)
    B = _f64(B)
    n = B.shape[1]
    _, _, mrp, mcol, _ = _host(M)
    av = None if A_val is None else _f64(A_val)
    C = np.empty((m, n), dtype=np.float64)
    port().orc_mxmm_spd(I64(m), _p(arp), _p(acol), _p(av), I64(n), _p(B), _p(mrp), _p(mcol), _p(C))
    return C


def ref_mxmm_spd(A, B, M, A_val=None):
    """The reference's own mxmm_spd (matrix_la.h:230-258), FP64."""
    m, k, arp, acol, _ = _host(A)
    B = _f64(B)
    n = B.shape[1]
    _, _, mrp, mcol, _ = _host(M)
    av = None if A_val is None else _f64(A_val)
    C = np.empty((m, n), dtype=np.float64)
    ref().ref_mxmm_spd(I64(m), I64(k), _p(arp), _p(acol), _p(av), I64(n), _p(B), _p(mrp), _p(mcol), _p(C))
    return C


def ktruss(A, k, record=64):
    m, _, rp, col, _ = _host(A)
    orp = np.zeros(m + 1, dtype=np.int64)
    ocol = np.zeros(max(len(col), 1), dtype=np.int32)
    nnz = ctypes.c_int64(0)
    iters = ctypes.c_int(0)
    per = np.zeros(record, dtype=np.int64)
    port().orc_ktruss(I64(m), _p(rp), _p(col), ctypes.c_int(k), _p(orp), _p(ocol), ctypes.byref(nnz),
                      ctypes.byref(iters), _p(per), ctypes.c_int(record))
    return orp, ocol[: nnz.value].copy(), int(iters.value), per[: min(iters.value, record)].copy()


def bc_f64(A, sources):
    m, _, rp, col, val = _host(A)
    src = np.ascontiguousarray(np.asarray(sources, dtype=np.int32))
    out = np.zeros(m, dtype=np.float64)
    port().orc_bc_f64(I64(m), _p(rp), _p(col), _p(val), _p(src), I64(len(src)), _p(out))
    return out


def mlp_loss_grad(w, X, Y, M, F, H, V):
    """FP64 loss and gradient of the scheduler MLP (checker of gk_mlp_loss_grad)."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.ascontiguousarray(Y, dtype=np.float32)
    M = np.ascontiguousarray(M, dtype=np.float32)
    grad = np.zeros(w.shape[0], dtype=np.float64)
    loss = ctypes.c_double(0.0)
    port().orc_mlp_loss_grad(ctypes.c_int(F), ctypes.c_int(H), ctypes.c_int(V), _p(w), _p(X), _p(Y), _p(M),
                             ctypes.c_int(X.shape[0]), ctypes.byref(loss), _p(grad))
    return float(loss.value), grad


def transpose(A):
    m, n, rp, col, val = _host(A)
    orp = np.zeros(n + 1, dtype=np.int64)
    ocol = np.zeros(max(len(col), 1), dtype=np.int32)
    oval = np.zeros(max(len(col), 1), dtype=np.int32)
    port().orc_transpose(I64(m), I64(n), _p(rp), _p(col), _p(val), _p(orp), _p(ocol), _p(oval))
    return orp, ocol[: len(col)], oval[: len(col)]


def extract_lower(A):
    m, _, rp, col, _ = _host(A)
    orp = np.zeros(m + 1, dtype=np.int64)
    ocol = np.zeros(max(len(col), 1), dtype=np.int32)
    nnz = ctypes.c_int64(0)
    port().orc_extract_lower(I64(m), _p(rp), _p(col), _p(orp), _p(ocol), ctypes.byref(nnz))
    return orp, ocol[: nnz.value].copy()


# ----- reference (compiled reference headers) -----------------------------------
ACCUM = {"msa": 0, "mca": 1, "naive": 2}


def ref_tc(A_sym, accum="msa", parallel=True):
    m, _, rp, col, _ = _host(A_sym)
    out = ctypes.c_int64(0)
    r = ref().ref_tc_sandia(ACCUM[accum], int(parallel), I64(m), _p(rp), _p(col), ctypes.byref(out))
    if r != 0:
        raise RuntimeError(f"reference tc failed ({r})")
    return int(out.value)


def ref_tc_rows(L, row_begin, row_end, parallel=True):
    m, _, rp, col, _ = _host(L)
    out = ctypes.c_int64(0)
    r = ref().ref_tc_rows(int(parallel), I64(m), _p(rp), _p(col), I64(row_begin), I64(row_end), ctypes.byref(out))
    if r != 0:
        raise RuntimeError(f"reference tc_rows failed ({r})")
    return int(out.value)


def ref_mxmm(A, B, M, accum="msa", parallel=True):
    am, an, arp, acol, aval = _host(A)
    bm, bn, brp, bcol, bval = _host(B)
    mm, mn, mrp, mcol, _ = _host(M)
    out = np.zeros(int(mrp[-1]), dtype=np.int32)
    r = ref().ref_mxmm(ACCUM[accum], int(parallel), I64(am), I64(an), _p(arp), _p(acol), _p(aval), I64(bm),
                       I64(bn), _p(brp), _p(bcol), _p(bval), I64(mm), I64(mn), _p(mrp), _p(mcol), _p(out))
    if r != 0:
        raise RuntimeError(f"reference mxmm failed ({r})")
    return out


def ref_ktruss(A_sym, k, accum="msa", parallel=True):
    m, _, rp, col, _ = _host(A_sym)
    orp = np.zeros(m + 1, dtype=np.int64)
    ocol = np.zeros(max(len(col), 1), dtype=np.int32)
    nnz = ctypes.c_int64(0)
    iters = ctypes.c_int(0)
    r = ref().ref_ktruss(ACCUM[accum], int(parallel), I64(m), _p(rp), _p(col), ctypes.c_int(k), _p(orp), _p(ocol),
                         ctypes.byref(nnz), ctypes.byref(iters))
    if r != 0:
        raise RuntimeError(f"reference ktruss failed ({r})")
    return orp, ocol[: nnz.value].copy(), int(iters.value)


def ref_read_matrix(path, fmt):
    """The reference's reader for `fmt` (mtx, crs, bin, graph, rmat): a CSR
    with the reference's Rst / Col / Val, or None if it cannot read the file."""
    m, n, nz = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
    f = ref().ref_read_matrix
    if f(str(path).encode(), fmt.encode(), ctypes.byref(m), ctypes.byref(n), ctypes.byref(nz), None, None, None) != 0:
        return None
    rp = np.zeros(m.value + 1, dtype=np.int64)
    col = np.zeros(nz.value, dtype=np.int32)
    val = np.zeros(nz.value, dtype=np.int32)
    f(str(path).encode(), fmt.encode(), ctypes.byref(m), ctypes.byref(n), ctypes.byref(nz), _p(rp), _p(col), _p(val))

    class _C:
        pass

    c = _C()
    c.m, c.n, c.nnz, c.rowptr, c.col, c.val = int(m.value), int(n.value), int(nz.value), rp, col, val
    return c


def ref_tc_vertex(A, accum=0, parallel=True):
    """The reference's triangle_counting_vertex (src/main.cpp:16-39), restated
    around its mxmm_msa / mxmm_mca."""
    m, _, rp, col, _ = _host(A)
    out = np.zeros(m, dtype=np.int32)
    r = ref().ref_tc_vertex(ctypes.c_int(accum), ctypes.c_int(1 if parallel else 0), I64(m), _p(rp), _p(col), _p(out))
    if r != 0:
        raise RuntimeError(f"reference tc_vertex failed ({r})")
    return out


def ref_tc_lu(A, accum=0, parallel=True):
    """The reference's triangle_counting_masked_lu (src/main.cpp:42-66)."""
    m, _, rp, col, _ = _host(A)
    out = ctypes.c_int64(0)
    r = ref().ref_tc_lu(ctypes.c_int(accum), ctypes.c_int(1 if parallel else 0), I64(m), _p(rp), _p(col),
                        ctypes.byref(out))
    if r != 0:
        raise RuntimeError(f"reference tc_lu failed ({r})")
    return int(out.value)


def ref_bc_float(A_sym, b, threads=1):
    """Reference BC (float, int32 path counts) with sources 0..b-1.  Runs with
    one OpenMP thread by default: with several threads the reference's row
    split can leave rows unassigned (include/betweenness_centrality.h:326-332)."""
    m, _, rp, col, _ = _host(A_sym)
    out = np.zeros(m, dtype=np.float32)
    old = ref().ref_get_threads()
    ref().ref_set_threads(int(threads))
    try:
        r = ref().ref_bc_batch(1, I64(m), _p(rp), _p(col), I64(b), _p(out))
    finally:
        ref().ref_set_threads(int(old))
    if r != 0:
        raise RuntimeError(f"reference bc failed ({r})")
    return out


def ref_transpose(A):
    m, n, rp, col, val = _host(A)
    orp = np.zeros(n + 1, dtype=np.int64)
    ocol = np.zeros(max(len(col), 1), dtype=np.int32)
    oval = np.zeros(max(len(col), 1), dtype=np.int32)
    ref().ref_transpose(I64(m), I64(n), _p(rp), _p(col), _p(val), _p(orp), _p(ocol), _p(oval))
    return orp, ocol[: len(col)], oval[: len(col)]


def ref_extract_lower(A):
    m, _, rp, col, _ = _host(A)
    orp = np.zeros(m + 1, dtype=np.int64)
    ocol = np.zeros(max(len(col), 1), dtype=np.int32)
    nnz = ctypes.c_int64(0)
    ref().ref_extract_lower(I64(m), _p(rp), _p(col), _p(orp), _p(ocol), ctypes.byref(nnz))
    return orp, ocol[: nnz.value].copy()


def ref_build_symm(L):
    m, _, rp, col, _ = _host(L)
    orp = np.zeros(m + 1, dtype=np.int64)
    ocol = np.zeros(max(2 * len(col), 1), dtype=np.int32)
    nnz = ctypes.c_int64(0)
    ref().ref_build_symm_from_lower(I64(m), _p(rp), _p(col), _p(orp), _p(ocol), ctypes.byref(nnz))
    return orp, ocol[: nnz.value].copy()


def relabel_sources_first(A, sources):
    """Permutation putting `sources` at labels 0..b-1 (rest in order) and the
    relabelled symmetric CSR, so that the reference's BC (sources 0..b-1,
    include/betweenness_centrality.h:445-447) runs on sampled sources."""
    m, _, rp, col, _ = _host(A)
    src = np.asarray(sources, dtype=np.int64)
    perm = np.full(m, -1, dtype=np.int64)  # old -> new
    perm[src] = np.arange(len(src))
    # Non-source vertices follow, isolated ones first: the reference's row
    # split (work_distribution, include/betweenness_centrality.h:326-332)
    # never assigns trailing empty rows to a team, which leaves stale row
    # pointers in its frontier and crashes; no trailing empty row avoids it.
    rest = np.setdiff1d(np.arange(m), src, assume_unique=False)
    deg = np.diff(rp)[rest]
    rest = np.concatenate([rest[deg == 0], rest[deg > 0]])
    perm[rest] = np.arange(len(src), m)
    rows = np.repeat(np.arange(m), np.diff(rp))
    nr, nc = perm[rows], perm[col.astype(np.int64)]
    order = np.lexsort((nc, nr))
    nr, nc = nr[order], nc[order]
    nrp = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(nr, minlength=m), out=nrp[1:])

    class _C:
        pass

    c = _C()
    c.m = c.n = m
    c.rowptr, c.col, c.val = nrp, nc.astype(np.int32), None
    return c, perm


# ----- synthetic inputs (independent of the product library) ---------------------
RMAT_ABC = (0.57, 0.19, 0.19)


class HostCsr:
    """A host CSR (numpy arrays), the fields the oracle functions read."""

    def __init__(self, m, rowptr, col):
        self.m = self.n = m
        self.rowptr = rowptr
        self.col = col
        self.val = None
        self.nnz = int(len(col))


def _take_graph(h, lower):
    lib = port()
    m, nnz = ctypes.c_int64(0), ctypes.c_int64(0)
    lib.orc_graph_info(h, ctypes.byref(m), ctypes.byref(nnz))
    rp = np.zeros(m.value + 1, dtype=np.int64)
    col = np.zeros(max(nnz.value, 1), dtype=np.int32)
    got = lib.orc_graph_copy(h, ctypes.c_int(1 if lower else 0), _p(rp), _p(col))
    lib.orc_graph_free(h)
    return HostCsr(m.value, rp, col[:got].copy())


def _gen_lib():
    lib = port()
    lib.orc_gen_rmat.restype = ctypes.c_void_p
    lib.orc_gen_rmat.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_uint64]
    lib.orc_gen_er.restype = ctypes.c_void_p
    lib.orc_gen_er.argtypes = [I64, I64, ctypes.c_uint64]
    lib.orc_graph_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_graph_copy.restype = I64
    lib.orc_graph_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_graph_free.argtypes = [ctypes.c_void_p]
    return lib


def gen_rmat(scale, edge_factor=16, seed=1, lower=False, abc=RMAT_ABC):
    """Seeded RMAT graph (symmetric, or its strict lower triangle) from the
    oracle's own restatement of the generator."""
    h = _gen_lib().orc_gen_rmat(scale, edge_factor, abc[0], abc[1], abc[2], seed)
    return _take_graph(h, lower)


def gen_er(n, nedges, seed=1, lower=False):
    h = _gen_lib().orc_gen_er(n, nedges, seed)
    return _take_graph(h, lower)
