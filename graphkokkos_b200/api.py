"""Python host API over the C ABI (include/gk_b200.h).

Mirrors the reference's operator surface (src/main.cpp:13-141,
include/matrix_la.h:562-694, include/betweenness_centrality.h:406-506) with
CSR matrices whose arrays are numpy arrays (host) or torch tensors (host or
CUDA).  Every call goes to the CUDA library; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import GkCsr, GkCsrMut, check

_SCHED = {"plain": _lib.GK_SCHED_PLAIN, "learned": _lib.GK_SCHED_LEARNED}
_ACCUM = {"auto": _lib.GK_ACCUM_AUTO, "msa": _lib.GK_ACCUM_MSA, "mca": _lib.GK_ACCUM_MCA, "hash": _lib.GK_ACCUM_HASH}
_SEMIRING = {"plus_times": _lib.GK_PLUS_TIMES, "plus_pair": _lib.GK_PLUS_PAIR}


def _is_torch(x):
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor)


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        if not x.flags.c_contiguous:
            raise ValueError("arrays must be contiguous")
        return x.ctypes.data
    if _is_torch(x):
        if not x.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return x.data_ptr()
    raise TypeError(f"unsupported array type {type(x)}")


def _on_cuda(x):
    return _is_torch(x) and x.is_cuda


def _stream(stream, *arrays):
    """cudaStream_t handle: the given one, else torch's current stream when the
    arrays live on a CUDA device, else the legacy default stream."""
    if stream is not None:
        return ctypes.c_void_p(int(stream))
    if any(_on_cuda(a) for a in arrays if a is not None):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(0)


@dataclass
class Csr:
    """CSR matrix: spMtx<T> (include/matrix.h:33-43) with int64 row pointers."""

    m: int
    n: int
    rowptr: object
    col: object
    val: object = None
    nnz: Optional[int] = None

    def __post_init__(self):
        if self.nnz is None:
            self.nnz = int(self.col.shape[0]) if self.col is not None else 0

    def as_gk(self) -> GkCsr:
        return GkCsr(self.m, self.n, self.nnz, _ptr(self.rowptr), _ptr(self.col), _ptr(self.val))

    @property
    def is_cuda(self):
        return _on_cuda(self.rowptr)

    def to(self, device):
        """Copy to a torch device ("cuda", "cpu") or to numpy (device=None)."""
        import torch

        def conv(a):
            if a is None:
                return None
            if device is None:
                return a.cpu().numpy() if _is_torch(a) else a
            t = torch.as_tensor(a) if not _is_torch(a) else a
            return t.to(device)

        return Csr(self.m, self.n, conv(self.rowptr), conv(self.col), conv(self.val), self.nnz)

    def numpy(self):
        return self.to(None)


def _empty_like_space(ref, shape, dtype):
    """An output array in the same memory space as `ref`."""
    if _on_cuda(ref):
        import torch
        tdt = {np.int64: torch.int64, np.int32: torch.int32, np.uint64: torch.int64, np.float64: torch.float64,
               np.float32: torch.float32}[dtype]
        return torch.empty(shape, dtype=tdt, device=ref.device)
    return np.empty(shape, dtype=dtype)


# ---------------------------------------------------------------------------
# masked SpGEMM family
# ---------------------------------------------------------------------------
def mxmm_masked(A: Csr, B: Csr, M: Csr, semiring="plus_times", sched="plain", accum="auto", out=None,
                stream=None):
    """C<M> = A·B; returns the nnz(M) values of C in M's pattern order
    (mxmm_msa / mxmm_mca, include/matrix_la.h:478-694)."""
    lib = _lib.load()
    if out is None:
        out = _empty_like_space(M.col, (M.nnz,), np.int32)
    a, b, m = A.as_gk(), B.as_gk(), M.as_gk()
    check(lib.gk_mxmm_masked(ctypes.byref(a), ctypes.byref(b), ctypes.byref(m), _ptr(out), _SEMIRING[semiring],
                             _SCHED[sched], _ACCUM[accum], _stream(stream, M.col)))
    return out


def tc_count(L: Csr, sched="plain", stream=None) -> int:
    """Triangle count from the strict lower triangle L (src/main.cpp:69-90)."""
    lib = _lib.load()
    out = ctypes.c_uint64(0)
    g = L.as_gk()
    check(lib.gk_tc_count(ctypes.byref(g), ctypes.addressof(out), _SCHED[sched], _stream(stream, L.col)))
    return int(out.value)


def tc_count_variant(L: Csr, variant: int, stream=None) -> int:
    """Triangle count with every row on one kernel variant (tests, autotuner)."""
    lib = _lib.load()
    out = ctypes.c_uint64(0)
    g = L.as_gk()
    check(lib.gk_tc_count_variant(ctypes.byref(g), int(variant), ctypes.addressof(out), _stream(stream, L.col)))
    return int(out.value)


def mxmm_masked_variant(A: Csr, B: Csr, M: Csr, variant: int, semiring="plus_times", out=None, stream=None):
    lib = _lib.load()
    if out is None:
        out = _empty_like_space(M.col, (M.nnz,), np.int32)
    a, b, m = A.as_gk(), B.as_gk(), M.as_gk()
    check(lib.gk_mxmm_masked_variant(ctypes.byref(a), ctypes.byref(b), ctypes.byref(m), _ptr(out),
                                     _SEMIRING[semiring], int(variant), _stream(stream, M.col)))
    return out


def num_variants() -> int:
    return int(_lib.load().gk_sched_num_variants())


def tc_count_device(L: Csr, out, sched="plain", stream=None):
    """Asynchronous variant: writes the count into a 1-element int64 CUDA tensor."""
    lib = _lib.load()
    g = L.as_gk()
    check(lib.gk_tc_count(ctypes.byref(g), _ptr(out), _SCHED[sched], _stream(stream, L.col)))
    return out


def tc_row_sums(L: Csr, sched="plain", stream=None):
    lib = _lib.load()
    out = _empty_like_space(L.rowptr, (L.m,), np.uint64)
    g = L.as_gk()
    check(lib.gk_tc_row_sums(ctypes.byref(g), _ptr(out), _SCHED[sched], _stream(stream, L.col)))
    return out


def mxmm_cmask(A: Csr, B: Csr, M: Csr, semiring="plus_times", stream=None) -> Csr:
    """C<!M> = A·B (mxmm_msa_cmask, include/matrix_la.h:733-934): C's entries
    are the columns a product reaches that are not in M's row; sorted rows.
    Returned in the memory space of A."""
    lib = _lib.load()
    sr = {"plus_times": 0, "plus_pair": 1}[semiring]
    ga, gb, gm = A.as_gk(), B.as_gk(), M.as_gk()
    st = _stream(stream, A.col)
    rp = _empty_like_space(A.rowptr, (A.m + 1,), np.int64)
    check(lib.gk_mxmm_cmask(ctypes.byref(ga), ctypes.byref(gb), ctypes.byref(gm), sr, _ptr(rp), None, None, st))
    nnz = int(rp[-1])
    col = _empty_like_space(A.col, (max(nnz, 1),), np.int32)
    val = _empty_like_space(A.col, (max(nnz, 1),), np.int32)
    check(lib.gk_mxmm_cmask(ctypes.byref(ga), ctypes.byref(gb), ctypes.byref(gm), sr, _ptr(rp), _ptr(col), _ptr(val),
                            st))
    return Csr(A.m, B.n, rp, col[:nnz], val[:nnz], nnz)


# ---------------------------------------------------------------------------
# operators of the reference's alternate BC formulation
# (include/matrix_la.h:182-328; dense operands are row-major float64)
# ---------------------------------------------------------------------------
def _dense(x):
    """A C-contiguous float64 array (numpy) or tensor (torch, same device)."""
    if _is_torch(x):
        import torch
        return x.to(torch.float64).contiguous()
    return np.ascontiguousarray(x, dtype=np.float64)


def add_nointersect(A: Csr, B: Csr, stream=None) -> Csr:
    """C = A + B for non-intersecting patterns (add_nointersect,
    include/matrix_la.h:287-328): each row the merge of A's and B's rows.
    Returned in the memory space of A; pattern-only operands count as 1."""
    lib = _lib.load()
    nnz = A.nnz + B.nnz
    rp = _empty_like_space(A.rowptr, (A.m + 1,), np.int64)
    col = _empty_like_space(A.rowptr, (max(nnz, 1),), np.int32)
    val = _empty_like_space(A.rowptr, (max(nnz, 1),), np.int32)
    ga, gb = A.as_gk(), B.as_gk()
    check(lib.gk_add_nointersect(ctypes.byref(ga), ctypes.byref(gb), _ptr(rp), _ptr(col), _ptr(val),
                                 _stream(stream, A.col, B.col)))
    return Csr(A.m, A.n, rp, col[:nnz], val[:nnz], nnz)


def dense_ewise_mult_masked(A, B, M: Csr, stream=None):
    """C<M> = A .* B for dense m x n A, B (eWiseMult, include/matrix_la.h:189-208):
    A(i,j)·B(i,j) on M's pattern, 0 elsewhere; returned like A."""
    lib = _lib.load()
    A, B = _dense(A), _dense(B)
    m, n = A.shape
    if tuple(B.shape) != (m, n):
        raise ValueError("A and B must have the same shape")
    C = _empty_like_space(A, (m, n), np.float64)
    gm = M.as_gk()
    check(lib.gk_dense_ewise_mult_masked(m, n, _ptr(A), _ptr(B), ctypes.byref(gm), _ptr(C), _stream(stream, A)))
    return C


def dense_fuse_ewise_mult_add(A, B, C, stream=None):
    """C += A .* B elementwise, in place (fuseEWiseMultAdd,
    include/matrix_la.h:182-187); C must be contiguous float64.  Returns C."""
    lib = _lib.load()
    A, B = _dense(A), _dense(B)
    if (str(C.dtype) not in ("float64", "torch.float64")) or not (C.is_contiguous() if _is_torch(C)
                                                                   else C.flags.c_contiguous):
        raise ValueError("C must be a contiguous float64 array")
    count = int(np.prod(tuple(C.shape)))
    if int(np.prod(tuple(A.shape))) != count or int(np.prod(tuple(B.shape))) != count:
        raise ValueError("A, B and C must have the same number of values")
    check(lib.gk_dense_fuse_ewise_mult_add(count, _ptr(A), _ptr(B), _ptr(C), _stream(stream, C)))
    return C


def mxmm_spd(A: Csr, B, M: Csr, A_val=None, out=None, stream=None):
    """C<M> = A·B with sparse A (m x k), dense B (k x n) and a dense result
    that is 0 outside M (mxmm_spd, include/matrix_la.h:230-258).  A's values:
    A_val (float64, nnz(A)) when given, else A.val, else 1.  `out` may be B
    itself, as in the reference's mxmm_spd(Af, W, S, W, Wbuf)."""
    lib = _lib.load()
    B = _dense(B)
    k, n = B.shape
    if k != A.n:
        raise ValueError("B must have A.n rows")
    if A_val is not None:
        A_val = _dense(A_val)
    C = out if out is not None else _empty_like_space(B, (A.m, n), np.float64)
    ga, gm = A.as_gk(), M.as_gk()
    check(lib.gk_mxmm_spd(ctypes.byref(ga), _ptr(A_val), _ptr(B), n, ctypes.byref(gm), _ptr(C),
                          _stream(stream, B, C)))
    return C


def tc_vertex(A: Csr, sched="plain", stream=None):
    """Triangles through each vertex of a symmetric adjacency
    (triangle_counting_vertex, src/main.cpp:16-39); int32 per vertex."""
    lib = _lib.load()
    out = _empty_like_space(A.rowptr, (A.m,), np.int32)
    g = A.as_gk()
    check(lib.gk_tc_vertex(ctypes.byref(g), _ptr(out), _SCHED[sched], _stream(stream, A.col)))
    return out


def tc_count_lu(A: Csr, sched="plain", stream=None) -> int:
    """Triangle count as sum(C<A> = L·U) / 2 (triangle_counting_masked_lu,
    src/main.cpp:42-66), from the symmetric adjacency A."""
    lib = _lib.load()
    out = ctypes.c_uint64(0)
    g = A.as_gk()
    check(lib.gk_tc_count_lu(ctypes.byref(g), ctypes.addressof(out), _SCHED[sched], _stream(stream, A.col)))
    return int(out.value)


def tc_count_batched(graphs: Sequence[Csr], sched="plain", stream=None):
    lib = _lib.load()
    n = len(graphs)
    arr = (GkCsr * max(n, 1))(*[g.as_gk() for g in graphs])
    out = np.zeros(n, dtype=np.uint64)
    check(lib.gk_tc_count_batched(arr, n, out.ctypes.data, _SCHED[sched],
                                  _stream(stream, *(g.col for g in graphs[:1]))))
    return out


def ktruss(A: Csr, k: int, sched="plain", stream=None):
    """k-truss (src/main.cpp:94-141); returns (truss CSR, iterations)."""
    lib = _lib.load()
    if _is_torch(A.rowptr):
        rp, col = A.rowptr.clone(), A.col.clone()
    else:
        rp, col = np.array(A.rowptr, copy=True), np.array(A.col, copy=True)
    g = GkCsrMut(A.m, A.n, A.nnz, _ptr(rp), _ptr(col))
    iters = ctypes.c_int(0)
    check(lib.gk_ktruss(ctypes.byref(g), int(k), ctypes.byref(iters), _SCHED[sched], _stream(stream, A.col)))
    nnz = int(g.nnz)
    return Csr(A.m, A.n, rp, col[:nnz], None, nnz), int(iters.value)


def bc_batch(A: Csr, sources, sched="plain", stream=None):
    """FP64 batched betweenness centrality over `sources`
    (include/betweenness_centrality.h:406-506)."""
    lib = _lib.load()
    if _on_cuda(A.rowptr):
        import torch
        src = torch.as_tensor(np.asarray(sources, dtype=np.int32)).to(A.rowptr.device)
    else:
        src = np.ascontiguousarray(np.asarray(sources, dtype=np.int32))
    out = _empty_like_space(A.rowptr, (A.m,), np.float64)
    g = A.as_gk()
    check(lib.gk_bc_batch(ctypes.byref(g), _ptr(src), int(len(src)), _ptr(out), _SCHED[sched],
                          _stream(stream, A.col)))
    return out


# ---------------------------------------------------------------------------
# CSR transforms
# ---------------------------------------------------------------------------
def extract_lower(A: Csr, stream=None) -> Csr:
    lib = _lib.load()
    rp = _empty_like_space(A.rowptr, (A.m + 1,), np.int64)
    col = _empty_like_space(A.col, (max(A.nnz, 1),), np.int32)
    nnz = ctypes.c_int64(0)
    g = A.as_gk()
    check(lib.gk_extract_lower(ctypes.byref(g), _ptr(rp), _ptr(col), ctypes.byref(nnz), _stream(stream, A.col)))
    n = int(nnz.value)
    return Csr(A.m, A.n, rp, col[:n], None, n)


def transpose(A: Csr, with_values=False, stream=None) -> Csr:
    lib = _lib.load()
    rp = _empty_like_space(A.rowptr, (A.n + 1,), np.int64)
    col = _empty_like_space(A.col, (max(A.nnz, 1),), np.int32)
    val = _empty_like_space(A.col, (max(A.nnz, 1),), np.int32) if with_values else None
    g = A.as_gk()
    check(lib.gk_transpose(ctypes.byref(g), _ptr(rp), _ptr(col), _ptr(val), _stream(stream, A.col)))
    return Csr(A.n, A.m, rp, col[:A.nnz], None if val is None else val[:A.nnz], A.nnz)


def build_symm_from_lower(L: Csr, with_values=False, stream=None) -> Csr:
    """Symmetric matrix merged from L and transpose(L) on the GPU
    (build_symm_from_lower, include/matrix.h:662-696)."""
    lib = _lib.load()
    nnz = 2 * L.nnz
    rp = _empty_like_space(L.rowptr, (L.m + 1,), np.int64)
    col = _empty_like_space(L.col, (max(nnz, 1),), np.int32)
    val = _empty_like_space(L.col, (max(nnz, 1),), np.int32) if with_values else None
    g = L.as_gk()
    check(lib.gk_build_symm_from_lower(ctypes.byref(g), _ptr(rp), _ptr(col), _ptr(val), _stream(stream, L.col)))
    return Csr(L.m, L.n, rp, col[:nnz], None if val is None else val[:nnz], nnz)


def build_adjacency_matrix(G: Csr, stream=None) -> Csr:
    """G's pattern with every value 1, on the GPU (build_adjacency_matrix,
    include/matrix.h:643-660)."""
    lib = _lib.load()
    rp = _empty_like_space(G.rowptr, (G.m + 1,), np.int64)
    col = _empty_like_space(G.col, (max(G.nnz, 1),), np.int32)
    val = _empty_like_space(G.col, (max(G.nnz, 1),), np.int32)
    g = G.as_gk()
    check(lib.gk_build_adjacency_matrix(ctypes.byref(g), _ptr(rp), _ptr(col), _ptr(val), _stream(stream, G.col)))
    return Csr(G.m, G.n, rp, col[:G.nnz], val[:G.nnz], G.nnz)


# ---------------------------------------------------------------------------
# graph generation
# ---------------------------------------------------------------------------
RMAT_ABC = (0.57, 0.19, 0.19)


def gen_rmat(scale, edge_factor=16, seed=1, abc=RMAT_ABC, device="cpu") -> Csr:
    """Seeded RMAT graph (symmetric, no self-loops/duplicates, sorted rows).
    device="cpu": host builder (numpy arrays); "cuda": device builder (torch)."""
    lib = _lib.load()
    m = 1 << scale
    a, b, c = abc
    if device == "cpu":
        h = ctypes.c_void_p()
        check(lib.gk_gen_rmat_host(scale, edge_factor, a, b, c, seed, ctypes.byref(h)))
        return _take_host_graph(lib, h)
    import torch
    nnz = ctypes.c_int64(0)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib.gk_gen_rmat(scale, edge_factor, a, b, c, seed, ctypes.byref(nnz), None, None, s))
    rp = torch.empty(m + 1, dtype=torch.int64, device=device)
    col = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=device)
    check(lib.gk_gen_rmat(scale, edge_factor, a, b, c, seed, ctypes.byref(nnz), _ptr(rp), _ptr(col), s))
    return Csr(m, m, rp, col[:nnz.value], None, int(nnz.value))


def uneven_batch_specs(ngraphs, seed0):
    """Parameters of an uneven many-graph batch: the first half Erdos-Renyi
    G(n, M) with n log-uniform in [1e3, 1e5] and average degree uniform in
    [4, 64] (M = n*d/2 sampled pairs), the second half RMAT with scale uniform
    in [10, 17] and edge factor 16.  Graph g has seed seed0 + g, which also
    draws its parameters.  Returns (kind, a, b, seed) tuples: ("er", n, M, seed)
    or ("rmat", scale, edge_factor, seed)."""
    specs = []
    for g in range(ngraphs):
        seed = seed0 + g
        rng = np.random.default_rng(seed)
        if g < ngraphs // 2:
            n = int(round(10 ** rng.uniform(3.0, 5.0)))
            d = float(rng.uniform(4.0, 64.0))
            specs.append(("er", n, max(1, int(n * d / 2)), seed))
        else:
            specs.append(("rmat", int(rng.integers(10, 18)), 16, seed))
    return specs


def gen_spec(spec, device="cuda") -> Csr:
    kind, a, b, seed = spec
    return gen_rmat(a, b, seed=seed, device=device) if kind == "rmat" else gen_er(a, b, seed=seed, device=device)


def disjoint_union(graphs: Sequence[Csr]) -> Csr:
    """Block-diagonal CSR of several square graphs (device tensors)."""
    import torch
    rps, cols = [], []
    vbase, ebase = 0, 0
    for G in graphs:
        rps.append(G.rowptr[:-1] + ebase)
        cols.append(G.col[:G.nnz] + vbase)
        vbase += G.m
        ebase += G.nnz
    dev = graphs[0].rowptr.device
    rps.append(torch.tensor([ebase], dtype=torch.int64, device=dev))
    return Csr(vbase, vbase, torch.cat(rps), torch.cat(cols), None, ebase)


def gen_er(n, nedges, seed=1, device="cpu") -> Csr:
    lib = _lib.load()
    if device == "cpu":
        h = ctypes.c_void_p()
        check(lib.gk_gen_er_host(n, nedges, seed, ctypes.byref(h)))
        return _take_host_graph(lib, h)
    import torch
    nnz = ctypes.c_int64(0)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib.gk_gen_er(n, nedges, seed, ctypes.byref(nnz), None, None, s))
    rp = torch.empty(n + 1, dtype=torch.int64, device=device)
    col = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=device)
    check(lib.gk_gen_er(n, nedges, seed, ctypes.byref(nnz), _ptr(rp), _ptr(col), s))
    return Csr(n, n, rp, col[:nnz.value], None, int(nnz.value))


def _take_host_graph(lib, h) -> Csr:
    m = ctypes.c_int64(0)
    nnz = ctypes.c_int64(0)
    lib.gk_host_graph_info(h, ctypes.byref(m), ctypes.byref(nnz))
    rp = np.empty(m.value + 1, dtype=np.int64)
    col = np.empty(nnz.value, dtype=np.int32)
    lib.gk_host_graph_copy(h, rp.ctypes.data, col.ctypes.data if nnz.value else None)
    lib.gk_host_graph_free(h)
    return Csr(int(m.value), int(m.value), rp, col, None, int(nnz.value))


FILE_FORMATS = {"auto": 0, "mtx": 1, "bin": 2, "crs": 3, "graph": 4, "rmat": 5}


def read_matrix(path, fmt="auto", sort=False) -> Csr:
    """Reads a matrix file in one of the reference's formats (mtx, bin, crs,
    graph, rmat; include/matrix.h:44-60) into a host CSR.  Rows keep the
    file's order, as the reference builds them; sort=True sorts every row's
    columns, which the products and algorithms here require.  The values are
    None for pattern files."""
    lib = _lib.load()
    h = ctypes.c_void_p()
    check(lib.gk_read_matrix(str(path).encode(), FILE_FORMATS[fmt], ctypes.byref(h)))
    if sort:
        check(lib.gk_host_graph_sort_rows(h))
    m = ctypes.c_int64(0)
    nnz = ctypes.c_int64(0)
    n = ctypes.c_int64(0)
    lib.gk_host_graph_info(h, ctypes.byref(m), ctypes.byref(nnz))
    rp = np.empty(m.value + 1, dtype=np.int64)
    col = np.empty(nnz.value, dtype=np.int32)
    val = np.empty(nnz.value, dtype=np.int32)
    lib.gk_host_graph_copy(h, rp.ctypes.data, col.ctypes.data if nnz.value else None)
    has = lib.gk_host_graph_values(h, val.ctypes.data if nnz.value else None, ctypes.byref(n))
    lib.gk_host_graph_free(h)
    return Csr(int(m.value), int(n.value), rp, col, val if has == 1 else None, int(nnz.value))


def write_matrix(path, A: Csr, fmt="auto"):
    """Writes a host CSR as MatrixMarket (mtx) or binary CSR (bin)."""
    lib = _lib.load()
    H = A.to(None) if _is_torch(A.rowptr) else A
    rp = np.ascontiguousarray(np.asarray(H.rowptr, dtype=np.int64))
    col = np.ascontiguousarray(np.asarray(H.col, dtype=np.int32))
    val = None if H.val is None else np.ascontiguousarray(np.asarray(H.val, dtype=np.int32))
    g = GkCsr(H.m, H.n, H.nnz, _ptr(rp), _ptr(col), _ptr(val))
    check(lib.gk_write_matrix(str(path).encode(), FILE_FORMATS[fmt], ctypes.byref(g)))


def lower_host(A: Csr) -> Csr:
    """Strict lower triangle of a host CSR with numpy (input preparation)."""
    rp = np.asarray(A.rowptr)
    col = np.asarray(A.col)
    rows = np.repeat(np.arange(A.m, dtype=np.int64), np.diff(rp))
    keep = col < rows
    cnt = np.bincount(rows[keep], minlength=A.m)
    lrp = np.zeros(A.m + 1, dtype=np.int64)
    np.cumsum(cnt, out=lrp[1:])
    lcol = np.ascontiguousarray(col[keep])
    return Csr(A.m, A.n, lrp, lcol, None, int(lcol.shape[0]))
