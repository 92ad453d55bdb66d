"""ctypes binding of libgk_b200.so (the C ABI declared in include/gk_b200.h).

The shared library is built in-tree (graphkokkos_b200/lib/libgk_b200.so) by
``graphkokkos_b200.build`` / ``__graft_entry__.build()``.  Loading fails
loudly when it is missing: there is no CPU fallback for any operation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgk_b200.so")

c_i64p = ctypes.POINTER(ctypes.c_int64)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_dblp = ctypes.POINTER(ctypes.c_double)
c_fltp = ctypes.POINTER(ctypes.c_float)
VP = ctypes.c_void_p


class GkCsr(ctypes.Structure):
    """struct gk_csr (include/gk_b200.h)."""

    _fields_ = [
        ("m", ctypes.c_int64),
        ("n", ctypes.c_int64),
        ("nnz", ctypes.c_int64),
        ("rowptr", VP),
        ("col", VP),
        ("val", VP),
    ]


class GkCsrMut(ctypes.Structure):
    """struct gk_csr_mut (include/gk_b200.h)."""

    _fields_ = [
        ("m", ctypes.c_int64),
        ("n", ctypes.c_int64),
        ("nnz", ctypes.c_int64),
        ("rowptr", VP),
        ("col", VP),
    ]


class GkProfRec(ctypes.Structure):
    """struct gk_prof_rec (include/gk_b200.h)."""

    _fields_ = [
        ("variant", ctypes.c_int),
        ("ms", ctypes.c_float),
        ("rows", ctypes.c_int64),
        ("sum_a", ctypes.c_int64),
        ("sum_m", ctypes.c_int64),
        ("sum_work", ctypes.c_int64),
    ]


GK_OK = 0
GK_ERR_ARG = 1
GK_ERR_OOM = 2
GK_ERR_CUDA = 3
GK_ERR_TIMEOUT = 4
GK_ERR_INVALID_CSR = 5
GK_ERR_UNSUPPORTED = 6

GK_PLUS_TIMES = 0
GK_PLUS_PAIR = 1
GK_SCHED_PLAIN = 0
GK_SCHED_LEARNED = 1
GK_ACCUM_AUTO = 0
GK_ACCUM_MSA = 1
GK_ACCUM_MCA = 2
GK_ACCUM_HASH = 3

# name -> (restype, argtypes); every symbol of include/gk_b200.h
SIGNATURES = {
    "gk_mxmm_masked": (ctypes.c_int, [ctypes.POINTER(GkCsr)] * 3 + [VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, VP]),
    "gk_tc_count": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, ctypes.c_int, VP]),
    "gk_tc_count_noalloc": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, ctypes.c_int, VP]),
    "gk_tc_count_variant":(ctypes.c_int, [ctypes.POINTER(GkCsr), ctypes.c_int, VP, VP]),
    "gk_mxmm_masked_variant": (ctypes.c_int, [ctypes.POINTER(GkCsr)] * 3 + [VP, ctypes.c_int, ctypes.c_int, VP]),
    "gk_tc_row_sums": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, ctypes.c_int, VP]),
    "gk_tc_vertex": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, ctypes.c_int, VP]),
    "gk_mxmm_cmask": (ctypes.c_int, [ctypes.POINTER(GkCsr)] * 3 + [ctypes.c_int, VP, VP, VP, VP]),
    "gk_tc_count_lu": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, ctypes.c_int, VP]),
    "gk_add_nointersect": (ctypes.c_int, [ctypes.POINTER(GkCsr)] * 2 + [VP, VP, VP, VP]),
    "gk_dense_ewise_mult_masked": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, VP, VP, ctypes.POINTER(GkCsr), VP,
                                                  VP]),
    "gk_dense_fuse_ewise_mult_add": (ctypes.c_int, [ctypes.c_int64, VP, VP, VP, VP]),
    "gk_mxmm_spd": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, VP, ctypes.c_int64, ctypes.POINTER(GkCsr), VP, VP]),
    "gk_tc_count_batched": (ctypes.c_int, [ctypes.POINTER(GkCsr), ctypes.c_int, VP, ctypes.c_int, VP]),
    "gk_ktruss": (ctypes.c_int, [ctypes.POINTER(GkCsrMut), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int, VP]),
    "gk_bc_batch": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, ctypes.c_int, VP, ctypes.c_int, VP]),
    "gk_extract_lower": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, VP, c_i64p, VP]),
    "gk_transpose": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, VP, VP, VP]),
    "gk_build_symm_from_lower": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, VP, VP, VP]),
    "gk_build_adjacency_matrix": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, VP, VP, VP]),
    "gk_gen_rmat": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_uint64, c_i64p, VP, VP, VP]),
    "gk_gen_er": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_uint64, c_i64p, VP, VP, VP]),
    "gk_gen_rmat_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_uint64, ctypes.POINTER(VP)]),
    "gk_gen_er_host": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_uint64, ctypes.POINTER(VP)]),
    "gk_host_graph_info": (ctypes.c_int, [VP, c_i64p, c_i64p]),
    "gk_host_graph_copy": (ctypes.c_int, [VP, VP, VP]),
    "gk_host_graph_free": (None, [VP]),
    "gk_read_matrix": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(VP)]),
    "gk_write_matrix": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(GkCsr)]),
    "gk_host_graph_values": (ctypes.c_int, [VP, VP, c_i64p]),
    "gk_host_graph_sort_rows": (ctypes.c_int, [VP]),
    "gk_sched_num_variants": (ctypes.c_int, []),
    "gk_sched_num_features": (ctypes.c_int, []),
    "gk_sched_model_size": (ctypes.c_size_t, []),
    "gk_sched_set_model": (ctypes.c_int, [VP, ctypes.c_size_t]),
    "gk_sched_load_model_file": (ctypes.c_int, [ctypes.c_char_p]),
    "gk_sched_has_model": (ctypes.c_int, []),
    "gk_sched_num_bins": (ctypes.c_int, []),
    "gk_sched_variant_allowed": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "gk_sched_bins": (ctypes.c_int, [ctypes.POINTER(GkCsr), ctypes.c_int, VP, VP, VP, VP, VP]),
    "gk_tune_run": (ctypes.c_int, [ctypes.POINTER(GkCsr), ctypes.c_int, VP, VP, VP, VP]),
    "gk_mlp_loss_grad": (ctypes.c_int, [VP, VP, VP, VP, ctypes.c_int, VP, VP, VP]),
    "gk_mlp_train": (ctypes.c_int, [VP, VP, VP, VP, ctypes.c_int, ctypes.c_int, ctypes.c_float, VP, VP]),
    "gk_mlp_forward": (ctypes.c_int, [VP, VP, ctypes.c_int, VP, VP]),
    "gk_bc_set_model": (ctypes.c_int, [VP, ctypes.c_size_t]),
    "gk_bc_load_model_file": (ctypes.c_int, [ctypes.c_char_p]),
    "gk_bc_has_model": (ctypes.c_int, []),
    "gk_bc_tune": (ctypes.c_int, [ctypes.POINTER(GkCsr), VP, ctypes.c_int, ctypes.c_int, VP, VP, VP, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_int), VP]),
    "gk_prof_enable": (ctypes.c_int, [ctypes.c_int]),
    "gk_prof_count": (ctypes.c_int, []),
    "gk_prof_flush": (ctypes.c_int, []),
    "gk_prof_get": (ctypes.c_int, [ctypes.c_int, VP]),
    "gk_launch_count": (ctypes.c_int64, []),
    "gk_last_error_string": (ctypes.c_char_p, []),
    "gk_version": (ctypes.c_int, []),
    "gk_inject_alloc_failure": (ctypes.c_int, [ctypes.c_int64]),
}

_lib = None


def load(required_symbols=None):
    """Loads libgk_b200.so and binds every declared symbol.

    Raises RuntimeError when the library has not been built: the package has
    no CPU fallback.
    """
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libgk_b200.so not found at {LIB_PATH}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        if required_symbols is not None and name not in required_symbols:
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class GkError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gk status {code}: {msg}")
        self.code = code


def check(status):
    if status != GK_OK:
        raise GkError(status, load().gk_last_error_string().decode(errors="replace"))
    return status
