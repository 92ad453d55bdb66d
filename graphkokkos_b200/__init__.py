"""GraphKokkos-B200: masked SpGEMM C<M> = A·B and triangle counting, k-truss
and batched betweenness centrality on one B200, behind the reference's
operator surface.  See include/gk_b200.h for the C ABI."""
from .api import (Csr, add_nointersect, bc_batch, build_adjacency_matrix, build_symm_from_lower,
                  dense_ewise_mult_masked, dense_fuse_ewise_mult_add, extract_lower, gen_er, gen_rmat, ktruss,
                  lower_host, mxmm_cmask, mxmm_masked, mxmm_masked_variant, mxmm_spd, num_variants, read_matrix,
                  tc_count, tc_count_batched, tc_count_device, tc_count_lu, tc_count_variant, tc_row_sums, tc_vertex,
                  transpose, write_matrix)
from ._lib import GkError, LIB_PATH, load

__all__ = [
    "Csr", "GkError", "LIB_PATH", "add_nointersect", "bc_batch", "build_adjacency_matrix", "build_symm_from_lower",
    "dense_ewise_mult_masked", "dense_fuse_ewise_mult_add", "extract_lower", "gen_er", "gen_rmat", "ktruss", "load",
    "lower_host", "mxmm_cmask", "mxmm_masked", "mxmm_masked_variant", "mxmm_spd", "num_variants", "read_matrix",
    "tc_count", "tc_count_batched", "tc_count_device", "tc_count_lu", "tc_count_variant", "tc_row_sums", "tc_vertex",
    "transpose", "write_matrix",
]
