/*
 * gk_b200.h — C ABI of the B200-native masked SpGEMM library.
 *
 * Drop-in boundary for GraphKokkos' hot path: the masked sparse
 * matrix-matrix multiply C<M> = A·B and the algorithms built on it
 * (triangle counting, k-truss, batched betweenness centrality).  The
 * reference exposes these as C++ templates over host-resident Kokkos Views;
 * this header exposes the same operations with plain pointers and sizes so
 * that any host language can bind them.
 *
 * Conventions
 *  - Matrices are CSR: int64 row pointers (m+1), int32 column indices sorted
 *    ascending within each row, optional int32 values (NULL: every stored
 *    value is 1, the adjacency convention of the reference's
 *    build_adjacency_matrix, include/matrix.h:643-660).
 *  - Every array pointer may be host memory or device memory of the current
 *    CUDA device.  Host inputs are copied to HBM inside the call; host outputs
 *    are copied back and the call returns after they are written.  With device
 *    outputs the call is asynchronous on `stream` (a cudaStream_t; NULL = the
 *    legacy default stream).
 *  - Every entry point returns a gk_status; on failure gk_last_error_string()
 *    describes the error for the calling host thread.  Calls on different
 *    streams may run concurrently.
 *  - Every matrix argument is checked on the device before any kernel indexes
 *    through it: row pointers from 0 to nnz and non-decreasing, columns in
 *    [0, n), and (except A of the masked products, A and B of the
 *    complement-masked product, and the inputs of gk_transpose and
 *    gk_bc_batch, whose order does not matter) columns strictly increasing
 *    within each row.  A violation returns GK_ERR_INVALID_CSR naming the
 *    matrix, the defect and the first bad row.  The check reads the result on
 *    the host (one synchronisation of `stream`); it is skipped inside a
 *    stream capture and when the environment sets GK_CHECK_CSR=0, in which
 *    case the caller guarantees well-formed input.
 *  - Results are bit-exact with the reference on the same inputs: integer
 *    outputs exactly, FP64 betweenness scores to round-off (the scheduler
 *    changes only the order of FP64 sums).
 */
#ifndef GK_B200_H
#define GK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference reports errors by throwing (include/matrix.h:45-60,
 * include/matrix_la.h:291-292); the ABI returns codes instead. */
typedef enum gk_status {
    GK_OK = 0,
    GK_ERR_ARG = 1,         /* bad argument (null pointer, shape mismatch, k < 3, ...) */
    GK_ERR_OOM = 2,         /* device memory exhausted */
    GK_ERR_CUDA = 3,        /* CUDA runtime error */
    GK_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    GK_ERR_INVALID_CSR = 5, /* rowptr not monotone, column out of range or unsorted */
    GK_ERR_UNSUPPORTED = 6  /* request outside what the library implements */
} gk_status;

/* Read-only CSR matrix (spMtx<T>, include/matrix.h:33-43: m, n, nz, Rst, Col, Val). */
typedef struct gk_csr {
    int64_t m, n, nnz;
    const int64_t *rowptr; /* m+1 entries */
    const int32_t *col;    /* nnz entries, sorted within each row */
    const int32_t *val;    /* nnz entries, or NULL for "all ones" */
} gk_csr;

/* Mutable pattern-only CSR, used in place by gk_ktruss. */
typedef struct gk_csr_mut {
    int64_t m, n, nnz;
    int64_t *rowptr; /* m+1 entries */
    int32_t *col;    /* capacity >= nnz on entry */
} gk_csr_mut;

/* Semiring of the product.  PLUS_TIMES is the reference's arithmetic
 * (accum(j) += a·b, include/matrix_la.h:624); PLUS_PAIR treats every stored
 * value as 1 (what triangle counting and k-truss compute on adjacency
 * matrices, whose values are all 1). */
typedef enum gk_semiring { GK_PLUS_TIMES = 0, GK_PLUS_PAIR = 1 } gk_semiring;

/* Row-bin scheduler.  PLAIN: the hand-written binning heuristic.  LEARNED:
 * the MLP loaded with gk_sched_set_model (GK_ERR_ARG if none is loaded).
 * The scheduler changes only which kernel variant processes a row, never the
 * arithmetic. */
typedef enum gk_sched { GK_SCHED_PLAIN = 0, GK_SCHED_LEARNED = 1 } gk_sched;

/* Accumulator families a caller may force (GK_ACCUM_AUTO lets the scheduler
 * choose).  MSA and MCA name the reference's two live accumulators
 * (include/matrix_la.h:562-694 and :478-528). */
typedef enum gk_accum {
    GK_ACCUM_AUTO = 0,
    GK_ACCUM_MSA = 1,  /* dense column-window accumulator in shared memory */
    GK_ACCUM_MCA = 2,  /* mask-compressed: slots = mask positions, binary search */
    GK_ACCUM_HASH = 3  /* hash of mask columns in shared memory */
} gk_accum;

/* C<M> = A·B.  Replaces the reference operator type
 *   mxmOp<T> = void(*)(bool, const spMtx<T>& A, const spMtx<T>& B,
 *                      const spMtx<T>& M, spMtx<T>& C)      (src/main.cpp:13-14)
 * implemented by mxmm_msa (include/matrix_la.h:562-635), mxmm_mca (:478-528)
 * and mxmm_naive (:936-1068).  C has exactly M's pattern, explicit zeros kept
 * (include/matrix_la.h:564-568): the ABI writes the nnz(M) values only,
 * parallel to M's col array, into C_val.  Requires A.m == M.m, A.n == B.m,
 * B.n == M.n.  `accum` forces an accumulator family (GK_ACCUM_AUTO: the
 * scheduler picks per row bin). */
int gk_mxmm_masked(const gk_csr *A, const gk_csr *B, const gk_csr *M, int32_t *C_val,
                   int semiring, int sched, int accum, void *stream);

/* Triangle count of the graph whose strict lower triangle is L:
 * sum of C<L> = L·L (plus-pair), as triangle_counting_masked_sandia
 * (src/main.cpp:69-90, after its untimed extract_lower_triangle at :71).
 * *count receives the uint64 total (the reference returns int64). */
int gk_tc_count(const gk_csr *L, uint64_t *count, int sched, void *stream);

/* Same count as gk_tc_count, for callers that cannot have the library allocate
 * GPU memory during the call (a process whose framework already reserved the
 * device's memory, or a host that forbids allocations in its processing loop).
 * No counterpart in the reference.  All scratch comes from one fixed 36 MiB
 * device array that this library holds on every GPU it is loaded on; L may
 * have at most 1,048,576 rows (GK_ERR_ARG beyond) and must be in device memory;
 * *count may be host or device memory.  The first call on a device looks up the
 * array's address, so make it before any stream capture.  Calls share the
 * array: calls that overlap on the GPU race. */
int gk_tc_count_noalloc(const gk_csr *L, uint64_t *count, int sched, void *stream);

/* Per-vertex sums of C<L> = L·L: row_sums[i] = sum_j C(i,j), the number of
 * triangles whose largest vertex is i (a fused-epilogue variant of
 * triangle_counting_vertex, src/main.cpp:16-39). */
int gk_tc_row_sums(const gk_csr *L, uint64_t *row_sums, int sched, void *stream);

/* Complement-masked product C<!M> = A·B (mxmm_msa_cmask,
 * include/matrix_la.h:733-934): row i of C holds every column reached by a
 * product A(i,k)·B(k,j) that is not a column of M's row i, in ascending
 * order (kept even where the sum is zero), with the sum of the products
 * (PLUS_TIMES; PLUS_PAIR counts them).  Unlike gk_mxmm_masked, C's pattern
 * is not known in advance, so two calls, as the reference's symbolic and
 * numeric passes: with C_col == NULL, C_rowptr (A.m + 1 entries) receives the
 * row pointers; then, with C_rowptr from that call and C_col / C_val of
 * C_rowptr[A.m] entries (C_val may be NULL), the columns and values. */
int gk_mxmm_cmask(const gk_csr *A, const gk_csr *B, const gk_csr *M, int semiring, int64_t *C_rowptr,
                  int32_t *C_col, int32_t *C_val, void *stream);

/* The operators of the reference's alternate (commented-out) BC formulation,
 * include/betweenness_centrality.h:5-123.  Dense matrices are row-major FP64
 * arrays (denseMtx, include/matrix.h:548-630: Val(i*n + j)); FP64 results
 * are bit-exact with the reference, whose `x += a * b` is one fused
 * multiply-add in its x86-64-v3 build. */

/* C = A + B for matrices whose patterns do not intersect (add_nointersect,
 * include/matrix_la.h:287-328): row i of C is the merge of A's and B's rows
 * (on an equal column, which the operator does not expect, B's entry comes
 * first).  C_rowptr (m+1) = A.rowptr + B.rowptr; C_col and C_val (may be
 * NULL) hold nnz(A) + nnz(B) entries; pattern-only operands count as 1.  The
 * reference's copy of a row's remaining B entries reads them at A's cursor
 * (:320-322); C here is the true merge. */
int gk_add_nointersect(const gk_csr *A, const gk_csr *B, int64_t *C_rowptr, int32_t *C_col, int32_t *C_val,
                       void *stream);

/* C<M> = A .* B on dense m x n operands (eWiseMult, include/matrix_la.h:189-208):
 * C(i,j) = A(i,j) * B(i,j) where M has an entry, 0 elsewhere. */
int gk_dense_ewise_mult_masked(int64_t m, int64_t n, const double *A, const double *B, const gk_csr *M, double *C,
                               void *stream);

/* C += A .* B over `count` values (fuseEWiseMultAdd, include/matrix_la.h:182-187). */
int gk_dense_fuse_ewise_mult_add(int64_t count, const double *A, const double *B, double *C, void *stream);

/* C<M> = A * B with sparse A (m x k), dense B (k x n) and dense C (m x n) that
 * is 0 outside M's pattern (mxmm_spd, include/matrix_la.h:230-258).  A's
 * values come from A_val (nnz(A) doubles) when given, else from A->val, else
 * 1.  C may be B itself (the reference calls mxmm_spd(Af, W, S, W, Wbuf)). */
int gk_mxmm_spd(const gk_csr *A, const double *A_val, const double *B, int64_t n, const gk_csr *M, double *C,
                void *stream);

/* Triangles through each vertex of a symmetric adjacency A:
 * counts[i] = (sum_j C(i,j)) >> 1 with C<A> = A·A, as int like the reference's
 * triangle_counting_vertex (src/main.cpp:16-39).  counts has A.m entries. */
int gk_tc_vertex(const gk_csr *A, int32_t *counts, int sched, void *stream);

/* Triangle count through the L·U formulation: L = tril(A), U = L^T,
 * *count = sum(C<A> = L·U) >> 1 (triangle_counting_masked_lu,
 * src/main.cpp:42-66).  A: symmetric adjacency, sorted rows. */
int gk_tc_count_lu(const gk_csr *A, uint64_t *count, int sched, void *stream);

/* Triangle counts of many independent graphs in one persistent launch:
 * counts[g] = gk_tc_count(&graphs[g]).  No reference counterpart (the
 * reference runs one graph per process, src/main.cpp:323-345). */
int gk_tc_count_batched(const gk_csr *graphs, int ngraphs, uint64_t *counts, int sched, void *stream);

/* k-truss of a symmetric adjacency matrix, in place: repeat S<C> = C·C,
 * keep the entries with S >= k-2, until nnz stops changing (k_truss,
 * src/main.cpp:94-141, with its View-size defect at :99/:118 not
 * reproduced).  On return inout->rowptr/col/nnz hold the truss and *iters the
 * number of passes (the reference's "Iterations:" line, :138).  k >= 3. */
int gk_ktruss(gk_csr_mut *inout, int k, int *iters, int sched, void *stream);

/* Batched betweenness centrality in FP64 over the given sources:
 * bc[v] = sum over sources s of Brandes' dependency delta_s(v), unnormalised,
 * as betweenness_centrality_batch (include/betweenness_centrality.h:406-506)
 * computes for sources 0..b-1 (:445-447).  A must be square.  bc has A.m
 * entries.  Sources must be distinct vertices.  sched picks each forward
 * level's kernel shape (pull or push): GK_SCHED_PLAIN by the direction-
 * optimising rule, GK_SCHED_LEARNED by the model of gk_bc_set_model. */
int gk_bc_batch(const gk_csr *A, const int32_t *sources, int nsources, double *bc, int sched,
                void *stream);

/* Same operations with every row forced onto one kernel variant
 * (0 <= variant < gk_sched_num_variants()): used to check each variant on its
 * own and by the autotuner.  No reference counterpart. */
int gk_tc_count_variant(const gk_csr *L, int variant, uint64_t *count, void *stream);
int gk_mxmm_masked_variant(const gk_csr *A, const gk_csr *B, const gk_csr *M, int32_t *C_val, int semiring,
                           int variant, void *stream);

/* ----- CSR transforms (device or host arrays; outputs sized by the caller) ----- */

/* Strict lower triangle (extract_lower_triangle, include/matrix.h:698-726).
 * out_rowptr: m+1; out_col capacity >= nnz(A) (the result has *out_nnz). */
int gk_extract_lower(const gk_csr *A, int64_t *out_rowptr, int32_t *out_col, int64_t *out_nnz,
                     void *stream);

/* CSR transpose (transpose, include/matrix_la.h:155-179).  out_rowptr: n+1,
 * out_col/out_val: nnz (out_val may be NULL). */
int gk_transpose(const gk_csr *A, int64_t *out_rowptr, int32_t *out_col, int32_t *out_val,
                 void *stream);

/* Symmetric matrix from its strict lower triangle (build_symm_from_lower,
 * include/matrix.h:662-696): row i of the result merges row i of L with row i
 * of transpose(L), the transpose's entry first on equal columns, values
 * carried (out_val may be NULL; L's NULL values count as 1).  L must be square
 * with sorted rows.  out_rowptr: m+1, out_col / out_val: 2*nnz(L). */
int gk_build_symm_from_lower(const gk_csr *L, int64_t *out_rowptr, int32_t *out_col, int32_t *out_val,
                             void *stream);

/* G's pattern with every value 1 (build_adjacency_matrix,
 * include/matrix.h:643-660).  out_rowptr: m+1, out_col / out_val: nnz. */
int gk_build_adjacency_matrix(const gk_csr *G, int64_t *out_rowptr, int32_t *out_col, int32_t *out_val,
                              void *stream);

/* ----- graph generation (device-side builder; host twin: gk_gen_*_host) ------- */

/* Seeded RMAT graph (2^scale vertices, edge_factor << scale edges) or
 * Erdos-Renyi G(n, nedges), symmetrised, self-loops and duplicates removed,
 * rows sorted.  Two calls: first with rowptr == NULL to learn *nnz (m is known
 * to the caller), then with device or host arrays of m+1 and nnz entries. */
int gk_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                int64_t *nnz, int64_t *rowptr, int32_t *col, void *stream);
int gk_gen_er(int64_t n, int64_t nedges, uint64_t seed, int64_t *nnz, int64_t *rowptr, int32_t *col,
              void *stream);

/* Host builders producing the identical CSR (C++/OpenMP). */
typedef struct gk_host_graph gk_host_graph;
int gk_gen_rmat_host(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                     gk_host_graph **out);
int gk_gen_er_host(int64_t n, int64_t nedges, uint64_t seed, gk_host_graph **out);
int gk_host_graph_info(const gk_host_graph *g, int64_t *m, int64_t *nnz);
int gk_host_graph_copy(const gk_host_graph *g, int64_t *rowptr, int32_t *col);
void gk_host_graph_free(gk_host_graph *g);

/* ----- sparse-matrix files (host memory) ------------------------------------ */

/* The reference's file formats (spMtx(const char *filename, format),
 * include/matrix.h:44-60): GK_FILE_AUTO picks by the file's extension. */
typedef enum gk_file_format {
    GK_FILE_AUTO = 0,
    GK_FILE_MTX = 1,    /* MatrixMarket coordinate (read_mtx_to_crs, matrix.h:259-395) */
    GK_FILE_BIN = 2,    /* binary CSR (read_bin_to_crs, matrix.h:418-456) */
    GK_FILE_CRS = 3,    /* text CSR (read_crs_to_crs, matrix.h:397-416) */
    GK_FILE_GRAPH = 4,  /* adjacency lines (read_graph_to_crs, matrix.h:458-486) */
    GK_FILE_RMAT = 5    /* edge pairs, symmetrised (read_rmat_to_crs, matrix.h:488-533) */
} gk_file_format;

/* Reads a matrix into a host graph handle (rows in the file's order, as the
 * reference builds them; see gk_host_graph_sort_rows).  Errors: GK_ERR_ARG
 * with gk_last_error_string(). */
int gk_read_matrix(const char *path, int format, gk_host_graph **out);
/* Writes A (host arrays) as mtx or bin; the bin layout is the reader's (the
 * reference's write_crs_to_bin, matrix.h:210-227, stores Rst in place of Col
 * and Val). */
int gk_write_matrix(const char *path, int format, const gk_csr *A);
/* Values of a handle: 1 and val[nnz] filled when the file carried values, 0
 * for a pattern (values 1); *n receives the column count. */
int gk_host_graph_values(const gk_host_graph *g, int32_t *val, int64_t *n);
/* Sorts the columns of every row (values alongside, stable). */
int gk_host_graph_sort_rows(gk_host_graph *g);

/* ----- scheduler ------------------------------------------------------------ */

/* Number of kernel variants the scheduler chooses among, and of the per-bin
 * features the learned model reads. */
int gk_sched_num_variants(void);
int gk_sched_num_features(void);

/* Loads the learned scheduler's MLP (float32 weights, layout documented in
 * graphkokkos_b200/sched.py); n_floats must match gk_sched_model_size(). */
size_t gk_sched_model_size(void);
int gk_sched_set_model(const float *weights, size_t n_floats);
int gk_sched_has_model(void);

/* Loads the learned scheduler's MLP from a model file, so that a C or C++ host
 * can use GK_SCHED_LEARNED without parsing anything itself.  File layout: the
 * 8 bytes "GKMLP001", a little-endian uint32 weight count (gk_sched_model_size()),
 * then the float32 weights little-endian.  The trained models ship as
 * graphkokkos_b200/sched/model.bin (row bins) and bc_model.bin (BC levels).
 * GK_ERR_ARG names what is wrong with a file that does not match.  No
 * counterpart in the reference, whose only schedule choice is the CLI's
 * accumulator name (src/main.cpp:194-212). */
int gk_sched_load_model_file(const char *path);

/* ----- autotuning and training of the learned scheduler (no reference
 * counterpart: the reference's only scheduling is the CLI's per-call accumulator
 * choice, src/main.cpp:194-212) ------------------------------------------------ */

/* Per-bin statistics of the rows of a product: the rows' count, summed mask /
 * A entries, summed streamed B entries (work) and the longest B row seen. */
typedef struct gk_bin_stat {
    int64_t rows, sum_m, sum_a, sum_work, max_b;
} gk_bin_stat;
int gk_sched_num_bins(void);
/* 1 if the learned scheduler may place `bin` on `variant` (0 otherwise). */
int gk_sched_variant_allowed(int bin, int variant);

/* mode 0: triangle counting on L (A = B = M = L, sum of C); mode 1: k-truss
 * support on a symmetric A (A = B = M = A, values written).  Fills, per bin,
 * the statistics, the plain heuristic's variant (or -1 for an empty bin), the
 * learned model's variant (NULL to skip; needs a loaded model) and the
 * gk_sched_num_features() features the model reads (NULL to skip). */
int gk_sched_bins(const gk_csr *G, int mode, gk_bin_stat *stats, int32_t *plain_variant, int32_t *learned_variant,
                  float *features, void *stream);

/* Runs the product of `mode` with bin b's rows on variant bin_variant[b]
 * (-1: rows skipped) and returns each variant kernel's CUDA-event time in
 * variant_ms[gk_sched_num_variants()] (synchronises); *sum (mode 0) receives
 * the partial sum of C over the rows that ran. */
int gk_tune_run(const gk_csr *G, int mode, const int32_t *bin_variant, float *variant_ms, uint64_t *sum,
                void *stream);

/* MLP of the learned scheduler, trained on the GPU by hand-written kernels.
 * w: gk_sched_model_size() floats (layout in graphkokkos_b200/csrc/gk_sched.cuh);
 * X: n x gk_sched_num_features(); Y, mask: n x gk_sched_num_variants() targets
 * (log2 ns per streamed B entry) and 0/1 weights.  All arrays are host memory. */
int gk_mlp_loss_grad(const float *w, const float *X, const float *Y, const float *mask, int n, float *loss,
                     float *grad, void *stream);
int gk_mlp_train(float *w, const float *X, const float *Y, const float *mask, int n, int epochs, float lr,
                 float *loss_trace, void *stream);
int gk_mlp_forward(const float *w, const float *X, int n, float *out, void *stream);

/* Forward-level shape of batched BC (pull: vertices gather from their
 * in-neighbours; push: frontier vertices scatter to their out-neighbours).
 * GK_SCHED_PLAIN picks by the direction-optimising rule, GK_SCHED_LEARNED by
 * an MLP of the same layout (gk_sched_model_size() floats) whose outputs 0 and
 * 1 predict log2 microseconds of a pull and a push level, loaded here.  The
 * shape changes only how the level is computed: sigma are integer path counts
 * in FP64, exact in any order of addition. */
int gk_bc_set_model(const float *weights, size_t n_floats);
int gk_bc_has_model(void);
/* Same from a model file (layout of gk_sched_load_model_file). */
int gk_bc_load_model_file(const char *path);

/* Autotuning run of gk_bc_batch (at most 512 sources, one chunk) with every
 * forward level on `shape` (0 pull, 1 push, -1 the plain rule), the levels
 * driven from the host: level_ms[i] receives the CUDA-event time of forward
 * level i+1 and level_feat[i*gk_sched_num_features()...] its features, for
 * i < min(*nlevels, max_levels); bc as gk_bc_batch. */
int gk_bc_tune(const gk_csr *A, const int32_t *sources, int nsources, int shape, double *bc, float *level_ms,
               float *level_feat, int max_levels, int *nlevels, void *stream);

/* ----- profiling (no reference counterpart; the reference prints chrono
 * brackets, src/main.cpp:74-86) -------------------------------------------------- */

/* One record per kernel-variant launch of a masked SpGEMM call made while
 * profiling is on: CUDA-event time of the launch and the rows / A entries /
 * mask entries / streamed B entries (work) it processed.
 * Mode 1 synchronises the stream after each call and fills the work fields;
 * mode 2 only brackets the launches with events (no synchronisation, work
 * fields 0) and gk_prof_flush() resolves them; mode 0 turns profiling off. */
typedef struct gk_prof_rec {
    int variant;
    float ms;
    int64_t rows, sum_a, sum_m, sum_work;
} gk_prof_rec;
int gk_prof_enable(int mode); /* also clears the records */
int gk_prof_flush(void);
int gk_prof_count(void);
int gk_prof_get(int i, gk_prof_rec *out);

/* Number of the library's own kernels launched so far in this process. */
int64_t gk_launch_count(void);

/* ----- misc ------------------------------------------------------------------- */
const char *gk_last_error_string(void);
int gk_version(void);

/* Test hook for error paths: after the next `after` scratch allocations of
 * this process (device or fixed-arena), the following one fails once with
 * GK_ERR_OOM; a negative value switches it off.  No counterpart in the
 * reference; it lets tests drive every allocation failure of an operator and
 * check that the library stays usable, without exhausting device memory. */
int gk_inject_alloc_failure(int64_t after);

#ifdef __cplusplus
}
#endif

#endif /* GK_B200_H */
