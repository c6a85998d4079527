/* grb_b200.h: C-ABI of the B200 semiring sparse-matrix-multiply library.
 *
 * Two groups of entry points, all extern "C" with plain pointers and sizes:
 *
 *  1. The drop-in boundary for SuiteSparse:GraphBLAS v9.3.1.  These take
 *     matrices exactly as the library's internal kernels see them (vectors of
 *     length vlen, int64 offsets/indices, GB_Type_code, GB_Opcode) and return
 *     results allocated with the library's own allocator, so a maintainer can
 *     call them from the library's method selectors in place of the CPU
 *     kernels (graphblas_b200/integration/gb_b200_gateway.c is that shim).
 *
 *  2. Device-resident matrices (grb_b200_dmatrix), used by the by-row host API
 *     in GraphBLAS_b200.h, by the batched kernel and by the request server:
 *     matrices stay in HBM between calls.
 *
 * Every call synchronises its own stream before returning.  Return values are
 * the reference's GrB_Info codes (Include/GraphBLAS.h:358-381):
 *   0 GrB_SUCCESS, 1 GrB_NO_VALUE (declined: the caller keeps its own path),
 *   -102 GrB_OUT_OF_MEMORY, -101 GrB_PANIC, -3 GrB_INVALID_VALUE,
 *   -6 GrB_DIMENSION_MISMATCH.
 */
#ifndef GRB_B200_H
#define GRB_B200_H

#include <stdint.h>
#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A sparse matrix as a set of vdim vectors of length vlen: the fields of
 * struct GB_Matrix_opaque the multiply kernels read
 * (Source/builtin/include/GB_matrix.h:213-235, 390, 455-515).  For a by-row
 * matrix the vectors are rows (vdim = nrows, vlen = ncols). */
typedef struct
{
    int64_t vlen;       /* length of each vector */
    int64_t vdim;       /* number of vectors */
    int64_t *p;         /* vdim+1 offsets */
    int64_t *i;         /* indices; a zombie holds -(i)-2 (GB_zombie.h:37) */
    void *x;            /* values: nnz entries, or 1 if iso; NULL = iso true */
    int type;           /* GB_Type_code (Source/builtin/include/GB_opaque.h:28) */
    bool iso;           /* all values equal x[0] */
    bool jumbled;       /* indices within a vector may be unsorted */
    int64_t nzombies;   /* number of zombies */
} grb_b200_matrix;

/* A built-in semiring: opcodes of the additive monoid and the multiplier
 * (GB_Opcode, Source/builtin/include/GB_opaque.h:209-247) and the type code
 * of the monoid (= the type of C). */
typedef struct
{
    int add_opcode;
    int mult_opcode;
    int type;
} grb_b200_semiring;

typedef void *(*grb_b200_malloc_fn)(size_t);
typedef void (*grb_b200_free_fn)(void *);

/* Initialise the device (idempotent).  Replaces GB_cuda_init
 * (CUDA/GB_cuda_init.c:18). */
int grb_b200_init(void);

/* Release cached device memory and streams.  No counterpart call in the
 * reference (its rmm pool is torn down by rmm_wrap_finalize,
 * rmm_wrap/rmm_wrap.h). */
int grb_b200_finalize(void);

/* Allocator used for every host array returned by the drop-in calls: the
 * library's GB_malloc function (Source/global/GB_Global.c:83-93,
 * GB_Global_malloc_function).  Default: malloc / free. */
void grb_b200_set_allocator(grb_b200_malloc_fn m, grb_b200_free_fn f);

/* True if the GPU takes this dot3 problem (sparse inputs, built-in semiring
 * in the compiled list, n and nnz below 2^31).  Replaces
 * GB_cuda_AxB_dot3_branch (CUDA/GB_cuda_AxB_dot3_branch.cpp:15). */
bool grb_b200_AxB_dot3_branch(const grb_b200_matrix *M,
                              const grb_b200_matrix *A,
                              const grb_b200_matrix *B,
                              const grb_b200_semiring *semiring, bool flipxy);

/* C<M> = A'*B by dot products (vector i of A with vector j of B, for every
 * entry i of vector j of M).  C gets M's pattern; empty dot products are
 * zombies, counted in C->nzombies; C->jumbled = M->jumbled.  Replaces
 * GB_AxB_dot3 (Source/mxm/GB_AxB_dot3.c:37-49) and GB_cuda_AxB_dot3
 * (CUDA/GB_cuda_AxB_dot3.cpp:35).  C->p, C->i, C->x are allocated with the
 * allocator above and owned by the caller. */
int grb_b200_AxB_dot3(grb_b200_matrix *C, const grb_b200_matrix *M,
                      bool Mask_struct, const grb_b200_matrix *A,
                      const grb_b200_matrix *B,
                      const grb_b200_semiring *semiring, bool flipxy);

/* C<M> = A*B by the saxpy method (C(:,j) = sum over k of A(:,k)*B(k,j), the
 * vectors of C being the vectors of B); M may be NULL, complemented or
 * structural.  The result is sorted, has no zombies, and *mask_applied is set
 * when M was used.  do_sort is accepted for signature parity; rows always come
 * back sorted.  Replaces GB_AxB_saxpy3 (Source/mxm/GB_AxB_saxpy3.h:19-36). */
int grb_b200_AxB_saxpy3(grb_b200_matrix *C, const grb_b200_matrix *M,
                        bool Mask_comp, bool Mask_struct,
                        const grb_b200_matrix *A, const grb_b200_matrix *B,
                        const grb_b200_semiring *semiring, bool flipxy,
                        bool *mask_applied, int do_sort);

/* s = reduce(A) with a built-in monoid (opcode, type of A), zombies skipped.
 * `out` receives one value of A's type.  Replaces GB_cuda_reduce_to_scalar
 * (CUDA/GB_cuda_reduce_to_scalar.cpp) / GB_reduce_to_scalar
 * (Source/reduce/GB_reduce_to_scalar.c:41). */
int grb_b200_reduce_to_scalar(void *out, const grb_b200_matrix *A,
                              int monoid_opcode);

/* Arm host-side allocation fault injection: the n-th following device
 * allocation fails (0 disarms), as the reference's malloc_debug counter does
 * for its own allocations (Source/global/GB_Global.c:83-93). */
void grb_b200_debug_fail_alloc(int64_t n);

/* Run this host thread's subsequent calls on the caller's CUDA stream
 * (a cudaStream_t; NULL returns to the library's stream pool).  Calls still
 * synchronise that stream before returning.  No counterpart in the
 * reference, whose GPU calls create a private stream each
 * (CUDA/GB_cuda_AxB_dot3.cpp:54). */
void grb_b200_set_stream(void *stream);

/* Keep a scratch buffer with a caller's stream (keep = true), as the
 * library's own streams have: the products, masked dot products, pull steps
 * and uploads run on that stream then take their temporary arrays from it
 * and stop allocating and freeing them call by call.  The buffer grows to
 * the largest call's need.  keep = false releases it, in the stream's order;
 * do that before destroying the stream.  No counterpart in the reference. */
int grb_b200_stream_keep_scratch(void *stream, bool keep);

/* Kernel timing with CUDA events recorded on the launching stream around
 * each launch of the hot kernels ("dot3", "saxpy3_numeric", ...).  Off by
 * default; the reference's equivalent is its GpuTimer
 * (CUDA/include/GB_cuda_timer.hpp) around the dot3 launches. */
void grb_b200_profile_enable(bool on);
/* Which launches get events: only those of kernel `kernel` (NULL: every
 * kernel), and of those one in `every` (a timed launch's two events cost
 * the stream several microseconds, which sampling spreads).  Applies to
 * launches after the call; the default is every launch of every kernel. */
int grb_b200_profile_select(const char *kernel, int every);
void grb_b200_profile_reset(void);
int grb_b200_profile(const char *kernel, double *total_ms, int64_t *launches);

/* ------------------------------------------------------------------------ */
/* Device-resident matrices (by-row CSR held in HBM)                        */
/* ------------------------------------------------------------------------ */

typedef struct grb_b200_dmatrix_s *grb_b200_dmatrix;

/* Upload host CSR (int64 offsets/indices, reference layout).  x == NULL makes
 * an iso-true pattern matrix. */
int grb_b200_dmatrix_upload(grb_b200_dmatrix *D, int64_t nrows, int64_t ncols,
                            const int64_t *p, const int64_t *i, const void *x,
                            int type, bool iso);

/* Download to host arrays allocated with the allocator above (zombies pruned
 * when prune is true, else returned as -(j)-2). */
int grb_b200_dmatrix_download(grb_b200_dmatrix D, int64_t **p, int64_t **i,
                              void **x, bool prune);

/* Copy a CSR matrix from the caller's arrays (host memory; page-locked
 * memory goes by DMA) and check it on the device: offsets start at 0, never
 * decrease and end at nnz = p[nrows], indices lie in [0, ncols), and no row
 * holds an index twice (rows given out of order are sorted on the device).
 * x holds nnz values of `type`.  GrB_INVALID_OBJECT when the arrays are not a
 * matrix.  The device half of GrB_Matrix_import's copy-and-check
 * (Source/import_export/GrB_Matrix_import.c:28-205, GB_import.c:330-367). */
int grb_b200_dmatrix_import(grb_b200_dmatrix *D, int64_t nrows, int64_t ncols,
                            const int64_t *p, const int64_t *i, const void *x,
                            int type);

/* Copy the live entries of D into the caller's arrays: nrows+1 offsets, then
 * nvals indices and nvals values (iso values expanded; x may be NULL).
 * nvals = stored entries - zombies (grb_b200_dmatrix_info).  The copy of
 * GrB_Matrix_export (Source/import_export/GrB_Matrix_export.c:38-215). */
int grb_b200_dmatrix_export(grb_b200_dmatrix D, int64_t *p, int64_t *i, void *x);

/* Serialized-matrix blobs in the reference's format (host code, no GPU).
 *
 * grb_b200_blob_decode reads a blob made by GxB_Matrix_serialize /
 * GrB_Matrix_serialize (Source/serialize/GB_serialize.c:43) the way
 * GB_deserialize reads it (Source/serialize/GB_deserialize.c:22): any of the
 * four sparsity forms, by row or by column, stored raw or LZ4 / LZ4HC
 * compressed.  The result is CSR by row with sorted rows: *Cp (nrows+1),
 * *Ci (nnz) and *Cx (nnz values, or one value when *iso) are malloc'ed and
 * the caller frees them.  expected_type 0 accepts any built-in type, else
 * the blob's type code must equal it.  GrB_INVALID_OBJECT for a malformed
 * blob, GrB_DOMAIN_MISMATCH for a type mismatch or a user-defined type,
 * GrB_NOT_IMPLEMENTED for ZSTD blocks (the reference's default compression)
 * and for built-in types outside bool/int32/uint32/int64/uint64/fp32/fp64.
 *
 * grb_b200_blob_encode writes an uncompressed sparse blob (the reference's
 * GxB_COMPRESSION_NONE form, which its deserializer reads) of a matrix given
 * compressed by row (p has nrows+1 entries, i column indices), or by column
 * when by_col (p has ncols+1 entries, i row indices; vectors are n-by-1 by
 * column).  x holds nnz values, or one value when iso.  blob_out NULL stores
 * the exact size in *blob_size; otherwise *blob_size is the room in
 * blob_out on input (GrB_INSUFFICIENT_SPACE when short) and the bytes
 * written on output (GrB_Matrix_serialize's contract). */
int grb_b200_blob_decode(const void *blob, size_t blob_size, int expected_type,
                         int64_t *nrows, int64_t *ncols, int *type, int64_t **Cp,
                         int64_t **Ci, void **Cx, bool *iso);
int grb_b200_blob_encode(void *blob_out, size_t *blob_size, int64_t nrows,
                         int64_t ncols, int type, const int64_t *p, const int64_t *i,
                         const void *x, bool iso, bool by_col);

int grb_b200_dmatrix_free(grb_b200_dmatrix *D);

/* nrows, ncols, stored entries (zombies included), zombies, type, iso */
int grb_b200_dmatrix_info(grb_b200_dmatrix D, int64_t *nrows, int64_t *ncols,
                          int64_t *nnz, int64_t *nzombies, int *type,
                          bool *iso);

/* The drop-in calls in two stages, for a caller that builds its own result
 * object: the product is left on the device as *C (free it with
 * grb_b200_dmatrix_free), grb_b200_dmatrix_info gives its sizes, and
 * grb_b200_dmatrix_copy_out copies it into arrays the caller allocated
 * with those sizes - the shim of the reference copies straight into the
 * arrays of the GrB_Matrix that GB_new_bix made (GB_AxB_dot3.c:172-176,
 * GB_AxB_saxpy3.c:242-244).  Same operands, rules and results as
 * grb_b200_AxB_dot3 / grb_b200_AxB_saxpy3 above (the dot3 result keeps
 * M's vector pointers and its zombies). */
int grb_b200_AxB_dot3_device(grb_b200_dmatrix *C, const grb_b200_matrix *M,
                             bool Mask_struct, const grb_b200_matrix *A,
                             const grb_b200_matrix *B,
                             const grb_b200_semiring *semiring, bool flipxy);

int grb_b200_AxB_saxpy3_device(grb_b200_dmatrix *C, const grb_b200_matrix *M,
                               bool Mask_comp, bool Mask_struct,
                               const grb_b200_matrix *A, const grb_b200_matrix *B,
                               const grb_b200_semiring *semiring, bool flipxy,
                               bool *mask_applied);

/* Every stored entry of D, zombies included (as GB_FLIP(i), the reference's
 * -(i)-2), into caller-owned arrays: p (vdim+1 offsets), i (nnz indices) and,
 * unless x is NULL, x (nnz values, iso values expanded).  Synchronous. */
int grb_b200_dmatrix_copy_out(grb_b200_dmatrix D, int64_t *p, int64_t *i, void *x);

/* C<M> = A*B' over M's pattern (row i of A . row j of B); zombies kept */
int grb_b200_dmxm_dot3(grb_b200_dmatrix *C, grb_b200_dmatrix M,
                       bool mask_struct, grb_b200_dmatrix A,
                       grb_b200_dmatrix B, const grb_b200_semiring *s);

/* C<M> = A*B row by row; M may be NULL */
int grb_b200_dmxm_saxpy3(grb_b200_dmatrix *C, grb_b200_dmatrix M,
                         bool mask_comp, bool mask_struct, grb_b200_dmatrix A,
                         grb_b200_dmatrix B, const grb_b200_semiring *s);

/* out = reduce(D) over live entries */
int grb_b200_dreduce(void *out, grb_b200_dmatrix D, int monoid_opcode);

/* Remove zombies (the zombie pruning of GB_wait, Source/wait/GB_wait.c:62) */
int grb_b200_dwait(grb_b200_dmatrix D);

/* An empty nrows-by-ncols device matrix of a type (GrB_Matrix_new,
 * Source/matrix/GrB_Matrix_new.c) */
int grb_b200_dmatrix_empty(grb_b200_dmatrix *D, int64_t nrows, int64_t ncols,
                           int type);

/* A device copy (GrB_Matrix_dup, Source/matrix/GrB_Matrix_dup.c) */
int grb_b200_dmatrix_dup(grb_b200_dmatrix *D, grb_b200_dmatrix A);

/* C<M,replace> = accum(C,T) in place; accum_opcode 0 = none.  Replaces
 * GB_accum_mask (Source/mask/GB_accum_mask.c:126). */
int grb_b200_daccum_mask(grb_b200_dmatrix C, grb_b200_dmatrix T,
                         grb_b200_dmatrix M, bool mask_comp, bool mask_struct,
                         bool replace, int accum_opcode);

/* B = A' (GB_transpose_cast, Source/transpose/GB_transpose_cast.c:18) */
int grb_b200_dtranspose(grb_b200_dmatrix *B, grb_b200_dmatrix A);

/* w<m> = A*u with u, m and w held as 1-by-n rows (GrB_mxv,
 * Source/mxm/GrB_mxv.c:18) */
int grb_b200_dmxv(grb_b200_dmatrix *w, grb_b200_dmatrix mask, bool mask_comp,
                  bool mask_struct, grb_b200_dmatrix A, grb_b200_dmatrix u,
                  const grb_b200_semiring *sr);

/* ------------------------------------------------------------------------ */
/* Batches of independent products                                          */
/* ------------------------------------------------------------------------ */

/* A batch of `count` independent products C_k = A_k * B_k (B_k = A_k when
 * Bp is NULL).  No counterpart in the reference, where the caller loops over
 * GrB_mxm (one GB_AxB_saxpy3 each, Source/mxm/GB_AxB_saxpy3.c:119).
 *
 * Inputs are concatenated CSR: instance k is a_nrows[k]-by-a_ncols[k]; its
 * a_nrows[k]+1 row offsets follow instance k-1's in Ap and index the shared
 * Aj/Ax arrays (Ap[0] = 0, offsets continue across instances).  B_k is
 * a_ncols[k]-by-b_ncols[k], laid out the same way in Bp/Bj/Bx.  Ax/Bx NULL:
 * pattern (iso one).  The batch is uploaded once as one block-diagonal
 * matrix; its symbolic phase runs at the first tune or run. */
typedef struct grb_b200_batch_s *grb_b200_batch;

int grb_b200_batch_create(grb_b200_batch *B, int count, const int64_t *a_nrows,
                          const int64_t *a_ncols, const int64_t *Ap,
                          const int64_t *Aj, const void *Ax,
                          const int64_t *b_ncols, const int64_t *Bp,
                          const int64_t *Bj, const void *Bx,
                          const grb_b200_semiring *semiring);

/* Pick bin thresholds, hash-table sizes and threads per row by timing a set
 * of candidate configurations on this batch (or reuse the cached choice for
 * its size class when use_cache); *best_ms gets the numeric time. */
int grb_b200_batch_tune(grb_b200_batch B, bool use_cache, double *best_ms);

/* Numeric phase for every instance; use_graph replays it as one captured
 * CUDA graph.  Synchronises before returning. */
int grb_b200_batch_run(grb_b200_batch B, bool use_graph);

/* Enqueue the captured graph on a caller's stream (NULL: the batch's own)
 * without waiting for it. */
int grb_b200_batch_enqueue(grb_b200_batch B, void *stream);

/* Sizes of the batch, its shared-memory bin count, the tuned numeric time
 * and the number of kernel launches in the captured graph (0 before the
 * first graph run). */
int grb_b200_batch_info(grb_b200_batch B, int64_t *total_rows, int64_t *nnz_c,
                        int64_t *capacity, int *nbins, double *tuned_ms,
                        int *graph_kernels);

/* Results, concatenated like the inputs (malloc'd, owned by the caller): Cp
 * holds a_nrows[k]+1 offsets per instance into Cj/Cx. */
int grb_b200_batch_result(grb_b200_batch B, int64_t **Cp, int64_t **Cj,
                          void **Cx, int64_t *nnz_per_instance);

/* The same results written into the caller's arrays (host memory; page-
 * locked memory is copied by DMA): Cp holds sum(a_nrows[k]+1) offsets, Cj and
 * Cx nnz_c entries (grb_b200_batch_info after a run). */
int grb_b200_batch_result_into(grb_b200_batch B, int64_t *Cp, int64_t *Cj, void *Cx,
                               int64_t *nnz_per_instance);

int grb_b200_batch_free(grb_b200_batch *B);

/* ------------------------------------------------------------------------ */
/* Request server over device-resident graphs                               */
/* ------------------------------------------------------------------------ */

/* No counterpart in the reference.  Request kinds: 1 = triangle count
 * (C<L> = L*U' plus_pair int64, then sum), 2 = SSSP relaxation step
 * (w = u' min.+ A, fp32, u a sparse frontier), 3 = product C = A*A
 * (plus_times fp64).  nslots worker streams run admitted requests
 * concurrently; a request is admitted when its estimated HBM footprint fits
 * in hbm_budget_bytes next to the running ones, and rejected
 * (GrB_OUT_OF_MEMORY status) if it never can. */
typedef struct grb_b200_server_s *grb_b200_server;

int grb_b200_server_create(grb_b200_server *S, int nslots,
                           int64_t hbm_budget_bytes, bool keep_results);

/* Upload a graph once: kind 1 takes a symmetric pattern (split into L, U),
 * kind 2 fp32 weights, kind 3 fp64 values; square n-by-n CSR. */
int grb_b200_server_add_graph(grb_b200_server S, int kind, int64_t n,
                              const int64_t *p, const int64_t *i, const void *x,
                              int *graph_id);

/* The same from a serialized blob (GxB_Matrix_serialize's format: any
 * sparsity form, raw, LZ4, LZ4HC or ZSTD; grb_b200_blob_decode reads it): a
 * square matrix, fp32 for kind 2 and fp64 for kind 3 (GrB_DOMAIN_MISMATCH
 * otherwise), any built-in type for kind 1 (only its pattern is used). */
int grb_b200_server_add_graph_blob(grb_b200_server S, int kind, const void *blob,
                                   size_t blob_size, int *graph_id);

/* Open-loop replay: request k of kind[k] on graph[k] arrives t_arrival[k]
 * seconds after the call; SSSP frontiers are fi/fx[fp[k] .. fp[k+1]). */
int grb_b200_server_replay(grb_b200_server S, int64_t nreq, const int *kind,
                           const int *graph, const double *t_arrival,
                           const int64_t *fp, const int64_t *fi,
                           const float *fx);

/* Outcome of request k: status (GrB_Info), count (triangles, or entries of
 * the result), checksum (sum of the result's values), latency (completion -
 * arrival) and queueing delay (start - arrival), in seconds. */
int grb_b200_server_request(grb_b200_server S, int64_t k, int *status,
                            int64_t *count, double *checksum, double *latency_s,
                            double *wait_s);

int grb_b200_server_result(grb_b200_server S, int64_t k, int64_t *p,
                           int64_t *i, void *x, int64_t *np, int64_t *ni);

int grb_b200_server_stats(grb_b200_server S, int64_t *admitted,
                          int64_t *rejected, int64_t *completed,
                          int64_t *failed, int64_t *peak_bytes,
                          int *peak_active, double *makespan_s);

/* Fusion of SSSP steps that wait together on the same graph: up to max_group
 * of them run as one product W = U min.+ A, one frontier per row of U (each
 * request's result and checksum are the same as when it runs alone).  1
 * turns fusion off; the default is 64.  Applies to the requests admitted
 * after the call. */
int grb_b200_server_set_fusion(grb_b200_server S, int max_group);

/* Products that fused more than one request, the requests they held, and the
 * largest group, over the last replay. */
int grb_b200_server_fusion_stats(grb_b200_server S, int64_t *fused_runs,
                                 int64_t *fused_requests, int *largest_group);

int grb_b200_server_free(grb_b200_server *S);

/* ------------------------------------------------------------------------ */
/* Masked dot products without any allocation                               */
/* ------------------------------------------------------------------------ */

/* Largest mask (number of entries) grb_b200_dot3_noalloc accepts. */
#define GRB_B200_DOT3_NOALLOC_MAX_ENTRIES 1048568

/* C<M> = A*B' over M's pattern, like grb_b200_dmxm_dot3, for callers that
 * cannot allocate device memory: a host application whose GPU memory belongs
 * to another allocator (a framework's caching pool or a preallocated arena
 * that must not be bypassed), or a latency-bound loop that must not call
 * cudaMalloc / cudaFree because those can synchronise the whole device.
 * This entry point has no counterpart in the reference.
 *
 * Every array is caller-owned device memory, by-row CSR with int32 offsets
 * and indices: M is nrows-by-ncols (structural; Mp has nrows+1 entries, Mj
 * has mnz), A is nrows-by-k and B is ncols-by-k (rows of both are the
 * operands of each dot product).  Ax/Bx hold values of the semiring's type
 * (one value when *_iso) and may be NULL when the multiplier does not read
 * them.  Outputs: Cj[p] = j for a live entry or -(j)-2 for a zombie (empty
 * dot product), Cx[p] its value, p over the mnz entries of M; C's row
 * offsets are Mp.  *nzombies (host) gets the zombie count.
 *
 * The work queue and counters live in a fixed 32 MiB device array inside the
 * library (held by every GPU that loads it until the process exits), so masks
 * above GRB_B200_DOT3_NOALLOC_MAX_ENTRIES entries are rejected with
 * GrB_INVALID_VALUE, as are dimensions of 2^31-1 or more.  Every entry takes
 * the merge / binary-search route (the shared-memory bitmap and hash routes
 * of the allocating entry point need per-call arrays), so counting semirings
 * on skewed graphs run slower here than through grb_b200_dmxm_dot3.  The call
 * changes no device-wide state: the default memory pool's settings are left
 * as the caller has them.  The first call on each device looks up that array's
 * device address, so make it before any stream capture.  Calls share the
 * array: calls that overlap on the same GPU (concurrent streams or threads)
 * race and must be serialised by the caller.  Runs on `stream` (a
 * cudaStream_t, NULL = legacy default stream) and synchronises it before
 * returning. */
int grb_b200_dot3_noalloc(int64_t nrows, int64_t ncols, int64_t mnz,
                          const int32_t *Mp, const int32_t *Mj,
                          const int32_t *Ap, const int32_t *Aj, const void *Ax,
                          bool A_iso, const int32_t *Bp, const int32_t *Bj,
                          const void *Bx, bool B_iso,
                          const grb_b200_semiring *semiring, int32_t *Cj,
                          void *Cx, int64_t *nzombies, void *stream);

#ifdef __cplusplus
}
#endif

#endif
