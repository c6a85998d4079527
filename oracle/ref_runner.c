// ref_runner.c: drives the reference SuiteSparse:GraphBLAS library (built
// from its own sources into oracle/_ref/ by oracle/ref.mk) through its public
// C API, on CSR arrays handed over from Python.  Test infrastructure only: it
// pins the oracle restatement to the reference's real output and times the
// reference's CPU path for the CPU baseline.  No product code links it.
//
// Matrices are moved in and out with GxB_Matrix_pack_CSR / unpack_CSR
// (Include/GraphBLAS.h:9449, :9976), so both sides see identical bytes.
// Operator / type codes are the reference's GB_Opcode / GB_Type_code numbers
// (Source/builtin/include/GB_opaque.h:28-42, 209-247).

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdbool.h>
#include <omp.h>
#include "GraphBLAS.h"

enum { T_BOOL = 1, T_INT32 = 6, T_UINT32 = 7, T_INT64 = 8, T_UINT64 = 9,
       T_FP32 = 10, T_FP64 = 11 };
enum { OP_FIRST = 72, OP_SECOND = 73, OP_ANY = 74, OP_PAIR = 75, OP_MIN = 76,
       OP_MAX = 77, OP_PLUS = 78, OP_MINUS = 79, OP_RMINUS = 80, OP_TIMES = 81,
       OP_DIV = 82, OP_LOR = 91, OP_LAND = 92, OP_LXOR = 93, OP_EQ = 102,
       OP_FIRSTI = 115, OP_FIRSTJ = 117, OP_SECONDI = 119, OP_SECONDJ = 121 };

static GrB_Type type_of(int t)
{
    switch (t)
    {
        case T_BOOL: return GrB_BOOL;
        case T_INT32: return GrB_INT32;
        case T_UINT32: return GrB_UINT32;
        case T_INT64: return GrB_INT64;
        case T_UINT64: return GrB_UINT64;
        case T_FP32: return GrB_FP32;
        case T_FP64: return GrB_FP64;
    }
    return NULL;
}

static size_t tsize(int t)
{
    switch (t)
    {
        case T_BOOL: return 1;
        case T_INT32: case T_UINT32: case T_FP32: return 4;
        default: return 8;
    }
}

#define BY_TYPE(PFX, SFX, t)                                                \
    switch (t) {                                                            \
        case T_BOOL: return PFX##BOOL##SFX;                                 \
        case T_INT32: return PFX##INT32##SFX;                               \
        case T_UINT32: return PFX##UINT32##SFX;                             \
        case T_INT64: return PFX##INT64##SFX;                               \
        case T_UINT64: return PFX##UINT64##SFX;                             \
        case T_FP32: return PFX##FP32##SFX;                                 \
        case T_FP64: return PFX##FP64##SFX;                                 \
    } return NULL;

#define BY_TYPE_NB(PFX, SFX, t)                                             \
    switch (t) {                                                            \
        case T_INT32: return PFX##INT32##SFX;                               \
        case T_UINT32: return PFX##UINT32##SFX;                             \
        case T_INT64: return PFX##INT64##SFX;                               \
        case T_UINT64: return PFX##UINT64##SFX;                             \
        case T_FP32: return PFX##FP32##SFX;                                 \
        case T_FP64: return PFX##FP64##SFX;                                 \
    } return NULL;

static GrB_Monoid monoid_of(int op, int t)
{
    if (t == T_BOOL)
    {
        // boolean PLUS/MAX are LOR and TIMES/MIN are LAND
        switch (op)
        {
            case OP_PLUS: case OP_MAX: case OP_LOR: return GrB_LOR_MONOID_BOOL;
            case OP_TIMES: case OP_MIN: case OP_LAND: return GrB_LAND_MONOID_BOOL;
            case OP_ANY: return GxB_ANY_BOOL_MONOID;
            case OP_LXOR: return GrB_LXOR_MONOID_BOOL;
        }
        return NULL;
    }
    switch (op)
    {
        case OP_PLUS:  { BY_TYPE_NB(GrB_PLUS_MONOID_, , t) }
        case OP_TIMES: { BY_TYPE_NB(GrB_TIMES_MONOID_, , t) }
        case OP_MIN:   { BY_TYPE_NB(GrB_MIN_MONOID_, , t) }
        case OP_MAX:   { BY_TYPE_NB(GrB_MAX_MONOID_, , t) }
        case OP_ANY:   { BY_TYPE_NB(GxB_ANY_, _MONOID, t) }
        case OP_LOR:   return GrB_LOR_MONOID_BOOL;
        case OP_LAND:  return GrB_LAND_MONOID_BOOL;
        case OP_LXOR:  return GrB_LXOR_MONOID_BOOL;
    }
    return NULL;
}

static GrB_BinaryOp binop_of(int op, int t)
{
    switch (op)
    {
        case OP_FIRST:  { BY_TYPE(GrB_FIRST_, , t) }
        case OP_SECOND: { BY_TYPE(GrB_SECOND_, , t) }
        case OP_PAIR:   { BY_TYPE(GxB_PAIR_, , t) }
        case OP_PLUS:   { BY_TYPE(GrB_PLUS_, , t) }
        case OP_MINUS:  { BY_TYPE(GrB_MINUS_, , t) }
        case OP_RMINUS: { BY_TYPE(GxB_RMINUS_, , t) }
        case OP_TIMES:  { BY_TYPE(GrB_TIMES_, , t) }
        case OP_DIV:    { BY_TYPE(GrB_DIV_, , t) }
        case OP_MIN:    { BY_TYPE(GrB_MIN_, , t) }
        case OP_MAX:    { BY_TYPE(GrB_MAX_, , t) }
        case OP_LOR:    { BY_TYPE(GxB_LOR_, , t) }
        case OP_LAND:   { BY_TYPE(GxB_LAND_, , t) }
        case OP_FIRSTI:  return t == T_INT32 ? GxB_FIRSTI_INT32 : GxB_FIRSTI_INT64;
        case OP_FIRSTJ:  return t == T_INT32 ? GxB_FIRSTJ_INT32 : GxB_FIRSTJ_INT64;
        case OP_SECONDI: return t == T_INT32 ? GxB_SECONDI_INT32 : GxB_SECONDI_INT64;
        case OP_SECONDJ: return t == T_INT32 ? GxB_SECONDJ_INT32 : GxB_SECONDJ_INT64;
    }
    return NULL;
}

int ref_init(int nthreads)
{
    static int done = 0;
    if (!done)
    {
        GrB_Info info = GrB_init(GrB_NONBLOCKING);
        if (info != GrB_SUCCESS) return (int)info;
        done = 1;
    }
    return (int)GxB_Global_Option_set_INT32(GxB_NTHREADS, nthreads);
}

int ref_set_nthreads(int nthreads)
{
    return (int)GxB_Global_Option_set_INT32(GxB_NTHREADS, nthreads);
}

// Build a by-row GrB_Matrix from CSR copies of the caller's arrays.
// x == NULL builds an iso-true pattern matrix of type t.
static GrB_Info make_csr(GrB_Matrix *A, int t, int64_t nrows, int64_t ncols,
                         const int64_t *p, const int64_t *i, const void *x)
{
    GrB_Info info = GrB_Matrix_new(A, type_of(t), nrows, ncols);
    if (info != GrB_SUCCESS) return info;
    GxB_Matrix_Option_set_INT32(*A, GxB_FORMAT, GxB_BY_ROW);
    int64_t nnz = p[nrows];
    size_t ts = tsize(t);
    GrB_Index *Ap = malloc((nrows + 1) * sizeof(int64_t));
    GrB_Index *Aj = malloc((nnz ? nnz : 1) * sizeof(int64_t));
    memcpy(Ap, p, (nrows + 1) * sizeof(int64_t));
    memcpy(Aj, i, nnz * sizeof(int64_t));
    void *Ax;
    bool iso = (x == NULL);
    if (iso)
    {
        Ax = calloc(1, 8);
        switch (t)
        {
            case T_BOOL: *(bool *)Ax = true; break;
            case T_INT32: *(int32_t *)Ax = 1; break;
            case T_UINT32: *(uint32_t *)Ax = 1; break;
            case T_INT64: *(int64_t *)Ax = 1; break;
            case T_UINT64: *(uint64_t *)Ax = 1; break;
            case T_FP32: *(float *)Ax = 1; break;
            case T_FP64: *(double *)Ax = 1; break;
        }
    }
    else
    {
        Ax = malloc((nnz ? nnz : 1) * ts);
        memcpy(Ax, x, nnz * ts);
    }
    return GxB_Matrix_pack_CSR(*A, &Ap, &Aj, &Ax, (nrows + 1) * sizeof(int64_t),
                               (nnz ? nnz : 1) * sizeof(int64_t),
                               iso ? 8 : (nnz ? nnz : 1) * ts, iso, false, NULL);
}

typedef struct
{
    int64_t nrows, nnz;
    int type;
    GrB_Index *p, *i;
    void *x;
    double seconds;
} ref_csr;

void ref_free(ref_csr *C)
{
    if (!C) return;
    free(C->p); free(C->i); free(C->x); free(C);
}

int64_t ref_nnz(const ref_csr *C) { return C->nnz; }
double ref_seconds(const ref_csr *C) { return C->seconds; }

void ref_export(const ref_csr *C, int64_t *p, int64_t *i, void *x)
{
    memcpy(p, C->p, (C->nrows + 1) * sizeof(int64_t));
    memcpy(i, C->i, C->nnz * sizeof(int64_t));
    if (x) memcpy(x, C->x, C->nnz * tsize(C->type));
}

// C<M> = accum (C, A*B) (or A*B') with the reference's GrB_mxm.
//   method: 0 auto, 1 dot (GxB_AxB_DOT), 2 Gustavson, 3 hash
//   transpose_b: the GrB_INP1 = GrB_TRAN descriptor (C = A*B')
//   Cin == NULL (Cp_in == NULL) starts from an empty C.
// Returns NULL on error; *info_out gets the GrB_Info.
ref_csr *ref_mxm(int64_t m, int64_t n, int64_t ncols,
    const int64_t *Ap, const int64_t *Ai, const void *Ax, int atype,
    int64_t bnrows, const int64_t *Bp, const int64_t *Bi, const void *Bx, int btype,
    const int64_t *Mp, const int64_t *Mi, const void *Mx, int mtype,
    const int64_t *Cp_in, const int64_t *Ci_in, const void *Cx_in,
    bool mask_struct, bool mask_comp, bool replace, bool transpose_b,
    int accum, int add, int mult, int ctype, int method, int *info_out)
{
    GrB_Matrix A = NULL, B = NULL, M = NULL, C = NULL;
    GrB_Semiring S = NULL;
    GrB_Descriptor D = NULL;
    ref_csr *R = NULL;
    GrB_Info info;
    int64_t bncols = transpose_b ? n : ncols;
    (void)bncols;
    #define TRY(x) { info = (x); if (info != GrB_SUCCESS) goto done; }
    TRY(make_csr(&A, atype, m, n, Ap, Ai, Ax));
    TRY(make_csr(&B, btype, bnrows, transpose_b ? n : ncols, Bp, Bi, Bx));
    if (Mp) TRY(make_csr(&M, mtype, m, ncols, Mp, Mi, Mx));
    if (Cp_in) TRY(make_csr(&C, ctype, m, ncols, Cp_in, Ci_in, Cx_in))
    else
    {
        TRY(GrB_Matrix_new(&C, type_of(ctype), m, ncols));
        GxB_Matrix_Option_set_INT32(C, GxB_FORMAT, GxB_BY_ROW);
    }
    TRY(GrB_Semiring_new(&S, monoid_of(add, ctype), binop_of(mult, ctype)));
    TRY(GrB_Descriptor_new(&D));
    if (mask_struct && mask_comp)
        TRY(GrB_Descriptor_set(D, GrB_MASK, GrB_COMP_STRUCTURE))
    else if (mask_struct) TRY(GrB_Descriptor_set(D, GrB_MASK, GrB_STRUCTURE))
    else if (mask_comp) TRY(GrB_Descriptor_set(D, GrB_MASK, GrB_COMP))
    if (replace) TRY(GrB_Descriptor_set(D, GrB_OUTP, GrB_REPLACE));
    if (transpose_b) TRY(GrB_Descriptor_set(D, GrB_INP1, GrB_TRAN));
    if (method == 1) TRY(GrB_Descriptor_set(D, GxB_AxB_METHOD, GxB_AxB_DOT))
    else if (method == 2) TRY(GrB_Descriptor_set(D, GxB_AxB_METHOD, GxB_AxB_GUSTAVSON))
    else if (method == 3) TRY(GrB_Descriptor_set(D, GxB_AxB_METHOD, GxB_AxB_HASH))
    double t0 = omp_get_wtime();
    TRY(GrB_mxm(C, M, accum ? binop_of(accum, ctype) : NULL, S, A, B, D));
    TRY(GrB_Matrix_wait(C, GrB_MATERIALIZE));
    double t1 = omp_get_wtime();
    R = calloc(1, sizeof(ref_csr));
    R->nrows = m; R->type = ctype; R->seconds = t1 - t0;
    GrB_Index psize, isize, xsize;
    bool iso = false;
    TRY(GxB_Matrix_unpack_CSR(C, &R->p, &R->i, &R->x, &psize, &isize, &xsize,
                              &iso, NULL, NULL));
    R->nnz = R->p[m];
    if (iso && R->nnz > 0)
    {
        size_t ts = tsize(ctype);
        void *x = malloc(R->nnz * ts);
        for (int64_t k = 0; k < R->nnz; k++)
            memcpy((char *)x + k * ts, R->x, ts);
        free(R->x);
        R->x = x;
    }
done:
    GrB_Matrix_free(&A); GrB_Matrix_free(&B); GrB_Matrix_free(&M);
    GrB_Matrix_free(&C); GrB_Semiring_free(&S); GrB_Descriptor_free(&D);
    if (info_out) *info_out = (int)info;
    if (info != GrB_SUCCESS) { ref_free(R); return NULL; }
    return R;
    #undef TRY
}

// Triangle count with the reference's dot3 path, as LAGraph does it:
// C<L> = L*U' (plus_pair int64, structural mask), ntri = sum (C).
// Runs `reps` timed repetitions; times[r] gets each one (mxm + reduce).
int ref_tricount(int64_t n, const int64_t *Lp, const int64_t *Li,
                 const int64_t *Up, const int64_t *Ui, int reps,
                 double *times, int64_t *ntri)
{
    GrB_Matrix L = NULL, U = NULL, C = NULL;
    GrB_Info info;
    #define TRY(x) { info = (x); if (info != GrB_SUCCESS) goto done; }
    TRY(make_csr(&L, T_BOOL, n, n, Lp, Li, NULL));
    TRY(make_csr(&U, T_BOOL, n, n, Up, Ui, NULL));
    for (int r = 0; r < reps; r++)
    {
        double t0 = omp_get_wtime();
        TRY(GrB_Matrix_new(&C, GrB_INT64, n, n));
        TRY(GrB_mxm(C, L, NULL, GxB_PLUS_PAIR_INT64, L, U, GrB_DESC_ST1));
        int64_t s = 0;
        TRY(GrB_Matrix_reduce_INT64(&s, NULL, GrB_PLUS_MONOID_INT64, C, NULL));
        double t1 = omp_get_wtime();
        GrB_Matrix_free(&C);
        times[r] = t1 - t0;
        *ntri = s;
    }
done:
    GrB_Matrix_free(&L); GrB_Matrix_free(&U); GrB_Matrix_free(&C);
    return (int)info;
    #undef TRY
}

// Level-synchronous BFS parents as in LAGraph's push step:
//   q<!struct(p), replace> = q any_secondi S ; p<struct(q)> = q
// The frontier is kept sparse (GxB_SPARSITY_CONTROL).  parent[v] = -1 when
// unreached.  Returns GrB_Info; *seconds gets the loop time.
int ref_bfs(int64_t n, const int64_t *Sp, const int64_t *Si, int64_t src,
            int64_t *parent, double *seconds, int *nlevels)
{
    GrB_Matrix S = NULL;
    GrB_Vector q = NULL, p = NULL;
    GrB_Info info;
    #define TRY(x) { info = (x); if (info != GrB_SUCCESS) goto done; }
    TRY(make_csr(&S, T_BOOL, n, n, Sp, Si, NULL));
    double t0 = omp_get_wtime();
    TRY(GrB_Vector_new(&q, GrB_INT64, n));
    TRY(GrB_Vector_new(&p, GrB_INT64, n));
    GxB_Vector_Option_set_INT32(q, GxB_SPARSITY_CONTROL, GxB_SPARSE);
    GxB_Vector_Option_set_INT32(p, GxB_SPARSITY_CONTROL, GxB_SPARSE);
    TRY(GrB_Vector_setElement_INT64(q, src, src));
    TRY(GrB_Vector_setElement_INT64(p, src, src));
    GrB_Index nq = 1;
    int lev = 0;
    while (nq > 0)
    {
        lev++;
        TRY(GrB_vxm(q, p, NULL, GxB_ANY_SECONDI_INT64, q, S, GrB_DESC_RSC));
        TRY(GrB_Vector_nvals(&nq, q));
        if (nq == 0) break;
        TRY(GrB_Vector_assign(p, q, NULL, q, GrB_ALL, n, GrB_DESC_S));
    }
    TRY(GrB_Vector_wait(p, GrB_MATERIALIZE));
    *seconds = omp_get_wtime() - t0;
    *nlevels = lev;
    for (int64_t v = 0; v < n; v++) parent[v] = -1;
    {
        GrB_Index np = 0;
        TRY(GrB_Vector_nvals(&np, p));
        GrB_Index *Iv = malloc((np ? np : 1) * sizeof(GrB_Index));
        int64_t *Xv = malloc((np ? np : 1) * sizeof(int64_t));
        GrB_Index nn = np;
        info = GrB_Vector_extractTuples_INT64(Iv, Xv, &nn, p);
        if (info == GrB_SUCCESS)
            for (GrB_Index t = 0; t < nn; t++) parent[Iv[t]] = Xv[t];
        free(Iv); free(Xv);
    }
done:
    GrB_Matrix_free(&S); GrB_Vector_free(&q); GrB_Vector_free(&p);
    return (int)info;
    #undef TRY
}

// A loop of `count` independent C_i = A_i*A_i (min_plus fp32 by default),
// the reference's per-call path for a batch of small problems.  Instance i
// uses rows [off[i], off[i+1]) of the concatenated row pointer arrays:
// Ap + poff[i] (n_i + 1 entries) indexes Ai + ioff[i] / Ax + ioff[i].
// nnz_out[i] gets nnz(C_i); returns GrB_Info, *seconds the loop time.
// Position-weighted digest of a CSR matrix (row, column and value bits of
// every entry, in storage order); the same function is oracle.csr_digest in
// Python, so results can be compared without moving them.
static uint64_t csr_digest(int64_t nrows, const GrB_Index *p, const GrB_Index *i,
                           const void *x, size_t ts)
{
    const uint64_t K1 = 0x9E3779B97F4A7C15ull, K2 = 0xC2B2AE3D27D4EB4Full;
    const uint64_t K3 = 0x165667B19E3779F9ull, K4 = 0x27D4EB2F165667C5ull;
    uint64_t h = (uint64_t)nrows * K1 + (uint64_t)p[nrows];
    for (int64_t r = 0; r < nrows; r++)
        for (GrB_Index t = p[r]; t < p[r + 1]; t++)
        {
            uint64_t bits = 0;
            memcpy(&bits, (const char *)x + t * ts, ts);
            h += (((uint64_t)r * K1 + (uint64_t)i[t]) * K2 + bits + 1) * ((uint64_t)t * K3 + K4);
        }
    return h;
}

// digest_out (optional, one per instance): csr_digest of each C_i after the
// timed loop
int ref_batch_square(int count, const int64_t *nsz, const int64_t *poff,
                     const int64_t *ioff, const int64_t *Ap, const int64_t *Ai,
                     const float *Ax, int add, int mult, int64_t *nnz_out,
                     double *seconds, uint64_t *digest_out)
{
    GrB_Info info = GrB_SUCCESS;
    GrB_Semiring S = NULL;
    GrB_Matrix *As = calloc(count, sizeof(GrB_Matrix));
    GrB_Matrix *Cs = calloc(count, sizeof(GrB_Matrix));
    #define TRY(x) { info = (x); if (info != GrB_SUCCESS) goto done; }
    TRY(GrB_Semiring_new(&S, monoid_of(add, T_FP32), binop_of(mult, T_FP32)));
    for (int b = 0; b < count; b++)
    {
        int64_t n = nsz[b];
        // rebase this instance's row pointers to start at zero
        int64_t *p = malloc((n + 1) * sizeof(int64_t));
        for (int64_t r = 0; r <= n; r++) p[r] = Ap[poff[b] + r] - Ap[poff[b]];
        info = make_csr(&As[b], T_FP32, n, n, p, Ai + ioff[b], Ax + ioff[b]);
        free(p);
        if (info != GrB_SUCCESS) goto done;
        TRY(GrB_Matrix_new(&Cs[b], GrB_FP32, n, n));
    }
    double t0 = omp_get_wtime();
    for (int b = 0; b < count; b++)
    {
        TRY(GrB_mxm(Cs[b], NULL, NULL, S, As[b], As[b], NULL));
        TRY(GrB_Matrix_wait(Cs[b], GrB_MATERIALIZE));
    }
    *seconds = omp_get_wtime() - t0;
    for (int b = 0; b < count; b++)
    {
        GrB_Index nv = 0;
        GrB_Matrix_nvals(&nv, Cs[b]);
        nnz_out[b] = (int64_t)nv;
        if (digest_out)
        {
            GrB_Index *p = NULL, *i = NULL, psz, isz, xsz;
            void *x = NULL;
            bool iso = false;
            TRY(GxB_Matrix_unpack_CSR(Cs[b], &p, &i, &x, &psz, &isz, &xsz, &iso, NULL,
                                      NULL));
            if (iso && p[nsz[b]] > 0)
            {
                // expand an iso result to one value per entry
                float v = *(float *)x;
                free(x);
                x = malloc(p[nsz[b]] * sizeof(float));
                for (GrB_Index t = 0; t < p[nsz[b]]; t++) ((float *)x)[t] = v;
            }
            digest_out[b] = csr_digest(nsz[b], p, i, x, sizeof(float));
            free(p); free(i); free(x);
        }
    }
done:
    for (int b = 0; b < count; b++)
    {
        GrB_Matrix_free(&As[b]);
        GrB_Matrix_free(&Cs[b]);
    }
    free(As); free(Cs);
    GrB_Semiring_free(&S);
    return (int)info;
    #undef TRY
}

//------------------------------------------------------------------------------
// The serving workload on the reference: the same open-loop request trace
// replayed through a pool of host threads over graphs held in CPU memory.
// Request kinds: 1 triangle count (C<L> = L*U' plus_pair int64, then sum),
// 2 SSSP relaxation step (w = u min.+ S, fp32, u a sparse frontier),
// 3 product C = S*S (plus_times fp64).  Each worker runs one request at a
// time with GxB_NTHREADS = nthreads_per_call; latency = completion - arrival.
//------------------------------------------------------------------------------

#include <pthread.h>
#include <time.h>

#define REF_SERVE_MAX_GRAPHS 64

static struct
{
    int ngraphs;
    int kind[REF_SERVE_MAX_GRAPHS];
    int64_t n[REF_SERVE_MAX_GRAPHS];
    GrB_Matrix S[REF_SERVE_MAX_GRAPHS], L[REF_SERVE_MAX_GRAPHS], U[REF_SERVE_MAX_GRAPHS];
} g_serve;

static double now_s(const struct timespec *t0)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)(t.tv_sec - t0->tv_sec) + 1e-9 * (double)(t.tv_nsec - t0->tv_nsec);
}

// Add a resident graph: kind 1 takes a symmetric pattern (split into strict
// lower / upper triangles here), kind 2 fp32 weights, kind 3 fp64 values.
int ref_serve_add_graph(int kind, int64_t n, const int64_t *p, const int64_t *i,
                        const void *x)
{
    if (g_serve.ngraphs >= REF_SERVE_MAX_GRAPHS) return (int)GrB_INVALID_VALUE;
    const int g = g_serve.ngraphs;
    GrB_Info info = GrB_SUCCESS;
    g_serve.S[g] = g_serve.L[g] = g_serve.U[g] = NULL;
    if (kind == 1)
    {
        int64_t *Lp = malloc((n + 1) * sizeof(int64_t)), *Up = malloc((n + 1) * sizeof(int64_t));
        int64_t *Li = malloc((p[n] / 2 + 1) * sizeof(int64_t));
        int64_t *Ui = malloc((p[n] / 2 + 1) * sizeof(int64_t));
        int64_t nl = 0, nu = 0;
        for (int64_t r = 0; r < n; r++)
        {
            Lp[r] = nl; Up[r] = nu;
            for (int64_t q = p[r]; q < p[r + 1]; q++)
            {
                if (i[q] < r) Li[nl++] = i[q];
                else if (i[q] > r) Ui[nu++] = i[q];
            }
        }
        Lp[n] = nl; Up[n] = nu;
        info = make_csr(&g_serve.L[g], T_BOOL, n, n, Lp, Li, NULL);
        if (info == GrB_SUCCESS) info = make_csr(&g_serve.U[g], T_BOOL, n, n, Up, Ui, NULL);
        free(Lp); free(Up); free(Li); free(Ui);
    }
    else
    {
        info = make_csr(&g_serve.S[g], kind == 2 ? T_FP32 : T_FP64, n, n, p, i, x);
    }
    if (info != GrB_SUCCESS) return (int)info;
    g_serve.kind[g] = kind;
    g_serve.n[g] = n;
    g_serve.ngraphs++;
    return (int)GrB_SUCCESS;
}

void ref_serve_clear(void)
{
    for (int g = 0; g < g_serve.ngraphs; g++)
    {
        GrB_Matrix_free(&g_serve.S[g]);
        GrB_Matrix_free(&g_serve.L[g]);
        GrB_Matrix_free(&g_serve.U[g]);
    }
    g_serve.ngraphs = 0;
}

typedef struct
{
    int64_t nreq;
    const int *kind, *graph;
    const double *t_arrival;
    const int64_t *fp, *fi;
    const float *fx;
    struct timespec t0;
    pthread_mutex_t mu;
    pthread_cond_t cv;
    int64_t submitted, next;
    // outputs
    int *status;
    int64_t *count;
    double *checksum, *latency;
} serve_run;

static int serve_one(serve_run *R, int64_t k)
{
    const int g = R->graph[k];
    const int64_t n = g_serve.n[g];
    GrB_Info info = GrB_SUCCESS;
    #define TRY(x) { info = (x); if (info != GrB_SUCCESS) goto done; }
    GrB_Matrix C = NULL;
    GrB_Vector u = NULL, w = NULL;
    GrB_Index *ui = NULL;
    if (R->kind[k] == 1)
    {
        int64_t s = 0;
        TRY(GrB_Matrix_new(&C, GrB_INT64, n, n));
        TRY(GrB_mxm(C, g_serve.L[g], NULL, GxB_PLUS_PAIR_INT64, g_serve.L[g], g_serve.U[g],
                    GrB_DESC_ST1));
        TRY(GrB_Matrix_reduce_INT64(&s, NULL, GrB_PLUS_MONOID_INT64, C, NULL));
        R->count[k] = s;
        R->checksum[k] = (double)s;
    }
    else if (R->kind[k] == 2)
    {
        const int64_t lo = R->fp[k], nu = R->fp[k + 1] - lo;
        ui = malloc((nu ? nu : 1) * sizeof(GrB_Index));
        for (int64_t t = 0; t < nu; t++) ui[t] = (GrB_Index)R->fi[lo + t];
        TRY(GrB_Vector_new(&u, GrB_FP32, n));
        TRY(GrB_Vector_build_FP32(u, ui, R->fx + lo, nu, GrB_FIRST_FP32));
        TRY(GrB_Vector_new(&w, GrB_FP32, n));
        TRY(GrB_vxm(w, NULL, NULL, GrB_MIN_PLUS_SEMIRING_FP32, u, g_serve.S[g], NULL));
        GrB_Index nv = 0;
        float sum = 0;
        TRY(GrB_Vector_nvals(&nv, w));
        TRY(GrB_Vector_reduce_FP32(&sum, NULL, GrB_PLUS_MONOID_FP32, w, NULL));
        R->count[k] = (int64_t)nv;
        R->checksum[k] = sum;
    }
    else
    {
        TRY(GrB_Matrix_new(&C, GrB_FP64, n, n));
        TRY(GrB_mxm(C, NULL, NULL, GrB_PLUS_TIMES_SEMIRING_FP64, g_serve.S[g], g_serve.S[g],
                    NULL));
        GrB_Index nv = 0;
        double sum = 0;
        TRY(GrB_Matrix_nvals(&nv, C));
        TRY(GrB_Matrix_reduce_FP64(&sum, NULL, GrB_PLUS_MONOID_FP64, C, NULL));
        R->count[k] = (int64_t)nv;
        R->checksum[k] = sum;
    }
done:
    GrB_Matrix_free(&C);
    GrB_Vector_free(&u);
    GrB_Vector_free(&w);
    free(ui);
    return (int)info;
    #undef TRY
}

static void *serve_worker(void *arg)
{
    serve_run *R = (serve_run *)arg;
    while (true)
    {
        pthread_mutex_lock(&R->mu);
        while (R->next >= R->submitted && R->submitted < R->nreq)
            pthread_cond_wait(&R->cv, &R->mu);
        if (R->next >= R->nreq) { pthread_mutex_unlock(&R->mu); break; }
        const int64_t k = R->next++;
        pthread_mutex_unlock(&R->mu);
        R->status[k] = serve_one(R, k);
        R->latency[k] = now_s(&R->t0) - R->t_arrival[k];
    }
    return NULL;
}

// Replay: request k arrives t_arrival[k] seconds after the call and is taken
// by the first free worker (FIFO).  Returns GrB_Info; *makespan gets the time
// to the last completion.
int ref_serve_replay(int nworkers, int nthreads_per_call, int64_t nreq, const int *kind,
                     const int *graph, const double *t_arrival, const int64_t *fp,
                     const int64_t *fi, const float *fx, int *status, int64_t *count,
                     double *checksum, double *latency, double *makespan)
{
    GxB_Global_Option_set_INT32(GxB_GLOBAL_NTHREADS, nthreads_per_call);
    serve_run R;
    memset(&R, 0, sizeof(R));
    R.nreq = nreq; R.kind = kind; R.graph = graph; R.t_arrival = t_arrival;
    R.fp = fp; R.fi = fi; R.fx = fx;
    R.status = status; R.count = count; R.checksum = checksum; R.latency = latency;
    pthread_mutex_init(&R.mu, NULL);
    pthread_cond_init(&R.cv, NULL);
    pthread_t *th = malloc(nworkers * sizeof(pthread_t));
    clock_gettime(CLOCK_MONOTONIC, &R.t0);
    for (int w = 0; w < nworkers; w++) pthread_create(&th[w], NULL, serve_worker, &R);
    for (int64_t k = 0; k < nreq; k++)
    {
        // open loop: wait for the arrival time, never for the workers
        const double wait = t_arrival[k] - now_s(&R.t0);
        if (wait > 0)
        {
            struct timespec ts = {(time_t)wait, (long)((wait - (double)(time_t)wait) * 1e9)};
            nanosleep(&ts, NULL);
        }
        pthread_mutex_lock(&R.mu);
        R.submitted = k + 1;
        pthread_cond_broadcast(&R.cv);
        pthread_mutex_unlock(&R.mu);
    }
    for (int w = 0; w < nworkers; w++) pthread_join(th[w], NULL);
    *makespan = now_s(&R.t0);
    free(th);
    pthread_mutex_destroy(&R.mu);
    pthread_cond_destroy(&R.cv);
    int info = 0;
    for (int64_t k = 0; k < nreq; k++) if (status[k] != 0) info = status[k];
    return info;
}

//------------------------------------------------------------------------------
// serialize / deserialize with the reference (GxB_Matrix_serialize,
// Include/GraphBLAS.h:10917; GxB_Matrix_deserialize, :10963), to pin the
// library's blob reader and writer to the reference's own blobs.
//------------------------------------------------------------------------------

// Blob of a CSR matrix (x == NULL: iso-true pattern of type t) stored with
// the given GxB_SPARSITY_CONTROL (1 hyper, 2 sparse, 4 bitmap, 8 full), by
// column when by_col, compressed with `method` (a GxB_COMPRESSION_* value).
// *blob is malloc'ed (the reference's default allocator); ref_blob_free.
int ref_serialize(int t, int64_t nrows, int64_t ncols, const int64_t *p,
                  const int64_t *i, const void *x, int sparsity, bool by_col,
                  int method, void **blob, uint64_t *blob_size)
{
    GrB_Matrix A = NULL;
    GrB_Descriptor D = NULL;
    GrB_Info info;
    GrB_Index size = 0;
    *blob = NULL;
    #define TRY(x) { info = (x); if (info != GrB_SUCCESS) goto done; }
    TRY(make_csr(&A, t, nrows, ncols, p, i, x));
    TRY(GxB_Matrix_Option_set_INT32(A, GxB_FORMAT, by_col ? GxB_BY_COL : GxB_BY_ROW));
    TRY(GxB_Matrix_Option_set_INT32(A, GxB_SPARSITY_CONTROL, sparsity));
    TRY(GrB_Matrix_wait(A, GrB_MATERIALIZE));
    TRY(GrB_Descriptor_new(&D));
    TRY(GxB_Desc_set_INT32(D, GxB_COMPRESSION, method));
    TRY(GxB_Matrix_serialize(blob, &size, A, D));
    *blob_size = (uint64_t)size;
done:
    GrB_Matrix_free(&A);
    GrB_Descriptor_free(&D);
    return (int)info;
    #undef TRY
}

void ref_blob_free(void *blob) { free(blob); }

// A blob read by the reference, returned as CSR by row with sorted rows
// (iso values expanded); *nrows_out / *ncols_out / *type_out describe it.
ref_csr *ref_deserialize(const void *blob, uint64_t blob_size, int64_t *nrows_out,
                         int64_t *ncols_out, int *type_out, int *info_out)
{
    GrB_Matrix C = NULL;
    GrB_Type type = NULL;
    ref_csr *R = NULL;
    GrB_Index nr = 0, nc = 0;
    GrB_Info info;
    #define TRY(x) { info = (x); if (info != GrB_SUCCESS) goto done; }
    TRY(GxB_Matrix_deserialize(&C, NULL, blob, (GrB_Index)blob_size, NULL));
    TRY(GrB_Matrix_nrows(&nr, C));
    TRY(GrB_Matrix_ncols(&nc, C));
    TRY(GxB_Matrix_type(&type, C));
    int code = 0;
    for (int t = 1; t <= 11 && !code; t++)
        if (tsize(t) && type_of(t) == type) code = t;
    if (!code) { info = GrB_DOMAIN_MISMATCH; goto done; }
    TRY(GxB_Matrix_Option_set_INT32(C, GxB_FORMAT, GxB_BY_ROW));
    TRY(GxB_Matrix_Option_set_INT32(C, GxB_SPARSITY_CONTROL, GxB_SPARSE));
    TRY(GrB_Matrix_wait(C, GrB_MATERIALIZE));
    R = calloc(1, sizeof(ref_csr));
    R->nrows = (int64_t)nr; R->type = code;
    GrB_Index psize, isize, xsize;
    bool iso = false;
    TRY(GxB_Matrix_unpack_CSR(C, &R->p, &R->i, &R->x, &psize, &isize, &xsize,
                              &iso, NULL, NULL));
    R->nnz = R->p[nr];
    if (iso && R->nnz > 0)
    {
        size_t ts = tsize(code);
        void *xx = malloc(R->nnz * ts);
        for (int64_t k = 0; k < R->nnz; k++)
            memcpy((char *)xx + k * ts, R->x, ts);
        free(R->x);
        R->x = xx;
    }
    *nrows_out = (int64_t)nr;
    *ncols_out = (int64_t)nc;
    *type_out = code;
done:
    GrB_Matrix_free(&C);
    if (info_out) *info_out = (int)info;
    if (info != GrB_SUCCESS) { ref_free(R); return NULL; }
    return R;
    #undef TRY
}
