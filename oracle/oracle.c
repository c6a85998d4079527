// oracle.c: CPU restatement of SuiteSparse:GraphBLAS v9.3.1 semiring matrix
// multiply, used ONLY as the test checker (tests/, the smoke check and the
// CPU-baseline leg of bench.py).  No product code links or calls it.
//
// It restates, in plain sequential C, the arithmetic that the reference's
// factory kernels perform, in the order they perform it:
//
//  * saxpy3, coarse Gustavson / coarse hash tasks
//    (Source/mxm/template/GB_AxB_saxpy3_coarseGus_noM_phase5.c:52-114 and
//    the _M / _notM / coarseHash variants): for each output vector, scan the
//    entries k of the "row" operand in ascending order, then the entries j of
//    B(k,:) in ascending order; the first product t for (i,j) is written
//    (GB_HX_WRITE, Hx[i] = t), later ones are folded with the monoid's
//    GB_UPDATE (Source/mxm/include/GB_mxm_shared_definitions.h:196-211).
//  * dot3 (Source/mxm/template/GB_AxB_dot_cij.c:516-652): for each mask entry
//    (i,j), merge A(i,:) and B(j,:) in ascending k; the first match does
//    GB_MULT, later ones GB_MULTADD (z = ADD(z, a*b)); a terminal monoid
//    (ANY) stops at the first match.  Entries with no match are zombies and
//    are dropped, as GB_wait does (Source/wait/GB_wait.c:62).
//  * the monoid UPDATE / ADD rules per semiring, e.g.
//    FactoryKernels/GB_AxB__min_plus_fp32.c:19-22 (ADD = fminf, UPDATE skips
//    NaN and keeps z when z <= t), GB_AxB__any_firstj_int64.c:19-22
//    (z = t: the last k wins), GB_AxB__plus_pair_int64.c:19-22.
//  * the mask (Source/mask/GB_mask.c semantics): structural = entry present,
//    valued = present and nonzero after cast to bool; complement inverts.
//  * GB_accum_mask (Source/mask/GB_accum_mask.c:126): Z = accum(C,T) on the
//    union of patterns (or Z = T), then C<M,replace> = Z.
//
// All matrices are sorted, duplicate-free CSR with int64 pointers/indices.
// Operator and type codes are the reference's GB_Opcode / GB_Type_code values
// (Source/builtin/include/GB_opaque.h:28-42, 209-247).

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdbool.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { T_BOOL = 1, T_INT32 = 6, T_UINT32 = 7, T_INT64 = 8, T_UINT64 = 9,
       T_FP32 = 10, T_FP64 = 11 };
enum { OP_FIRST = 72, OP_SECOND = 73, OP_ANY = 74, OP_PAIR = 75, OP_MIN = 76,
       OP_MAX = 77, OP_PLUS = 78, OP_MINUS = 79, OP_RMINUS = 80, OP_TIMES = 81,
       OP_DIV = 82, OP_LOR = 91, OP_LAND = 92, OP_LXOR = 93, OP_EQ = 102,
       OP_FIRSTI = 115, OP_FIRSTI1 = 116, OP_FIRSTJ = 117, OP_FIRSTJ1 = 118,
       OP_SECONDI = 119, OP_SECONDI1 = 120, OP_SECONDJ = 121,
       OP_SECONDJ1 = 122 };

static size_t tsize(int t)
{
    switch (t)
    {
        case T_BOOL: return 1;
        case T_INT32: case T_UINT32: case T_FP32: return 4;
        default: return 8;
    }
}

// A scalar held in the widest form of its type.
typedef union { bool b; int32_t i32; uint32_t u32; int64_t i64; uint64_t u64;
                float f32; double f64; } val_t;

static val_t load(const void *x, int t, int64_t p)
{
    val_t v; memset(&v, 0, sizeof(v));
    switch (t)
    {
        case T_BOOL:   v.b   = ((const bool *)x)[p] ; break;
        case T_INT32:  v.i32 = ((const int32_t *)x)[p] ; break;
        case T_UINT32: v.u32 = ((const uint32_t *)x)[p] ; break;
        case T_INT64:  v.i64 = ((const int64_t *)x)[p] ; break;
        case T_UINT64: v.u64 = ((const uint64_t *)x)[p] ; break;
        case T_FP32:   v.f32 = ((const float *)x)[p] ; break;
        case T_FP64:   v.f64 = ((const double *)x)[p] ; break;
    }
    return v;
}

static void store(void *x, int t, int64_t p, val_t v)
{
    switch (t)
    {
        case T_BOOL:   ((bool *)x)[p]     = v.b ; break;
        case T_INT32:  ((int32_t *)x)[p]  = v.i32 ; break;
        case T_UINT32: ((uint32_t *)x)[p] = v.u32 ; break;
        case T_INT64:  ((int64_t *)x)[p]  = v.i64 ; break;
        case T_UINT64: ((uint64_t *)x)[p] = v.u64 ; break;
        case T_FP32:   ((float *)x)[p]    = v.f32 ; break;
        case T_FP64:   ((double *)x)[p]   = v.f64 ; break;
    }
}

static bool truthy(val_t v, int t)
{
    switch (t)
    {
        case T_BOOL: return v.b;
        case T_INT32: return v.i32 != 0;
        case T_UINT32: return v.u32 != 0;
        case T_INT64: return v.i64 != 0;
        case T_UINT64: return v.u64 != 0;
        case T_FP32: return v.f32 != 0;
        default: return v.f64 != 0;
    }
}

static val_t from_i64(int64_t x, int t)
{
    val_t v; memset(&v, 0, sizeof(v));
    switch (t)
    {
        case T_BOOL: v.b = (x != 0); break;
        case T_INT32: v.i32 = (int32_t)x; break;
        case T_UINT32: v.u32 = (uint32_t)x; break;
        case T_INT64: v.i64 = x; break;
        case T_UINT64: v.u64 = (uint64_t)x; break;
        case T_FP32: v.f32 = (float)x; break;
        default: v.f64 = (double)x; break;
    }
    return v;
}

// Binary operator z = f(x,y) on type t (integer + - * wrap, as the reference
// compiles with -fwrapv).  Positional operators take (i,k,j).
static val_t binop(int op, int t, val_t x, val_t y, int64_t i, int64_t k,
                   int64_t j)
{
    val_t z; memset(&z, 0, sizeof(z));
    switch (op)
    {
        case OP_FIRST: return x;
        case OP_SECOND: return y;
        case OP_PAIR: return from_i64(1, t);
        case OP_FIRSTI: return from_i64(i, t);
        case OP_FIRSTI1: return from_i64(i + 1, t);
        case OP_FIRSTJ: return from_i64(k, t);
        case OP_FIRSTJ1: return from_i64(k + 1, t);
        case OP_SECONDI: return from_i64(k, t);
        case OP_SECONDI1: return from_i64(k + 1, t);
        case OP_SECONDJ: return from_i64(j, t);
        case OP_SECONDJ1: return from_i64(j + 1, t);
        default: break;
    }
    #define ARITH(F, field, ty)                                              \
        switch (op) {                                                        \
        case OP_PLUS:   z.field = (ty)(x.field + y.field); break;            \
        case OP_MINUS:  z.field = (ty)(x.field - y.field); break;            \
        case OP_RMINUS: z.field = (ty)(y.field - x.field); break;            \
        case OP_TIMES:  z.field = (ty)(x.field * y.field); break;            \
        case OP_MIN:    z.field = F##min(x.field, y.field); break;           \
        case OP_MAX:    z.field = F##max(x.field, y.field); break;           \
        case OP_LOR:  z.field = (ty)((x.field != 0) || (y.field != 0)); break;\
        case OP_LAND: z.field = (ty)((x.field != 0) && (y.field != 0)); break;\
        case OP_LXOR: z.field = (ty)((x.field != 0) != (y.field != 0)); break;\
        case OP_EQ:   z.field = (ty)(x.field == y.field); break;             \
        case OP_ANY:  z.field = y.field; break;                              \
        default: break; }
    #define imin(a,b) ((a) < (b) ? (a) : (b))
    #define imax(a,b) ((a) > (b) ? (a) : (b))
    switch (t)
    {
        case T_BOOL:
            switch (op)
            {
                case OP_PLUS: case OP_LOR: case OP_MAX: z.b = x.b || y.b; break;
                case OP_TIMES: case OP_LAND: case OP_MIN: z.b = x.b && y.b; break;
                case OP_LXOR: case OP_MINUS: case OP_RMINUS: z.b = x.b != y.b; break;
                case OP_EQ: z.b = x.b == y.b; break;
                case OP_ANY: z.b = y.b; break;
                default: break;
            }
            break;
        case T_INT32:
        {
            // wrap-around arithmetic through unsigned
            uint32_t a = (uint32_t)x.i32, b = (uint32_t)y.i32;
            switch (op)
            {
                case OP_PLUS: z.i32 = (int32_t)(a + b); break;
                case OP_MINUS: z.i32 = (int32_t)(a - b); break;
                case OP_RMINUS: z.i32 = (int32_t)(b - a); break;
                case OP_TIMES: z.i32 = (int32_t)(a * b); break;
                case OP_MIN: z.i32 = imin(x.i32, y.i32); break;
                case OP_MAX: z.i32 = imax(x.i32, y.i32); break;
                case OP_LOR: z.i32 = (x.i32 != 0) || (y.i32 != 0); break;
                case OP_LAND: z.i32 = (x.i32 != 0) && (y.i32 != 0); break;
                case OP_LXOR: z.i32 = (x.i32 != 0) != (y.i32 != 0); break;
                case OP_EQ: z.i32 = x.i32 == y.i32; break;
                case OP_ANY: z.i32 = y.i32; break;
                default: break;
            }
            break;
        }
        case T_INT64:
        {
            uint64_t a = (uint64_t)x.i64, b = (uint64_t)y.i64;
            switch (op)
            {
                case OP_PLUS: z.i64 = (int64_t)(a + b); break;
                case OP_MINUS: z.i64 = (int64_t)(a - b); break;
                case OP_RMINUS: z.i64 = (int64_t)(b - a); break;
                case OP_TIMES: z.i64 = (int64_t)(a * b); break;
                case OP_MIN: z.i64 = imin(x.i64, y.i64); break;
                case OP_MAX: z.i64 = imax(x.i64, y.i64); break;
                case OP_LOR: z.i64 = (x.i64 != 0) || (y.i64 != 0); break;
                case OP_LAND: z.i64 = (x.i64 != 0) && (y.i64 != 0); break;
                case OP_LXOR: z.i64 = (x.i64 != 0) != (y.i64 != 0); break;
                case OP_EQ: z.i64 = x.i64 == y.i64; break;
                case OP_ANY: z.i64 = y.i64; break;
                default: break;
            }
            break;
        }
        case T_UINT32:
            switch (op)
            {
                case OP_PLUS: z.u32 = x.u32 + y.u32; break;
                case OP_MINUS: z.u32 = x.u32 - y.u32; break;
                case OP_RMINUS: z.u32 = y.u32 - x.u32; break;
                case OP_TIMES: z.u32 = x.u32 * y.u32; break;
                case OP_MIN: z.u32 = imin(x.u32, y.u32); break;
                case OP_MAX: z.u32 = imax(x.u32, y.u32); break;
                case OP_LOR: z.u32 = (x.u32 != 0) || (y.u32 != 0); break;
                case OP_LAND: z.u32 = (x.u32 != 0) && (y.u32 != 0); break;
                case OP_LXOR: z.u32 = (x.u32 != 0) != (y.u32 != 0); break;
                case OP_EQ: z.u32 = x.u32 == y.u32; break;
                case OP_ANY: z.u32 = y.u32; break;
                default: break;
            }
            break;
        case T_UINT64:
            switch (op)
            {
                case OP_PLUS: z.u64 = x.u64 + y.u64; break;
                case OP_MINUS: z.u64 = x.u64 - y.u64; break;
                case OP_RMINUS: z.u64 = y.u64 - x.u64; break;
                case OP_TIMES: z.u64 = x.u64 * y.u64; break;
                case OP_MIN: z.u64 = imin(x.u64, y.u64); break;
                case OP_MAX: z.u64 = imax(x.u64, y.u64); break;
                case OP_LOR: z.u64 = (x.u64 != 0) || (y.u64 != 0); break;
                case OP_LAND: z.u64 = (x.u64 != 0) && (y.u64 != 0); break;
                case OP_LXOR: z.u64 = (x.u64 != 0) != (y.u64 != 0); break;
                case OP_EQ: z.u64 = x.u64 == y.u64; break;
                case OP_ANY: z.u64 = y.u64; break;
                default: break;
            }
            break;
        case T_FP32:
            switch (op)
            {
                case OP_PLUS: z.f32 = x.f32 + y.f32; break;
                case OP_MINUS: z.f32 = x.f32 - y.f32; break;
                case OP_RMINUS: z.f32 = y.f32 - x.f32; break;
                case OP_TIMES: z.f32 = x.f32 * y.f32; break;
                case OP_DIV: z.f32 = x.f32 / y.f32; break;
                case OP_MIN: z.f32 = fminf(x.f32, y.f32); break;
                case OP_MAX: z.f32 = fmaxf(x.f32, y.f32); break;
                case OP_LOR: z.f32 = (x.f32 != 0) || (y.f32 != 0); break;
                case OP_LAND: z.f32 = (x.f32 != 0) && (y.f32 != 0); break;
                case OP_LXOR: z.f32 = (x.f32 != 0) != (y.f32 != 0); break;
                case OP_EQ: z.f32 = x.f32 == y.f32; break;
                case OP_ANY: z.f32 = y.f32; break;
                default: break;
            }
            break;
        case T_FP64:
            switch (op)
            {
                case OP_PLUS: z.f64 = x.f64 + y.f64; break;
                case OP_MINUS: z.f64 = x.f64 - y.f64; break;
                case OP_RMINUS: z.f64 = y.f64 - x.f64; break;
                case OP_TIMES: z.f64 = x.f64 * y.f64; break;
                case OP_DIV: z.f64 = x.f64 / y.f64; break;
                case OP_MIN: z.f64 = fmin(x.f64, y.f64); break;
                case OP_MAX: z.f64 = fmax(x.f64, y.f64); break;
                case OP_LOR: z.f64 = (x.f64 != 0) || (y.f64 != 0); break;
                case OP_LAND: z.f64 = (x.f64 != 0) && (y.f64 != 0); break;
                case OP_LXOR: z.f64 = (x.f64 != 0) != (y.f64 != 0); break;
                case OP_EQ: z.f64 = x.f64 == y.f64; break;
                case OP_ANY: z.f64 = y.f64; break;
                default: break;
            }
            break;
    }
    #undef ARITH
    return z;
}

// saxpy3 coarse-task update z = UPDATE(z, t)
// (GB_UPDATE of FactoryKernels/GB_AxB__<add>_<mult>_<type>.c).  For MIN/MAX on
// floating point the update skips a NaN t and keeps z unless t is strictly
// better or z is NaN; for ANY it is z = t.
static val_t monoid_update(int add, int t, val_t z, val_t tv)
{
    if (t == T_FP32 && (add == OP_MIN || add == OP_MAX))
    {
        float a = z.f32, b = tv.f32;
        if (!isnan(b) && !(add == OP_MIN ? islessequal(a, b) : isgreaterequal(a, b)))
            z.f32 = b;
        return z;
    }
    if (t == T_FP64 && (add == OP_MIN || add == OP_MAX))
    {
        double a = z.f64, b = tv.f64;
        if (!isnan(b) && !(add == OP_MIN ? islessequal(a, b) : isgreaterequal(a, b)))
            z.f64 = b;
        return z;
    }
    if (add == OP_ANY) return tv;
    return binop(add, t, z, tv, 0, 0, 0);
}

// dot-product fold z = ADD(z, t): the monoid's binary operator (fminf/fmaxf
// for floating MIN/MAX, GB_AxB__min_plus_fp32.c:21)
static val_t monoid_add(int add, int t, val_t z, val_t tv)
{
    return binop(add, t, z, tv, 0, 0, 0);
}

static bool mask_allows(const int64_t *Mp, const int64_t *Mi, const void *Mx,
                        int mtype, bool structural, bool comp, int64_t i,
                        int64_t j)
{
    bool present = false;
    if (Mp)
    {
        int64_t lo = Mp[i], hi = Mp[i + 1] - 1;
        while (lo <= hi)
        {
            int64_t mid = lo + (hi - lo) / 2;
            if (Mi[mid] == j)
            {
                present = structural || Mx == NULL ||
                          truthy(load(Mx, mtype, mid), mtype);
                break;
            }
            if (Mi[mid] < j) lo = mid + 1; else hi = mid - 1;
        }
    }
    else
    {
        present = false;     // no mask given: complement of empty = all
        return comp ? true : true;
    }
    return comp ? !present : present;
}

//------------------------------------------------------------------------------
// result holder
//------------------------------------------------------------------------------

typedef struct
{
    int64_t nrows, ncols, nnz;
    int type;
    int64_t *p, *i;
    void *x;
} oracle_csr;

void oracle_free(oracle_csr *C)
{
    if (!C) return;
    free(C->p); free(C->i); free(C->x); free(C);
}

int64_t oracle_nnz(const oracle_csr *C) { return C->nnz; }

void oracle_export(const oracle_csr *C, int64_t *p, int64_t *i, void *x)
{
    memcpy(p, C->p, (size_t)(C->nrows + 1) * sizeof(int64_t));
    memcpy(i, C->i, (size_t)C->nnz * sizeof(int64_t));
    if (x) memcpy(x, C->x, (size_t)C->nnz * tsize(C->type));
}

static int cmp_i64(const void *a, const void *b)
{
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

//------------------------------------------------------------------------------
// saxpy: C<M> = A*B row by row (coarse Gustavson, k ascending)
//------------------------------------------------------------------------------

// A: m-by-n, B: n-by-ncols.  Ax/Bx may be NULL for pattern-only operands
// (PAIR or positional multiplier).  Mp == NULL means no mask (mask_comp is then
// ignored).  ctype is the semiring's output type.
oracle_csr *oracle_saxpy(int64_t m, int64_t ncols,
    const int64_t *Ap, const int64_t *Ai, const void *Ax, int atype,
    const int64_t *Bp, const int64_t *Bi, const void *Bx, int btype,
    const int64_t *Mp, const int64_t *Mi, const void *Mx, int mtype,
    bool mask_struct, bool mask_comp, int add, int mult, int ctype)
{
    oracle_csr *C = (oracle_csr *)calloc(1, sizeof(oracle_csr));
    C->nrows = m; C->ncols = ncols; C->type = ctype;
    C->p = (int64_t *)calloc((size_t)m + 1, sizeof(int64_t));
    int64_t **rows_i = (int64_t **)calloc((size_t)m, sizeof(int64_t *));
    char **rows_x = (char **)calloc((size_t)m, sizeof(char *));
    const size_t cs = tsize(ctype);
    #pragma omp parallel
    {
        val_t *H = (val_t *)malloc((size_t)ncols * sizeof(val_t));
        char *Hf = (char *)calloc((size_t)ncols, 1);
        int64_t *pat = (int64_t *)malloc((size_t)ncols * sizeof(int64_t));
        #pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < m; i++)
        {
            int64_t cnt = 0;
            for (int64_t pa = Ap[i]; pa < Ap[i + 1]; pa++)
            {
                int64_t k = Ai[pa];
                val_t a = Ax ? load(Ax, atype, pa) : from_i64(0, ctype);
                for (int64_t pb = Bp[k]; pb < Bp[k + 1]; pb++)
                {
                    int64_t j = Bi[pb];
                    if (Mp && !mask_allows(Mp, Mi, Mx, mtype, mask_struct,
                                           mask_comp, i, j))
                        continue;
                    val_t b = Bx ? load(Bx, btype, pb) : from_i64(0, ctype);
                    val_t t = binop(mult, ctype, a, b, i, k, j);
                    if (!Hf[j]) { Hf[j] = 1; H[j] = t; pat[cnt++] = j; }
                    else H[j] = monoid_update(add, ctype, H[j], t);
                }
            }
            qsort(pat, (size_t)cnt, sizeof(int64_t), cmp_i64);
            rows_i[i] = (int64_t *)malloc((size_t)(cnt ? cnt : 1) * sizeof(int64_t));
            rows_x[i] = (char *)malloc((size_t)(cnt ? cnt : 1) * cs);
            for (int64_t t = 0; t < cnt; t++)
            {
                int64_t j = pat[t];
                rows_i[i][t] = j;
                store(rows_x[i], ctype, t, H[j]);
                Hf[j] = 0;
            }
            C->p[i + 1] = cnt;
        }
        free(H); free(Hf); free(pat);
    }
    for (int64_t i = 0; i < m; i++) C->p[i + 1] += C->p[i];
    C->nnz = C->p[m];
    C->i = (int64_t *)malloc((size_t)(C->nnz ? C->nnz : 1) * sizeof(int64_t));
    C->x = malloc((size_t)(C->nnz ? C->nnz : 1) * cs);
    for (int64_t i = 0; i < m; i++)
    {
        int64_t n = C->p[i + 1] - C->p[i];
        memcpy(C->i + C->p[i], rows_i[i], (size_t)n * sizeof(int64_t));
        memcpy((char *)C->x + C->p[i] * cs, rows_x[i], (size_t)n * cs);
        free(rows_i[i]); free(rows_x[i]);
    }
    free(rows_i); free(rows_x);
    return C;
}

//------------------------------------------------------------------------------
// dot3: C<M> = A*B' (C(i,j) = A(i,:) . B(j,:) for (i,j) in M), zombies dropped
//------------------------------------------------------------------------------

oracle_csr *oracle_dot3(int64_t m, int64_t ncols,
    const int64_t *Ap, const int64_t *Ai, const void *Ax, int atype,
    const int64_t *Bp, const int64_t *Bi, const void *Bx, int btype,
    const int64_t *Mp, const int64_t *Mi, const void *Mx, int mtype,
    bool mask_struct, int add, int mult, int ctype)
{
    oracle_csr *C = (oracle_csr *)calloc(1, sizeof(oracle_csr));
    C->nrows = m; C->ncols = ncols; C->type = ctype;
    const size_t cs = tsize(ctype);
    const int64_t mnz = Mp[m];
    C->p = (int64_t *)calloc((size_t)m + 1, sizeof(int64_t));
    int64_t *Ci = (int64_t *)malloc((size_t)(mnz ? mnz : 1) * sizeof(int64_t));
    char *Cx = (char *)malloc((size_t)(mnz ? mnz : 1) * cs);
    char *live = (char *)calloc((size_t)(mnz ? mnz : 1), 1);
    const bool terminal_any = (add == OP_ANY);
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < m; i++)
    {
        for (int64_t pm = Mp[i]; pm < Mp[i + 1]; pm++)
        {
            int64_t j = Mi[pm];
            if (!mask_struct && Mx && !truthy(load(Mx, mtype, pm), mtype))
                continue;   // valued mask entry that is false: zombie
            int64_t pa = Ap[i], pa_end = Ap[i + 1];
            int64_t pb = Bp[j], pb_end = Bp[j + 1];
            bool exists = false;
            val_t cij; memset(&cij, 0, sizeof(cij));
            while (pa < pa_end && pb < pb_end)
            {
                int64_t ka = Ai[pa], kb = Bi[pb];
                if (ka < kb) pa++;
                else if (kb < ka) pb++;
                else
                {
                    val_t a = Ax ? load(Ax, atype, pa) : from_i64(0, ctype);
                    val_t b = Bx ? load(Bx, btype, pb) : from_i64(0, ctype);
                    val_t t = binop(mult, ctype, a, b, i, ka, j);
                    if (!exists) { cij = t; exists = true; }
                    else cij = monoid_add(add, ctype, cij, t);
                    if (terminal_any) break;
                    pa++; pb++;
                }
            }
            if (exists)
            {
                Ci[pm] = j;
                store(Cx, ctype, pm, cij);
                live[pm] = 1;
            }
        }
    }
    // drop zombies (GB_wait)
    int64_t w = 0;
    for (int64_t i = 0; i < m; i++)
    {
        for (int64_t pm = Mp[i]; pm < Mp[i + 1]; pm++)
        {
            if (!live[pm]) continue;
            Ci[w] = Ci[pm];
            memmove(Cx + w * cs, Cx + pm * cs, cs);
            w++;
        }
        C->p[i + 1] = w;
    }
    C->nnz = w;
    C->i = Ci; C->x = Cx;
    free(live);
    return C;
}

//------------------------------------------------------------------------------
// triangle count: sum over (i,j) in L of |L(i,:) & U(j,:)| (plus_pair dot3)
//------------------------------------------------------------------------------

int64_t oracle_tricount(int64_t n, const int64_t *Lp, const int64_t *Li,
                        const int64_t *Up, const int64_t *Ui)
{
    int64_t total = 0;
    #pragma omp parallel for schedule(dynamic, 256) reduction(+:total)
    for (int64_t i = 0; i < n; i++)
    {
        for (int64_t pm = Lp[i]; pm < Lp[i + 1]; pm++)
        {
            int64_t j = Li[pm];
            int64_t pa = Lp[i], pa_end = Lp[i + 1];
            int64_t pb = Up[j], pb_end = Up[j + 1];
            while (pa < pa_end && pb < pb_end)
            {
                int64_t a = Li[pa], b = Ui[pb];
                if (a < b) pa++;
                else if (b < a) pb++;
                else { total++; pa++; pb++; }
            }
        }
    }
    return total;
}

//------------------------------------------------------------------------------
// accumulate + mask write-back: C<M,replace> = accum (C, T)
//------------------------------------------------------------------------------

// accum == 0 means no accumulator (Z = T).  Mp == NULL means no mask.
oracle_csr *oracle_accum_mask(int64_t m, int64_t ncols,
    const int64_t *Cp, const int64_t *Ci, const void *Cx,
    const int64_t *Tp, const int64_t *Ti, const void *Tx,
    const int64_t *Mp, const int64_t *Mi, const void *Mx, int mtype,
    bool mask_struct, bool mask_comp, bool replace, int accum, int ctype)
{
    oracle_csr *R = (oracle_csr *)calloc(1, sizeof(oracle_csr));
    R->nrows = m; R->ncols = ncols; R->type = ctype;
    const size_t cs = tsize(ctype);
    int64_t cap = Cp[m] + Tp[m] + 1;
    R->p = (int64_t *)calloc((size_t)m + 1, sizeof(int64_t));
    R->i = (int64_t *)malloc((size_t)cap * sizeof(int64_t));
    R->x = malloc((size_t)cap * cs);
    int64_t w = 0;
    for (int64_t i = 0; i < m; i++)
    {
        int64_t pc = Cp[i], pc_end = Cp[i + 1], pt = Tp[i], pt_end = Tp[i + 1];
        while (pc < pc_end || pt < pt_end)
        {
            int64_t jc = pc < pc_end ? Ci[pc] : INT64_MAX;
            int64_t jt = pt < pt_end ? Ti[pt] : INT64_MAX;
            int64_t j = jc < jt ? jc : jt;
            bool has_c = (jc == j), has_t = (jt == j);
            val_t c = has_c ? load(Cx, ctype, pc) : from_i64(0, ctype);
            val_t t = has_t ? load(Tx, ctype, pt) : from_i64(0, ctype);
            if (has_c) pc++;
            if (has_t) pt++;
            // Z(i,j)
            bool has_z; val_t z;
            if (accum)
            {
                has_z = has_c || has_t;
                z = (has_c && has_t) ? binop(accum, ctype, c, t, i, j, j)
                                     : (has_c ? c : t);
            }
            else { has_z = has_t; z = t; }
            bool allow = Mp ? mask_allows(Mp, Mi, Mx, mtype, mask_struct,
                                          mask_comp, i, j)
                            : true;
            if (allow)
            {
                if (has_z) { R->i[w] = j; store(R->x, ctype, w, z); w++; }
            }
            else if (!replace && has_c)
            {
                R->i[w] = j; store(R->x, ctype, w, c); w++;
            }
        }
        R->p[i + 1] = w;
    }
    R->nnz = w;
    return R;
}

//------------------------------------------------------------------------------
// BFS parents: loop of q<!p,struct,replace> = q any_secondi S, p<q> = q
//------------------------------------------------------------------------------

// parent[v] = -1 when unreached; level[v] likewise.  The ANY monoid keeps the
// last contribution in ascending k (coarse-task z = t), so parent(j) is the
// largest frontier vertex adjacent to j.  Returns the number of levels.
int oracle_bfs(int64_t n, const int64_t *Sp, const int64_t *Si, int64_t src,
               int64_t *parent, int64_t *level)
{
    for (int64_t v = 0; v < n; v++) { parent[v] = -1; level[v] = -1; }
    int64_t *q = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    int64_t *nq = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    int64_t *cand = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    for (int64_t v = 0; v < n; v++) cand[v] = -1;
    int64_t nqn = 1;
    q[0] = src; parent[src] = src; level[src] = 0;
    int lev = 0;
    while (nqn > 0)
    {
        lev++;
        // frontier q is sorted ascending; scanning it in order and overwriting
        // leaves the largest k in cand[j]
        for (int64_t t = 0; t < nqn; t++)
        {
            int64_t k = q[t];
            for (int64_t p = Sp[k]; p < Sp[k + 1]; p++)
            {
                int64_t j = Si[p];
                if (parent[j] >= 0) continue;     // complemented mask
                cand[j] = k;
            }
        }
        int64_t m = 0;
        for (int64_t j = 0; j < n; j++)
        {
            if (cand[j] >= 0)
            {
                parent[j] = cand[j]; level[j] = lev; nq[m++] = j; cand[j] = -1;
            }
        }
        int64_t *tmp = q; q = nq; nq = tmp;
        nqn = m;
    }
    free(q); free(nq); free(cand);
    return lev;
}
