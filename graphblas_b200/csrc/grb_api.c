// grb_api.c: the GraphBLAS C API for the multiply path (include/
// GraphBLAS_b200.h), written in C over the device-resident C-ABI of
// libgrb_b200.so (include/grb_b200.h).
//
// This is the layer the reference implements in Source/mxm/GrB_mxm.c:18,
// GrB_vxm.c:19, GrB_mxv.c:18 (argument checks, descriptor decoding), GB_mxm.c:24
// (dimension and domain checks, transplant or GB_accum_mask) and
// GB_AxB_meta.c:41 (method choice).  The method choice here:
//   * C<M> = A*B' with a plain (not complemented) mask, or any mask-driven
//     product the descriptor asks to compute by dot products
//     (GxB_AxB_METHOD = GxB_AxB_DOT): masked dot3 over M's pattern
//     (as GB_AxB_meta_adotb_control / GB_AxB_dot3_control pick dot3);
//   * everything else: row-wise saxpy3, with M or !M applied inside;
//   * A' or B' operands the kernels cannot read directly are transposed on
//     the device first (GB_transpose_cast).
// The result T is moved into C when no accumulator and no leftover mask work
// remain (GB_transplant_conform, GB_mxm.c:193); otherwise the device
// accumulate/mask kernel writes C<M,replace> = accum(C,T) (GB_accum_mask,
// GB_mxm.c:206).
//
// Matrices keep a host copy (int64 CSR, the reference's layout) and a device
// copy; operations run on the device copy and invalidate the host copy, which
// is rebuilt on demand (wait, extractTuples, unpack).

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdbool.h>
#include "GraphBLAS_b200.h"
#include "grb_b200.h"

#define MAGIC 0x72eeb200ULL
#define FREED 0xdeadb200ULL

//------------------------------------------------------------------------------
// objects
//------------------------------------------------------------------------------

struct GB_Type_opaque { int code; size_t size; };
struct GB_BinaryOp_opaque { int opcode; GrB_Type type; };
struct GB_Monoid_opaque { int opcode; GrB_Type type; };
struct GB_Semiring_opaque { int add, mult; GrB_Type type; bool user; };
struct GB_Descriptor_opaque { int outp, mask, inp0, inp1, method; bool user; };

struct GB_Matrix_opaque
{
    uint64_t magic;
    GrB_Type type;
    int64_t nrows, ncols;
    bool host_ok;               // host copy below is current
    int64_t *hp, *hi;
    void *hx;
    bool hiso;
    bool dev_ok;                // device copy is current
    grb_b200_dmatrix dev;
};

struct GB_Vector_opaque { struct GB_Matrix_opaque m; };   // a 1-by-n row

static struct GB_Type_opaque T_BOOL_ = {1, 1}, T_INT32_ = {6, 4},
    T_UINT32_ = {7, 4}, T_INT64_ = {8, 8}, T_UINT64_ = {9, 8},
    T_FP32_ = {10, 4}, T_FP64_ = {11, 8};
GrB_Type GrB_BOOL = &T_BOOL_, GrB_INT32 = &T_INT32_, GrB_UINT32 = &T_UINT32_,
    GrB_INT64 = &T_INT64_, GrB_UINT64 = &T_UINT64_, GrB_FP32 = &T_FP32_,
    GrB_FP64 = &T_FP64_;

enum { OP_FIRST = 72, OP_SECOND = 73, OP_ANY = 74, OP_PAIR = 75, OP_MIN = 76,
       OP_MAX = 77, OP_PLUS = 78, OP_MINUS = 79, OP_RMINUS = 80, OP_TIMES = 81,
       OP_LOR = 91, OP_LAND = 92, OP_LXOR = 93, OP_FIRSTI = 115,
       OP_FIRSTJ = 117, OP_SECONDI = 119, OP_SECONDJ = 121 };

#define DEF_OP(NAME, OPC, TP) \
    static struct GB_BinaryOp_opaque NAME##_ = {OPC, &TP}; \
    GrB_BinaryOp NAME = &NAME##_;
#define DEF_OPS_OF(T, TP) \
    DEF_OP(GrB_FIRST_##T, OP_FIRST, TP) DEF_OP(GrB_SECOND_##T, OP_SECOND, TP) \
    DEF_OP(GrB_PLUS_##T, OP_PLUS, TP) DEF_OP(GrB_MINUS_##T, OP_MINUS, TP) \
    DEF_OP(GrB_TIMES_##T, OP_TIMES, TP) DEF_OP(GrB_MIN_##T, OP_MIN, TP) \
    DEF_OP(GrB_MAX_##T, OP_MAX, TP) DEF_OP(GxB_PAIR_##T, OP_PAIR, TP) \
    DEF_OP(GxB_ANY_##T, OP_ANY, TP)
DEF_OPS_OF(BOOL, T_BOOL_)
DEF_OPS_OF(INT32, T_INT32_)
DEF_OPS_OF(INT64, T_INT64_)
DEF_OPS_OF(FP32, T_FP32_)
DEF_OPS_OF(FP64, T_FP64_)
DEF_OP(GrB_LOR, OP_LOR, T_BOOL_)
DEF_OP(GrB_LAND, OP_LAND, T_BOOL_)
DEF_OP(GrB_LXOR, OP_LXOR, T_BOOL_)
DEF_OP(GxB_FIRSTI_INT32, OP_FIRSTI, T_INT32_)
DEF_OP(GxB_FIRSTI_INT64, OP_FIRSTI, T_INT64_)
DEF_OP(GxB_FIRSTJ_INT32, OP_FIRSTJ, T_INT32_)
DEF_OP(GxB_FIRSTJ_INT64, OP_FIRSTJ, T_INT64_)
DEF_OP(GxB_SECONDI_INT32, OP_SECONDI, T_INT32_)
DEF_OP(GxB_SECONDI_INT64, OP_SECONDI, T_INT64_)
DEF_OP(GxB_SECONDJ_INT32, OP_SECONDJ, T_INT32_)
DEF_OP(GxB_SECONDJ_INT64, OP_SECONDJ, T_INT64_)

#define DEF_MON(NAME, OPC, TP) \
    static struct GB_Monoid_opaque NAME##_ = {OPC, &TP}; \
    GrB_Monoid NAME = &NAME##_;
#define DEF_MONS_OF(T, TP) \
    DEF_MON(GrB_PLUS_MONOID_##T, OP_PLUS, TP) \
    DEF_MON(GrB_TIMES_MONOID_##T, OP_TIMES, TP) \
    DEF_MON(GrB_MIN_MONOID_##T, OP_MIN, TP) \
    DEF_MON(GrB_MAX_MONOID_##T, OP_MAX, TP) \
    DEF_MON(GxB_ANY_##T##_MONOID, OP_ANY, TP)
DEF_MONS_OF(INT32, T_INT32_)
DEF_MONS_OF(INT64, T_INT64_)
DEF_MONS_OF(FP32, T_FP32_)
DEF_MONS_OF(FP64, T_FP64_)
DEF_MON(GrB_LOR_MONOID_BOOL, OP_LOR, T_BOOL_)
DEF_MON(GrB_LAND_MONOID_BOOL, OP_LAND, T_BOOL_)
DEF_MON(GxB_ANY_BOOL_MONOID, OP_ANY, T_BOOL_)

#define DEF_SR(NAME, ADD, MULT, TP) \
    static struct GB_Semiring_opaque NAME##_ = {ADD, MULT, &TP, false}; \
    GrB_Semiring NAME = &NAME##_;
DEF_SR(GrB_PLUS_TIMES_SEMIRING_FP64, OP_PLUS, OP_TIMES, T_FP64_)
DEF_SR(GrB_PLUS_TIMES_SEMIRING_FP32, OP_PLUS, OP_TIMES, T_FP32_)
DEF_SR(GrB_PLUS_TIMES_SEMIRING_INT64, OP_PLUS, OP_TIMES, T_INT64_)
DEF_SR(GrB_PLUS_TIMES_SEMIRING_INT32, OP_PLUS, OP_TIMES, T_INT32_)
DEF_SR(GxB_PLUS_PAIR_INT64, OP_PLUS, OP_PAIR, T_INT64_)
DEF_SR(GxB_PLUS_PAIR_INT32, OP_PLUS, OP_PAIR, T_INT32_)
DEF_SR(GxB_PLUS_PAIR_FP64, OP_PLUS, OP_PAIR, T_FP64_)
DEF_SR(GrB_MIN_PLUS_SEMIRING_FP32, OP_MIN, OP_PLUS, T_FP32_)
DEF_SR(GrB_MIN_PLUS_SEMIRING_FP64, OP_MIN, OP_PLUS, T_FP64_)
DEF_SR(GrB_MIN_PLUS_SEMIRING_INT64, OP_MIN, OP_PLUS, T_INT64_)
DEF_SR(GrB_MIN_PLUS_SEMIRING_INT32, OP_MIN, OP_PLUS, T_INT32_)
DEF_SR(GrB_MAX_PLUS_SEMIRING_FP64, OP_MAX, OP_PLUS, T_FP64_)
DEF_SR(GrB_MAX_PLUS_SEMIRING_FP32, OP_MAX, OP_PLUS, T_FP32_)
DEF_SR(GrB_MIN_TIMES_SEMIRING_FP64, OP_MIN, OP_TIMES, T_FP64_)
DEF_SR(GrB_MAX_TIMES_SEMIRING_FP64, OP_MAX, OP_TIMES, T_FP64_)
DEF_SR(GrB_MIN_SECOND_SEMIRING_FP32, OP_MIN, OP_SECOND, T_FP32_)
DEF_SR(GrB_MIN_SECOND_SEMIRING_FP64, OP_MIN, OP_SECOND, T_FP64_)
DEF_SR(GrB_MIN_FIRST_SEMIRING_FP32, OP_MIN, OP_FIRST, T_FP32_)
DEF_SR(GrB_MIN_FIRST_SEMIRING_FP64, OP_MIN, OP_FIRST, T_FP64_)
DEF_SR(GxB_PLUS_FIRST_FP64, OP_PLUS, OP_FIRST, T_FP64_)
DEF_SR(GxB_PLUS_SECOND_FP64, OP_PLUS, OP_SECOND, T_FP64_)
DEF_SR(GxB_ANY_SECONDI_INT64, OP_ANY, OP_SECONDI, T_INT64_)
DEF_SR(GxB_ANY_FIRSTJ_INT64, OP_ANY, OP_FIRSTJ, T_INT64_)
DEF_SR(GxB_ANY_FIRSTI_INT64, OP_ANY, OP_FIRSTI, T_INT64_)
DEF_SR(GxB_ANY_SECONDJ_INT64, OP_ANY, OP_SECONDJ, T_INT64_)
DEF_SR(GxB_ANY_SECONDI_INT32, OP_ANY, OP_SECONDI, T_INT32_)
DEF_SR(GxB_ANY_FIRSTJ_INT32, OP_ANY, OP_FIRSTJ, T_INT32_)
DEF_SR(GxB_MIN_SECONDI_INT64, OP_MIN, OP_SECONDI, T_INT64_)
DEF_SR(GxB_MIN_FIRSTJ_INT64, OP_MIN, OP_FIRSTJ, T_INT64_)
DEF_SR(GxB_MIN_FIRSTI_INT64, OP_MIN, OP_FIRSTI, T_INT64_)
DEF_SR(GxB_MIN_SECONDJ_INT64, OP_MIN, OP_SECONDJ, T_INT64_)
DEF_SR(GxB_MAX_SECONDI_INT64, OP_MAX, OP_SECONDI, T_INT64_)
DEF_SR(GxB_MAX_FIRSTJ_INT64, OP_MAX, OP_FIRSTJ, T_INT64_)
DEF_SR(GxB_ANY_PAIR_BOOL, OP_ANY, OP_PAIR, T_BOOL_)
DEF_SR(GrB_LOR_LAND_SEMIRING_BOOL, OP_LOR, OP_LAND, T_BOOL_)
DEF_SR(GxB_ANY_PAIR_INT64, OP_ANY, OP_PAIR, T_INT64_)
DEF_SR(GxB_ANY_TIMES_FP64, OP_ANY, OP_TIMES, T_FP64_)

#define DEF_DESC(NAME, O, M, I0, I1) \
    static struct GB_Descriptor_opaque NAME##_ = {O, M, I0, I1, 0, false}; \
    GrB_Descriptor NAME = &NAME##_;
#define R GrB_REPLACE
#define S GrB_STRUCTURE
#define CM GrB_COMP
#define SC GrB_COMP_STRUCTURE
#define TR GrB_TRAN
DEF_DESC(GrB_DESC_T1, 0, 0, 0, TR)
DEF_DESC(GrB_DESC_T0, 0, 0, TR, 0)
DEF_DESC(GrB_DESC_T0T1, 0, 0, TR, TR)
DEF_DESC(GrB_DESC_C, 0, CM, 0, 0)
DEF_DESC(GrB_DESC_CT1, 0, CM, 0, TR)
DEF_DESC(GrB_DESC_CT0, 0, CM, TR, 0)
DEF_DESC(GrB_DESC_CT0T1, 0, CM, TR, TR)
DEF_DESC(GrB_DESC_S, 0, S, 0, 0)
DEF_DESC(GrB_DESC_ST1, 0, S, 0, TR)
DEF_DESC(GrB_DESC_ST0, 0, S, TR, 0)
DEF_DESC(GrB_DESC_ST0T1, 0, S, TR, TR)
DEF_DESC(GrB_DESC_SC, 0, SC, 0, 0)
DEF_DESC(GrB_DESC_SCT1, 0, SC, 0, TR)
DEF_DESC(GrB_DESC_SCT0, 0, SC, TR, 0)
DEF_DESC(GrB_DESC_SCT0T1, 0, SC, TR, TR)
DEF_DESC(GrB_DESC_R, R, 0, 0, 0)
DEF_DESC(GrB_DESC_RT1, R, 0, 0, TR)
DEF_DESC(GrB_DESC_RT0, R, 0, TR, 0)
DEF_DESC(GrB_DESC_RT0T1, R, 0, TR, TR)
DEF_DESC(GrB_DESC_RC, R, CM, 0, 0)
DEF_DESC(GrB_DESC_RCT1, R, CM, 0, TR)
DEF_DESC(GrB_DESC_RCT0, R, CM, TR, 0)
DEF_DESC(GrB_DESC_RCT0T1, R, CM, TR, TR)
DEF_DESC(GrB_DESC_RS, R, S, 0, 0)
DEF_DESC(GrB_DESC_RST1, R, S, 0, TR)
DEF_DESC(GrB_DESC_RST0, R, S, TR, 0)
DEF_DESC(GrB_DESC_RST0T1, R, S, TR, TR)
DEF_DESC(GrB_DESC_RSC, R, SC, 0, 0)
DEF_DESC(GrB_DESC_RSCT1, R, SC, 0, TR)
DEF_DESC(GrB_DESC_RSCT0, R, SC, TR, 0)
DEF_DESC(GrB_DESC_RSCT0T1, R, SC, TR, TR)
#undef R
#undef S
#undef CM
#undef SC
#undef TR

static const GrB_Index all_marker = 0;
const GrB_Index *GrB_ALL = &all_marker;

//------------------------------------------------------------------------------
// context
//------------------------------------------------------------------------------

static bool g_init = false;

GrB_Info GrB_init(GrB_Mode mode)
{
    if (mode != GrB_NONBLOCKING && mode != GrB_BLOCKING) return GrB_INVALID_VALUE;
    if (g_init) return GrB_INVALID_VALUE;          // as the reference: once only
    int info = grb_b200_init();
    if (info != 0) return (GrB_Info)info;
    g_init = true;
    return GrB_SUCCESS;
}

GrB_Info GrB_finalize(void)
{
    if (g_init) grb_b200_finalize();
    g_init = false;
    return GrB_SUCCESS;
}

#define CHECK_INIT if (!g_init) return GrB_PANIC
#define CHECK(x) { GrB_Info info_ = (GrB_Info)(x); if (info_ != GrB_SUCCESS) return info_; }
#define OBJ_OK(A) ((A) != NULL && (A)->magic == MAGIC)

//------------------------------------------------------------------------------
// semirings and descriptors
//------------------------------------------------------------------------------

GrB_Info GrB_Semiring_new(GrB_Semiring *semiring, GrB_Monoid add,
                          GrB_BinaryOp multiply)
{
    if (!semiring || !add || !multiply) return GrB_NULL_POINTER;
    struct GB_Semiring_opaque *s = calloc(1, sizeof(*s));
    if (!s) return GrB_OUT_OF_MEMORY;
    s->add = add->opcode;
    s->mult = multiply->opcode;
    s->type = add->type;
    s->user = true;
    *semiring = s;
    return GrB_SUCCESS;
}

GrB_Info GrB_Semiring_free(GrB_Semiring *semiring)
{
    if (semiring && *semiring && (*semiring)->user) free(*semiring);
    if (semiring) *semiring = NULL;
    return GrB_SUCCESS;
}

GrB_Info GrB_Descriptor_new(GrB_Descriptor *desc)
{
    if (!desc) return GrB_NULL_POINTER;
    struct GB_Descriptor_opaque *d = calloc(1, sizeof(*d));
    if (!d) return GrB_OUT_OF_MEMORY;
    d->user = true;
    *desc = d;
    return GrB_SUCCESS;
}

GrB_Info GrB_Descriptor_set(GrB_Descriptor d, GrB_Desc_Field field,
                            GrB_Desc_Value val)
{
    if (!d) return GrB_NULL_POINTER;
    if (!d->user) return GrB_INVALID_VALUE;        // predefined: read-only
    switch (field)
    {
        case GrB_OUTP:
            if (val != GrB_DEFAULT && val != GrB_REPLACE) return GrB_INVALID_VALUE;
            d->outp = val; break;
        case GrB_MASK:
            if (val != GrB_DEFAULT && val != GrB_COMP && val != GrB_STRUCTURE &&
                val != GrB_COMP_STRUCTURE) return GrB_INVALID_VALUE;
            // COMP and STRUCTURE accumulate, as in the reference
            d->mask = (val == GrB_DEFAULT) ? 0 : (d->mask | val);
            break;
        case GrB_INP0:
            if (val != GrB_DEFAULT && val != GrB_TRAN) return GrB_INVALID_VALUE;
            d->inp0 = val; break;
        case GrB_INP1:
            if (val != GrB_DEFAULT && val != GrB_TRAN) return GrB_INVALID_VALUE;
            d->inp1 = val; break;
        case GxB_AxB_METHOD:
            if (val != GrB_DEFAULT && val != GxB_AxB_GUSTAVSON && val != GxB_AxB_DOT &&
                val != GxB_AxB_HASH && val != GxB_AxB_SAXPY) return GrB_INVALID_VALUE;
            d->method = val; break;
        case GxB_SORT:
            break;                                  // output is always sorted
        default:
            return GrB_INVALID_VALUE;
    }
    return GrB_SUCCESS;
}

GrB_Info GrB_Descriptor_free(GrB_Descriptor *desc)
{
    if (desc && *desc && (*desc)->user) free(*desc);
    if (desc) *desc = NULL;
    return GrB_SUCCESS;
}

typedef struct { bool replace, comp, strct, tA, tB; int method; } dflags;

static dflags decode(const GrB_Descriptor d)
{
    dflags f = {false, false, false, false, false, 0};
    if (d)
    {
        f.replace = d->outp == GrB_REPLACE;
        f.comp = (d->mask & GrB_COMP) != 0;
        f.strct = (d->mask & GrB_STRUCTURE) != 0;
        f.tA = d->inp0 == GrB_TRAN;
        f.tB = d->inp1 == GrB_TRAN;
        f.method = d->method;
    }
    return f;
}

//------------------------------------------------------------------------------
// matrices: host/device copies
//------------------------------------------------------------------------------

static void host_free(GrB_Matrix A)
{
    free(A->hp); free(A->hi); free(A->hx);
    A->hp = NULL; A->hi = NULL; A->hx = NULL;
    A->host_ok = false;
}

static void dev_drop(GrB_Matrix A)
{
    if (A->dev) grb_b200_dmatrix_free(&A->dev);
    A->dev = NULL;
    A->dev_ok = false;
}

// an empty matrix has an all-zero host copy
static GrB_Info host_empty(GrB_Matrix A)
{
    host_free(A);
    A->hp = calloc((size_t)A->nrows + 1, sizeof(int64_t));
    A->hi = malloc(sizeof(int64_t));
    A->hx = malloc(A->type->size);
    if (!A->hp || !A->hi || !A->hx) { host_free(A); return GrB_OUT_OF_MEMORY; }
    A->hiso = false;
    A->host_ok = true;
    return GrB_SUCCESS;
}

static GrB_Info to_dev(GrB_Matrix A)
{
    if (A->dev_ok) return GrB_SUCCESS;
    if (!A->host_ok) CHECK(host_empty(A));
    dev_drop(A);
    int info = grb_b200_dmatrix_upload(&A->dev, A->nrows, A->ncols, A->hp, A->hi,
                                       A->hx, A->type->code, A->hiso);
    if (info != 0) { A->dev = NULL; return (GrB_Info)info; }
    A->dev_ok = true;
    return GrB_SUCCESS;
}

static GrB_Info to_host(GrB_Matrix A)
{
    if (A->host_ok) return GrB_SUCCESS;
    if (!A->dev_ok) return host_empty(A);
    int64_t *p = NULL, *i = NULL;
    void *x = NULL;
    int info = grb_b200_dmatrix_download(A->dev, &p, &i, &x, true);
    if (info != 0) return (GrB_Info)info;
    host_free(A);
    A->hp = p; A->hi = i; A->hx = x;
    bool iso = false;
    grb_b200_dmatrix_info(A->dev, NULL, NULL, NULL, NULL, NULL, &iso);
    A->hiso = iso;
    A->host_ok = true;
    return GrB_SUCCESS;
}

// the matrix now holds device matrix D (ownership taken); the host copy is stale
static void set_dev(GrB_Matrix A, grb_b200_dmatrix D)
{
    dev_drop(A);
    host_free(A);
    A->dev = D;
    A->dev_ok = true;
}

static int64_t nvals_of(GrB_Matrix A)
{
    if (A->dev_ok)
    {
        int64_t nnz = 0, nz = 0;
        grb_b200_dmatrix_info(A->dev, NULL, NULL, &nnz, &nz, NULL, NULL);
        return nnz - nz;
    }
    if (A->host_ok) return A->hp[A->nrows];
    return 0;
}

static GrB_Info matrix_init(GrB_Matrix A, GrB_Type type, int64_t nrows, int64_t ncols)
{
    memset(A, 0, sizeof(*A));
    A->magic = MAGIC;
    A->type = type;
    A->nrows = nrows;
    A->ncols = ncols;
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_new(GrB_Matrix *A, GrB_Type type, GrB_Index nrows,
                        GrB_Index ncols)
{
    CHECK_INIT;
    if (!A || !type) return GrB_NULL_POINTER;
    *A = NULL;
    if (nrows > INT32_MAX || ncols > INT32_MAX) return GrB_INVALID_VALUE;
    GrB_Matrix M = malloc(sizeof(*M));
    if (!M) return GrB_OUT_OF_MEMORY;
    matrix_init(M, type, (int64_t)nrows, (int64_t)ncols);
    *A = M;
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_free(GrB_Matrix *A)
{
    if (!A || !*A) return GrB_SUCCESS;
    if ((*A)->magic == MAGIC)
    {
        host_free(*A);
        dev_drop(*A);
        (*A)->magic = FREED;
        free(*A);
    }
    *A = NULL;
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_dup(GrB_Matrix *C, const GrB_Matrix A)
{
    CHECK_INIT;
    if (!C || !A) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    CHECK(GrB_Matrix_new(C, A->type, A->nrows, A->ncols));
    if (A->dev_ok)
    {
        grb_b200_dmatrix D = NULL;
        int info = grb_b200_dmatrix_dup(&D, A->dev);
        if (info != 0) { GrB_Matrix_free(C); return (GrB_Info)info; }
        set_dev(*C, D);
    }
    else if (A->host_ok)
    {
        int64_t nnz = A->hp[A->nrows];
        size_t xs = A->hiso ? A->type->size : (size_t)(nnz ? nnz : 1) * A->type->size;
        GrB_Matrix X = *C;
        X->hp = malloc((size_t)(A->nrows + 1) * 8);
        X->hi = malloc((size_t)(nnz ? nnz : 1) * 8);
        X->hx = malloc(xs);
        if (!X->hp || !X->hi || !X->hx) { GrB_Matrix_free(C); return GrB_OUT_OF_MEMORY; }
        memcpy(X->hp, A->hp, (size_t)(A->nrows + 1) * 8);
        memcpy(X->hi, A->hi, (size_t)nnz * 8);
        if (A->hx) memcpy(X->hx, A->hx, A->hiso ? A->type->size : (size_t)nnz * A->type->size);
        X->hiso = A->hiso;
        X->host_ok = true;
    }
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_clear(GrB_Matrix A)
{
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    dev_drop(A);
    return host_empty(A);
}

GrB_Info GrB_Matrix_nrows(GrB_Index *n, const GrB_Matrix A)
{
    if (!n) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    *n = (GrB_Index)A->nrows;
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_ncols(GrB_Index *n, const GrB_Matrix A)
{
    if (!n) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    *n = (GrB_Index)A->ncols;
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_nvals(GrB_Index *nvals, const GrB_Matrix A)
{
    if (!nvals) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    *nvals = (GrB_Index)nvals_of(A);
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_wait(GrB_Matrix A, GrB_WaitMode mode)
{
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    if (mode != GrB_COMPLETE && mode != GrB_MATERIALIZE) return GrB_INVALID_VALUE;
    if (A->dev_ok)
    {
        int info = grb_b200_dwait(A->dev);        // kill zombies on the device
        if (info != 0) return (GrB_Info)info;
    }
    return GrB_SUCCESS;
}

GrB_Info GxB_Matrix_pack_CSR(GrB_Matrix A, GrB_Index **Ap, GrB_Index **Aj,
                             void **Ax, GrB_Index Ap_size, GrB_Index Aj_size,
                             GrB_Index Ax_size, bool iso, bool jumbled,
                             const GrB_Descriptor desc)
{
    (void)desc;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    if (!Ap || !Aj || !Ax || !*Ap || !*Aj) return GrB_NULL_POINTER;
    if (Ap_size < (GrB_Index)(A->nrows + 1) * sizeof(int64_t)) return GrB_INVALID_VALUE;
    int64_t nnz = (int64_t)(*Ap)[A->nrows];
    if (Aj_size < (GrB_Index)nnz * sizeof(int64_t)) return GrB_INVALID_VALUE;
    if (iso ? Ax_size < A->type->size : Ax_size < (GrB_Index)nnz * A->type->size)
        return GrB_INVALID_VALUE;
    if (jumbled)
    {
        // sort each row (values move along): the device kernels take sorted rows
        int64_t *p = (int64_t *)*Ap, *j = (int64_t *)*Aj;
        size_t ts = A->type->size;
        char *x = (char *)*Ax;
        char tmp[16];
        for (int64_t r = 0; r < A->nrows; r++)
            for (int64_t a = p[r] + 1; a < p[r + 1]; a++)
                for (int64_t b = a; b > p[r] && j[b - 1] > j[b]; b--)
                {
                    int64_t t = j[b]; j[b] = j[b - 1]; j[b - 1] = t;
                    if (!iso && x)
                    {
                        memcpy(tmp, x + b * ts, ts);
                        memcpy(x + b * ts, x + (b - 1) * ts, ts);
                        memcpy(x + (b - 1) * ts, tmp, ts);
                    }
                }
    }
    dev_drop(A);
    host_free(A);
    A->hp = (int64_t *)*Ap; A->hi = (int64_t *)*Aj; A->hx = *Ax;
    A->hiso = iso;
    A->host_ok = true;
    *Ap = NULL; *Aj = NULL; *Ax = NULL;
    return GrB_SUCCESS;
}

GrB_Info GxB_Matrix_unpack_CSR(GrB_Matrix A, GrB_Index **Ap, GrB_Index **Aj,
                               void **Ax, GrB_Index *Ap_size,
                               GrB_Index *Aj_size, GrB_Index *Ax_size,
                               bool *iso, bool *jumbled,
                               const GrB_Descriptor desc)
{
    (void)desc;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    if (!Ap || !Aj || !Ax || !Ap_size || !Aj_size || !Ax_size) return GrB_NULL_POINTER;
    CHECK(to_host(A));
    int64_t nnz = A->hp[A->nrows];
    *Ap = (GrB_Index *)A->hp; *Aj = (GrB_Index *)A->hi; *Ax = A->hx;
    *Ap_size = (GrB_Index)(A->nrows + 1) * 8;
    *Aj_size = (GrB_Index)(nnz ? nnz : 1) * 8;
    *Ax_size = A->hiso ? A->type->size : (GrB_Index)(nnz ? nnz : 1) * A->type->size;
    if (iso) *iso = A->hiso;
    else if (A->hiso && nnz > 1)
    {
        // caller cannot take an iso matrix: expand the value
        void *x = malloc((size_t)nnz * A->type->size);
        if (!x) return GrB_OUT_OF_MEMORY;
        for (int64_t k = 0; k < nnz; k++)
            memcpy((char *)x + k * A->type->size, A->hx, A->type->size);
        free(A->hx);
        *Ax = x;
        *Ax_size = (GrB_Index)nnz * A->type->size;
    }
    if (jumbled) *jumbled = false;
    A->hp = NULL; A->hi = NULL; A->hx = NULL;
    A->host_ok = false;
    dev_drop(A);
    return GrB_SUCCESS;
}

#define EXTRACT(T, CT, CODE) \
GrB_Info GrB_Matrix_extractTuples_##T(GrB_Index *I, GrB_Index *J, CT *X, \
                                      GrB_Index *nvals, const GrB_Matrix A) \
{ \
    if (!nvals) return GrB_NULL_POINTER; \
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT; \
    if (X && A->type->code != CODE) return GrB_DOMAIN_MISMATCH; \
    CHECK(to_host(A)); \
    int64_t nnz = A->hp[A->nrows]; \
    if (*nvals < (GrB_Index)nnz) return GrB_INSUFFICIENT_SPACE; \
    for (int64_t r = 0; r < A->nrows; r++) \
        for (int64_t q = A->hp[r]; q < A->hp[r + 1]; q++) \
        { \
            if (I) I[q] = (GrB_Index)r; \
            if (J) J[q] = (GrB_Index)A->hi[q]; \
            if (X) X[q] = ((CT *)A->hx)[A->hiso ? 0 : q]; \
        } \
    *nvals = (GrB_Index)nnz; \
    return GrB_SUCCESS; \
}
EXTRACT(BOOL, bool, 1)
EXTRACT(INT32, int32_t, 6)
EXTRACT(INT64, int64_t, 8)
EXTRACT(FP32, float, 10)
EXTRACT(FP64, double, 11)
#undef EXTRACT

//------------------------------------------------------------------------------
// import / export: copies between the caller's CSR arrays and the device
// (GrB_Matrix_import.c:28-205, GrB_Matrix_export.c:38-215,
// GrB_Matrix_exportSize.c).  Only GrB_CSR_FORMAT is supported here; the
// arrays go straight to or from HBM (no host copy is kept), and the import
// is checked on the device as the reference's secure import checks it.
//------------------------------------------------------------------------------

static GrB_Info import_any(GrB_Matrix *A, GrB_Type type, int code, GrB_Index nrows,
                           GrB_Index ncols, const GrB_Index *Ap, const GrB_Index *Ai,
                           const void *Ax, GrB_Index Ap_len, GrB_Index Ai_len,
                           GrB_Index Ax_len, GrB_Format format)
{
    CHECK_INIT;
    if (!A) return GrB_NULL_POINTER;
    *A = NULL;
    if (!type || !Ax || !Ap || !Ai) return GrB_NULL_POINTER;
    if (type->code != code) return GrB_DOMAIN_MISMATCH;
    if (format == GrB_CSC_FORMAT || format == GrB_COO_FORMAT) return GrB_NOT_IMPLEMENTED;
    if (format != GrB_CSR_FORMAT) return GrB_INVALID_VALUE;
    if (Ap_len < nrows + 1) return GrB_INVALID_VALUE;
    const GrB_Index nvals = Ap[nrows];
    if (Ai_len < nvals || Ax_len < nvals) return GrB_INVALID_VALUE;
    GrB_Matrix M = NULL;
    CHECK(GrB_Matrix_new(&M, type, nrows, ncols));
    int info = grb_b200_dmatrix_import(&M->dev, (int64_t)nrows, (int64_t)ncols,
                                       (const int64_t *)Ap, (const int64_t *)Ai, Ax,
                                       type->code);
    if (info != 0) { M->dev = NULL; GrB_Matrix_free(&M); return (GrB_Info)info; }
    M->dev_ok = true;
    *A = M;
    return GrB_SUCCESS;
}

static GrB_Info export_any(GrB_Index *Ap, GrB_Index *Ai, void *Ax, int code,
                           GrB_Index *Ap_len, GrB_Index *Ai_len, GrB_Index *Ax_len,
                           GrB_Format format, GrB_Matrix A)
{
    if (!Ap || !Ai || !Ax || !Ap_len || !Ai_len || !Ax_len) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    if (A->type->code != code) return GrB_DOMAIN_MISMATCH;
    if (format == GrB_CSC_FORMAT || format == GrB_COO_FORMAT) return GrB_NOT_IMPLEMENTED;
    if (format != GrB_CSR_FORMAT) return GrB_INVALID_VALUE;
    const GrB_Index nvals = (GrB_Index)nvals_of(A);
    const GrB_Index plen = (GrB_Index)A->nrows + 1;
    if (plen > *Ap_len || nvals > *Ai_len || nvals > *Ax_len) return GrB_INSUFFICIENT_SPACE;
    if (A->dev_ok)
    {
        // straight from HBM into the caller's arrays
        int info = grb_b200_dmatrix_export(A->dev, (int64_t *)Ap, (int64_t *)Ai, Ax);
        if (info != 0) return (GrB_Info)info;
    }
    else
    {
        if (!A->host_ok) CHECK(host_empty(A));
        memcpy(Ap, A->hp, plen * sizeof(int64_t));
        memcpy(Ai, A->hi, nvals * sizeof(int64_t));
        for (GrB_Index k = 0; k < nvals; k++)
            memcpy((char *)Ax + k * A->type->size,
                   (char *)A->hx + (A->hiso ? 0 : k) * A->type->size, A->type->size);
    }
    *Ap_len = plen;
    *Ai_len = nvals;
    *Ax_len = nvals;
    return GrB_SUCCESS;
}

#define IMPORT_EXPORT(T, CT, CODE) \
GrB_Info GrB_Matrix_import_##T(GrB_Matrix *A, GrB_Type type, GrB_Index nrows, \
    GrB_Index ncols, const GrB_Index *Ap, const GrB_Index *Ai, const CT *Ax, \
    GrB_Index Ap_len, GrB_Index Ai_len, GrB_Index Ax_len, GrB_Format format) \
{ \
    return import_any(A, type, CODE, nrows, ncols, Ap, Ai, Ax, Ap_len, Ai_len, \
                      Ax_len, format); \
} \
GrB_Info GrB_Matrix_export_##T(GrB_Index *Ap, GrB_Index *Ai, CT *Ax, \
    GrB_Index *Ap_len, GrB_Index *Ai_len, GrB_Index *Ax_len, GrB_Format format, \
    GrB_Matrix A) \
{ \
    return export_any(Ap, Ai, Ax, CODE, Ap_len, Ai_len, Ax_len, format, A); \
}
IMPORT_EXPORT(BOOL, bool, 1)
IMPORT_EXPORT(INT32, int32_t, 6)
IMPORT_EXPORT(UINT32, uint32_t, 7)
IMPORT_EXPORT(INT64, int64_t, 8)
IMPORT_EXPORT(UINT64, uint64_t, 9)
IMPORT_EXPORT(FP32, float, 10)
IMPORT_EXPORT(FP64, double, 11)
#undef IMPORT_EXPORT

GrB_Info GrB_Matrix_exportSize(GrB_Index *Ap_len, GrB_Index *Ai_len,
                               GrB_Index *Ax_len, GrB_Format format, GrB_Matrix A)
{
    if (!Ap_len || !Ai_len || !Ax_len) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    if (format == GrB_CSC_FORMAT || format == GrB_COO_FORMAT) return GrB_NOT_IMPLEMENTED;
    if (format != GrB_CSR_FORMAT) return GrB_INVALID_VALUE;
    const GrB_Index nvals = (GrB_Index)nvals_of(A);
    *Ap_len = (GrB_Index)A->nrows + 1;
    *Ai_len = nvals;
    *Ax_len = nvals;
    return GrB_SUCCESS;
}

//------------------------------------------------------------------------------
// serialize / deserialize (Source/serialize/GrB_Matrix_serialize.c,
// GxB_Matrix_serialize.c, GrB_Matrix_serializeSize.c, GxB_Matrix_deserialize.c,
// GrB_Matrix_deserialize.c, GxB_Vector_serialize.c, GxB_Vector_deserialize.c).
// A blob is written from the matrix's CSR arrays (one download from HBM when
// the matrix lives there) in the reference's uncompressed format, and a blob
// read is decoded on the host into the matrix's host copy, which goes to HBM
// at its first use on the device.
//------------------------------------------------------------------------------

static GrB_Type type_of_code(int code)
{
    switch (code)
    {
        case 1: return GrB_BOOL;
        case 6: return GrB_INT32;
        case 7: return GrB_UINT32;
        case 8: return GrB_INT64;
        case 9: return GrB_UINT64;
        case 10: return GrB_FP32;
        case 11: return GrB_FP64;
    }
    return NULL;
}

// blob of A (a 1-by-n vector is written as the reference's n-by-1 column);
// blob == NULL: *size gets the exact size
static GrB_Info serialize_any(void *blob, size_t *size, GrB_Matrix A, bool vector)
{
    CHECK(to_host(A));
    if (vector)
        return (GrB_Info)grb_b200_blob_encode(blob, size, A->ncols, 1, A->type->code,
                                              A->hp, A->hi, A->hx, A->hiso, true);
    return (GrB_Info)grb_b200_blob_encode(blob, size, A->nrows, A->ncols, A->type->code,
                                          A->hp, A->hi, A->hx, A->hiso, false);
}

GrB_Info GrB_Matrix_serializeSize(GrB_Index *blob_size_handle, GrB_Matrix A)
{
    if (!blob_size_handle) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    size_t size = 0;
    CHECK(serialize_any(NULL, &size, A, false));
    *blob_size_handle = (GrB_Index)size;
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_serialize(void *blob, GrB_Index *blob_size_handle, GrB_Matrix A)
{
    if (!blob || !blob_size_handle) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    size_t size = (size_t)*blob_size_handle;
    CHECK(serialize_any(blob, &size, A, false));
    *blob_size_handle = (GrB_Index)size;
    return GrB_SUCCESS;
}

static GrB_Info serialize_alloc(void **blob_handle, GrB_Index *blob_size_handle,
                                GrB_Matrix A, bool vector)
{
    size_t size = 0;
    CHECK(serialize_any(NULL, &size, A, vector));
    void *blob = malloc(size);
    if (!blob) return GrB_OUT_OF_MEMORY;
    GrB_Info info = serialize_any(blob, &size, A, vector);
    if (info != GrB_SUCCESS) { free(blob); return info; }
    *blob_handle = blob;
    *blob_size_handle = (GrB_Index)size;
    return GrB_SUCCESS;
}

GrB_Info GxB_Matrix_serialize(void **blob_handle, GrB_Index *blob_size_handle,
                              GrB_Matrix A, const GrB_Descriptor desc)
{
    (void)desc;
    if (!blob_handle || !blob_size_handle) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    return serialize_alloc(blob_handle, blob_size_handle, A, false);
}

// decode a blob into a new matrix whose host copy holds the arrays
static GrB_Info deserialize_any(GrB_Matrix *C, GrB_Type type, const void *blob,
                                GrB_Index blob_size)
{
    CHECK_INIT;
    if (!C || !blob) return GrB_NULL_POINTER;
    *C = NULL;
    int64_t nrows = 0, ncols = 0, *p = NULL, *i = NULL;
    void *x = NULL;
    int code = 0;
    bool iso = false;
    CHECK(grb_b200_blob_decode(blob, (size_t)blob_size, type ? type->code : 0, &nrows,
                               &ncols, &code, &p, &i, &x, &iso));
    GrB_Matrix M = NULL;
    GrB_Info info = GrB_Matrix_new(&M, type_of_code(code), (GrB_Index)nrows,
                                   (GrB_Index)ncols);
    if (info != GrB_SUCCESS) { free(p); free(i); free(x); return info; }
    if (!i) i = malloc(sizeof(int64_t));          // the host copy keeps non-NULL arrays
    if (!x) x = calloc(1, M->type->size);
    if (!i || !x) { free(p); free(i); free(x); GrB_Matrix_free(&M); return GrB_OUT_OF_MEMORY; }
    M->hp = p; M->hi = i; M->hx = x;
    M->hiso = iso;
    M->host_ok = true;
    *C = M;
    return GrB_SUCCESS;
}

GrB_Info GrB_Matrix_deserialize(GrB_Matrix *C, GrB_Type type, const void *blob,
                                GrB_Index blob_size)
{
    return deserialize_any(C, type, blob, blob_size);
}

GrB_Info GxB_Matrix_deserialize(GrB_Matrix *C, GrB_Type type, const void *blob,
                                GrB_Index blob_size, const GrB_Descriptor desc)
{
    (void)desc;
    return deserialize_any(C, type, blob, blob_size);
}

//------------------------------------------------------------------------------
// vectors (1-by-n rows inside)
//------------------------------------------------------------------------------

#define VM(v) (&(v)->m)
#define VOK(v) ((v) != NULL && (v)->m.magic == MAGIC)

GrB_Info GrB_Vector_new(GrB_Vector *v, GrB_Type type, GrB_Index n)
{
    CHECK_INIT;
    if (!v || !type) return GrB_NULL_POINTER;
    *v = NULL;
    if (n > INT32_MAX) return GrB_INVALID_VALUE;
    GrB_Vector w = malloc(sizeof(*w));
    if (!w) return GrB_OUT_OF_MEMORY;
    matrix_init(VM(w), type, 1, (int64_t)n);
    *v = w;
    return GrB_SUCCESS;
}

GrB_Info GrB_Vector_free(GrB_Vector *v)
{
    if (!v || !*v) return GrB_SUCCESS;
    if ((*v)->m.magic == MAGIC)
    {
        host_free(VM(*v));
        dev_drop(VM(*v));
        (*v)->m.magic = FREED;
        free(*v);
    }
    *v = NULL;
    return GrB_SUCCESS;
}

GrB_Info GrB_Vector_dup(GrB_Vector *w, const GrB_Vector u)
{
    if (!w || !u) return GrB_NULL_POINTER;
    if (!VOK(u)) return GrB_UNINITIALIZED_OBJECT;
    GrB_Matrix C = NULL;
    CHECK(GrB_Matrix_dup(&C, VM(u)));
    GrB_Vector v = malloc(sizeof(*v));
    if (!v) { GrB_Matrix_free(&C); return GrB_OUT_OF_MEMORY; }
    v->m = *C;
    free(C);                                       // contents moved into v
    *w = v;
    return GrB_SUCCESS;
}

GrB_Info GrB_Vector_clear(GrB_Vector v)
{
    if (!VOK(v)) return GrB_UNINITIALIZED_OBJECT;
    return GrB_Matrix_clear(VM(v));
}

GrB_Info GrB_Vector_size(GrB_Index *n, const GrB_Vector v)
{
    if (!n) return GrB_NULL_POINTER;
    if (!VOK(v)) return GrB_UNINITIALIZED_OBJECT;
    *n = (GrB_Index)v->m.ncols;
    return GrB_SUCCESS;
}

GrB_Info GrB_Vector_nvals(GrB_Index *nvals, const GrB_Vector v)
{
    if (!VOK(v)) return GrB_UNINITIALIZED_OBJECT;
    return GrB_Matrix_nvals(nvals, VM(v));
}

GrB_Info GrB_Vector_wait(GrB_Vector v, GrB_WaitMode mode)
{
    if (!VOK(v)) return GrB_UNINITIALIZED_OBJECT;
    return GrB_Matrix_wait(VM(v), mode);
}

static GrB_Info vector_set(GrB_Vector w, const void *x, int code, GrB_Index i)
{
    if (!VOK(w)) return GrB_UNINITIALIZED_OBJECT;
    GrB_Matrix A = VM(w);
    if (A->type->code != code) return GrB_DOMAIN_MISMATCH;
    if ((int64_t)i >= A->ncols) return GrB_INVALID_INDEX;
    CHECK(to_host(A));
    size_t ts = A->type->size;
    int64_t nnz = A->hp[1];
    // expand an iso value before writing a single entry
    if (A->hiso && nnz > 0)
    {
        void *nx = malloc((size_t)nnz * ts);
        if (!nx) return GrB_OUT_OF_MEMORY;
        for (int64_t k = 0; k < nnz; k++) memcpy((char *)nx + k * ts, A->hx, ts);
        free(A->hx);
        A->hx = nx;
        A->hiso = false;
    }
    A->hiso = false;
    int64_t lo = 0, hi = nnz;
    while (lo < hi) { int64_t mid = (lo + hi) / 2; if (A->hi[mid] < (int64_t)i) lo = mid + 1; else hi = mid; }
    if (lo < nnz && A->hi[lo] == (int64_t)i)
    {
        memcpy((char *)A->hx + lo * ts, x, ts);
    }
    else
    {
        int64_t *ni = realloc(A->hi, (size_t)(nnz + 1) * 8);
        if (!ni) return GrB_OUT_OF_MEMORY;
        A->hi = ni;
        void *nx = realloc(A->hx, (size_t)(nnz + 1) * ts);
        if (!nx) return GrB_OUT_OF_MEMORY;
        A->hx = nx;
        memmove(A->hi + lo + 1, A->hi + lo, (size_t)(nnz - lo) * 8);
        memmove((char *)A->hx + (lo + 1) * ts, (char *)A->hx + lo * ts, (size_t)(nnz - lo) * ts);
        A->hi[lo] = (int64_t)i;
        memcpy((char *)A->hx + lo * ts, x, ts);
        A->hp[1] = nnz + 1;
    }
    dev_drop(A);
    return GrB_SUCCESS;
}

GrB_Info GrB_Vector_setElement_BOOL(GrB_Vector w, bool x, GrB_Index i) { return vector_set(w, &x, 1, i); }
GrB_Info GrB_Vector_setElement_INT32(GrB_Vector w, int32_t x, GrB_Index i) { return vector_set(w, &x, 6, i); }
GrB_Info GrB_Vector_setElement_INT64(GrB_Vector w, int64_t x, GrB_Index i) { return vector_set(w, &x, 8, i); }
GrB_Info GrB_Vector_setElement_FP32(GrB_Vector w, float x, GrB_Index i) { return vector_set(w, &x, 10, i); }
GrB_Info GrB_Vector_setElement_FP64(GrB_Vector w, double x, GrB_Index i) { return vector_set(w, &x, 11, i); }

GrB_Info GxB_Vector_pack_CSC(GrB_Vector v, GrB_Index **vi, void **vx,
                             GrB_Index vi_size, GrB_Index vx_size, bool iso,
                             GrB_Index nvals, bool jumbled,
                             const GrB_Descriptor desc)
{
    (void)desc;
    if (!VOK(v)) return GrB_UNINITIALIZED_OBJECT;
    if (!vi || !vx || !*vi) return GrB_NULL_POINTER;
    GrB_Matrix A = VM(v);
    if (vi_size < nvals * sizeof(int64_t)) return GrB_INVALID_VALUE;
    if (iso ? vx_size < A->type->size : vx_size < nvals * A->type->size)
        return GrB_INVALID_VALUE;
    int64_t *p = malloc(2 * sizeof(int64_t));
    if (!p) return GrB_OUT_OF_MEMORY;
    p[0] = 0; p[1] = (int64_t)nvals;
    GrB_Index *pp = (GrB_Index *)p;
    GrB_Info info = GxB_Matrix_pack_CSR(A, &pp, vi, vx, 2 * sizeof(int64_t), vi_size,
                                        vx_size, iso, jumbled, NULL);
    if (info != GrB_SUCCESS) free(p);
    return info;
}

GrB_Info GxB_Vector_unpack_CSC(GrB_Vector v, GrB_Index **vi, void **vx,
                               GrB_Index *vi_size, GrB_Index *vx_size,
                               bool *iso, GrB_Index *nvals, bool *jumbled,
                               const GrB_Descriptor desc)
{
    (void)desc;
    if (!VOK(v)) return GrB_UNINITIALIZED_OBJECT;
    if (!nvals) return GrB_NULL_POINTER;
    GrB_Index *p = NULL, psize = 0;
    CHECK(GxB_Matrix_unpack_CSR(VM(v), &p, vi, vx, &psize, vi_size, vx_size, iso,
                                jumbled, NULL));
    *nvals = p[1];
    free(p);
    return GrB_SUCCESS;
}

// a vector held on the device goes straight into the caller's I and X (its
// one row's indices and values), with no host copy in between
static GrB_Info vector_extract_dev(GrB_Index *I, void *X, GrB_Index *nvals, GrB_Vector v)
{
    GrB_Matrix A = VM(v);
    const int64_t nv = nvals_of(A);
    if (*nvals < (GrB_Index)nv) return GrB_INSUFFICIENT_SPACE;
    int64_t p2[2];
    int64_t *ii = (int64_t *)I;
    void *xx = X;
    int64_t *tmp_i = NULL;
    if (!ii)
    {
        tmp_i = malloc((size_t)(nv ? nv : 1) * sizeof(int64_t));
        if (!tmp_i) return GrB_OUT_OF_MEMORY;
        ii = tmp_i;
    }
    int info = grb_b200_dmatrix_export(A->dev, p2, ii, xx);
    free(tmp_i);
    if (info != 0) return (GrB_Info)info;
    *nvals = (GrB_Index)nv;
    return GrB_SUCCESS;
}

#define VEXTRACT(T, CT, CODE) \
GrB_Info GrB_Vector_extractTuples_##T(GrB_Index *I, CT *X, GrB_Index *nvals, \
                                      const GrB_Vector v) \
{ \
    if (!nvals) return GrB_NULL_POINTER; \
    if (!VOK(v)) return GrB_UNINITIALIZED_OBJECT; \
    if (X && VM(v)->type->code != CODE) return GrB_DOMAIN_MISMATCH; \
    if (VM(v)->dev_ok && !VM(v)->host_ok) return vector_extract_dev(I, X, nvals, v); \
    return GrB_Matrix_extractTuples_##T(NULL, I, X, nvals, VM(v)); \
}
VEXTRACT(BOOL, bool, 1)
VEXTRACT(INT32, int32_t, 6)
VEXTRACT(INT64, int64_t, 8)
VEXTRACT(FP32, float, 10)
VEXTRACT(FP64, double, 11)
#undef VEXTRACT

GrB_Info GxB_Vector_serialize(void **blob_handle, GrB_Index *blob_size_handle,
                              GrB_Vector u, const GrB_Descriptor desc)
{
    (void)desc;
    if (!blob_handle || !blob_size_handle) return GrB_NULL_POINTER;
    if (!VOK(u)) return GrB_UNINITIALIZED_OBJECT;
    return serialize_alloc(blob_handle, blob_size_handle, VM(u), true);
}

// a vector blob holds an n-by-1 matrix; its entries become the one row here
GrB_Info GxB_Vector_deserialize(GrB_Vector *w, GrB_Type type, const void *blob,
                                GrB_Index blob_size, const GrB_Descriptor desc)
{
    (void)desc;
    if (!w) return GrB_NULL_POINTER;
    *w = NULL;
    GrB_Matrix C = NULL;
    CHECK(deserialize_any(&C, type, blob, blob_size));
    if (C->ncols != 1) { GrB_Matrix_free(&C); return GrB_INVALID_OBJECT; }
    const int64_t n = C->nrows, nnz = C->hp[n];
    int64_t *p = malloc(2 * sizeof(int64_t));
    int64_t *ii = malloc((size_t)(nnz ? nnz : 1) * sizeof(int64_t));
    if (!p || !ii) { free(p); free(ii); GrB_Matrix_free(&C); return GrB_OUT_OF_MEMORY; }
    for (int64_t r = 0; r < n; r++)
        if (C->hp[r + 1] > C->hp[r]) ii[C->hp[r]] = r;   // the value order is kept
    p[0] = 0;
    p[1] = nnz;
    GrB_Vector v = malloc(sizeof(*v));
    if (!v) { free(p); free(ii); GrB_Matrix_free(&C); return GrB_OUT_OF_MEMORY; }
    matrix_init(VM(v), C->type, 1, n);
    v->m.hp = p; v->m.hi = ii; v->m.hx = C->hx;
    v->m.hiso = C->hiso;
    v->m.host_ok = true;
    C->hx = NULL;
    GrB_Matrix_free(&C);
    *w = v;
    return GrB_SUCCESS;
}

//------------------------------------------------------------------------------
// the multiply path
//------------------------------------------------------------------------------

static bool reads_a(int mult) { return !(mult == OP_PAIR || mult == OP_SECOND || (mult >= OP_FIRSTI && mult <= 122)); }
static bool reads_b(int mult) { return !(mult == OP_PAIR || mult == OP_FIRST || (mult >= OP_FIRSTI && mult <= 122)); }

// operand swap of a multiplier (y (x) x instead of x (x) y); -1 if positional
static int flip_mult(int m)
{
    switch (m)
    {
        case OP_FIRST: return OP_SECOND;
        case OP_SECOND: return OP_FIRST;
        case OP_MINUS: return OP_RMINUS;
        case OP_RMINUS: return OP_MINUS;
        default: return (m >= OP_FIRSTI && m <= 122) ? -1 : m;
    }
}

static GrB_Info check_domains(const GrB_Semiring s, GrB_Matrix C, GrB_BinaryOp accum,
                              GrB_Matrix A, GrB_Matrix B)
{
    if (reads_a(s->mult) && A->type != s->type) return GrB_DOMAIN_MISMATCH;
    if (reads_b(s->mult) && B->type != s->type) return GrB_DOMAIN_MISMATCH;
    if (C->type != s->type) return GrB_DOMAIN_MISMATCH;
    if (accum && accum->type != C->type && accum->opcode != OP_LOR &&
        accum->opcode != OP_LAND) return GrB_DOMAIN_MISMATCH;
    return GrB_SUCCESS;
}

// write T into C honouring mask/accum/replace (T is consumed)
static GrB_Info write_back(GrB_Matrix C, grb_b200_dmatrix T, GrB_Matrix M,
                           bool mask_applied, GrB_BinaryOp accum, dflags f)
{
    bool direct = !accum && (M == NULL || (mask_applied && (f.replace || nvals_of(C) == 0)));
    if (direct)
    {
        set_dev(C, T);
        return GrB_SUCCESS;
    }
    GrB_Info info = to_dev(C);
    if (info == GrB_SUCCESS && M) info = to_dev(M);
    if (info == GrB_SUCCESS)
        info = (GrB_Info)grb_b200_daccum_mask(C->dev, T, M ? M->dev : NULL, f.comp,
                                              f.strct, f.replace,
                                              accum ? accum->opcode : 0);
    grb_b200_dmatrix_free(&T);
    if (info == GrB_SUCCESS) host_free(C);
    return info;
}

GrB_Info GrB_mxm(GrB_Matrix C, const GrB_Matrix M, const GrB_BinaryOp accum,
                 const GrB_Semiring s, const GrB_Matrix A, const GrB_Matrix B,
                 const GrB_Descriptor desc)
{
    CHECK_INIT;
    if (!C || !s || !A || !B) return GrB_NULL_POINTER;
    if (!OBJ_OK(C) || !OBJ_OK(A) || !OBJ_OK(B) || (M && !OBJ_OK(M)))
        return GrB_UNINITIALIZED_OBJECT;
    dflags f = decode(desc);
    int64_t anr = f.tA ? A->ncols : A->nrows, anc = f.tA ? A->nrows : A->ncols;
    int64_t bnr = f.tB ? B->ncols : B->nrows, bnc = f.tB ? B->nrows : B->ncols;
    if (anc != bnr || C->nrows != anr || C->ncols != bnc) return GrB_DIMENSION_MISMATCH;
    if (M && (M->nrows != C->nrows || M->ncols != C->ncols)) return GrB_DIMENSION_MISMATCH;
    CHECK(check_domains(s, C, accum, A, B));
    // C<!NULL> = ...: nothing is written; replace still clears C
    if (!M && f.comp) return f.replace ? GrB_Matrix_clear(C) : GrB_SUCCESS;
    CHECK(to_dev(A));
    CHECK(to_dev(B));
    if (M) CHECK(to_dev(M));
    grb_b200_semiring sr = {s->add, s->mult, s->type->code};
    grb_b200_dmatrix dA = A->dev, tA = NULL, dB = NULL, tB = NULL, T = NULL;
    int info = 0;
    if (f.tA) { info = grb_b200_dtranspose(&tA, A->dev); dA = tA; }
    bool use_dot = M && !f.comp && (f.tB || f.method == GxB_AxB_DOT) &&
                   f.method != GxB_AxB_GUSTAVSON && f.method != GxB_AxB_HASH;
    bool mask_applied = false;
    if (info == 0)
    {
        if (use_dot)
        {
            // rows of B' are the rows of B; otherwise transpose B first
            if (f.tB) dB = B->dev;
            else { info = grb_b200_dtranspose(&tB, B->dev); dB = tB; }
            if (info == 0) info = grb_b200_dmxm_dot3(&T, M->dev, f.strct, dA, dB, &sr);
        }
        else
        {
            if (f.tB) { info = grb_b200_dtranspose(&tB, B->dev); dB = tB; }
            else dB = B->dev;
            if (info == 0)
                info = grb_b200_dmxm_saxpy3(&T, M ? M->dev : NULL, f.comp, f.strct, dA,
                                            dB, &sr);
        }
        mask_applied = (M != NULL);
    }
    if (tA) grb_b200_dmatrix_free(&tA);
    if (tB) grb_b200_dmatrix_free(&tB);
    if (info == 1) return GrB_NOT_IMPLEMENTED;     // semiring not compiled
    if (info != 0) return (GrB_Info)info;
    return write_back(C, T, M, mask_applied, accum, f);
}

// w' = u'*A (tA = false) or u'*A' (tA = true), i.e. GrB_vxm; GrB_mxv maps here
static GrB_Info vector_times(GrB_Vector w, const GrB_Vector mask,
                             const GrB_BinaryOp accum, const GrB_Semiring s,
                             const GrB_Vector u, const GrB_Matrix A, dflags f,
                             bool row_form)
{
    // row_form: w = u'*A with the multiplier applied as u(k) (x) A(k,j)
    // else:     w = A*u with A(i,k) (x) u(k)
    GrB_Matrix W = VM(w), U = VM(u), Mk = mask ? VM(mask) : NULL;
    if (!Mk && f.comp) return f.replace ? GrB_Matrix_clear(W) : GrB_SUCCESS;
    CHECK(to_dev(A));
    CHECK(to_dev(U));
    if (Mk) CHECK(to_dev(Mk));
    int info = 0;
    grb_b200_dmatrix T = NULL, tmp = NULL;
    grb_b200_semiring sr = {s->add, s->mult, s->type->code};
    if (row_form)
    {
        // saxpy3 with u as a 1-row matrix: needs A by rows (transpose if A')
        grb_b200_dmatrix dA = A->dev;
        if (f.tA) { info = grb_b200_dtranspose(&tmp, A->dev); dA = tmp; }
        if (info == 0)
            info = grb_b200_dmxm_saxpy3(&T, Mk ? Mk->dev : NULL, f.comp, f.strct, U->dev,
                                        dA, &sr);
    }
    else
    {
        grb_b200_dmatrix dA = A->dev;
        if (f.tA) { info = grb_b200_dtranspose(&tmp, A->dev); dA = tmp; }
        if (info == 0)
            info = grb_b200_dmxv(&T, Mk ? Mk->dev : NULL, f.comp, f.strct, dA, U->dev, &sr);
    }
    if (tmp) grb_b200_dmatrix_free(&tmp);
    if (info == 1) return GrB_NOT_IMPLEMENTED;
    if (info != 0) return (GrB_Info)info;
    return write_back(W, T, Mk, Mk != NULL, accum, f);
}

GrB_Info GrB_vxm(GrB_Vector w, const GrB_Vector mask, const GrB_BinaryOp accum,
                 const GrB_Semiring s, const GrB_Vector u, const GrB_Matrix A,
                 const GrB_Descriptor desc)
{
    CHECK_INIT;
    if (!w || !s || !u || !A) return GrB_NULL_POINTER;
    if (!VOK(w) || !VOK(u) || !OBJ_OK(A) || (mask && !VOK(mask)))
        return GrB_UNINITIALIZED_OBJECT;
    dflags f = decode(desc);
    // GrB_vxm's matrix is its second input (GrB_INP1)
    bool tA = f.tB;
    int64_t anr = tA ? A->ncols : A->nrows, anc = tA ? A->nrows : A->ncols;
    if (u->m.ncols != anr || w->m.ncols != anc) return GrB_DIMENSION_MISMATCH;
    if (mask && mask->m.ncols != w->m.ncols) return GrB_DIMENSION_MISMATCH;
    CHECK(check_domains(s, VM(w), accum, VM(u), A));
    dflags g = f;
    g.tA = tA;
    if (!tA) return vector_times(w, mask, accum, s, u, A, g, true);
    // w' = u'*A' = (A*u)': the row kernel of A with the operands swapped
    int fm = flip_mult(s->mult);
    if (fm < 0) return GrB_NOT_IMPLEMENTED;
    struct GB_Semiring_opaque s2 = *s;
    s2.mult = fm;
    g.tA = false;
    return vector_times(w, mask, accum, &s2, u, A, g, false);
}

GrB_Info GrB_mxv(GrB_Vector w, const GrB_Vector mask, const GrB_BinaryOp accum,
                 const GrB_Semiring s, const GrB_Matrix A, const GrB_Vector u,
                 const GrB_Descriptor desc)
{
    CHECK_INIT;
    if (!w || !s || !u || !A) return GrB_NULL_POINTER;
    if (!VOK(w) || !VOK(u) || !OBJ_OK(A) || (mask && !VOK(mask)))
        return GrB_UNINITIALIZED_OBJECT;
    dflags f = decode(desc);
    int64_t anr = f.tA ? A->ncols : A->nrows, anc = f.tA ? A->nrows : A->ncols;
    if (u->m.ncols != anc || w->m.ncols != anr) return GrB_DIMENSION_MISMATCH;
    if (mask && mask->m.ncols != w->m.ncols) return GrB_DIMENSION_MISMATCH;
    CHECK(check_domains(s, VM(w), accum, A, VM(u)));
    if (!f.tA) return vector_times(w, mask, accum, s, u, A, f, false);
    // w = A'*u = (u'*A)': the row-form kernel with the operands swapped
    int fm = flip_mult(s->mult);
    if (fm < 0) return GrB_NOT_IMPLEMENTED;
    struct GB_Semiring_opaque s2 = *s;
    s2.mult = fm;
    dflags g = f;
    g.tA = false;
    return vector_times(w, mask, accum, &s2, u, A, g, true);
}

//------------------------------------------------------------------------------
// the callers on either side of the multiply
//------------------------------------------------------------------------------

GrB_Info GrB_Vector_assign(GrB_Vector w, const GrB_Vector mask,
                           const GrB_BinaryOp accum, const GrB_Vector u,
                           const GrB_Index *I, GrB_Index ni,
                           const GrB_Descriptor desc)
{
    CHECK_INIT;
    if (!w || !u) return GrB_NULL_POINTER;
    if (!VOK(w) || !VOK(u) || (mask && !VOK(mask))) return GrB_UNINITIALIZED_OBJECT;
    if (I != GrB_ALL) return GrB_NOT_IMPLEMENTED;     // only w<m>(:) = u here
    if ((int64_t)ni != w->m.ncols || u->m.ncols != w->m.ncols) return GrB_DIMENSION_MISMATCH;
    if (mask && mask->m.ncols != w->m.ncols) return GrB_DIMENSION_MISMATCH;
    if (u->m.type != w->m.type) return GrB_DOMAIN_MISMATCH;
    dflags f = decode(desc);
    GrB_Matrix W = VM(w), U = VM(u), Mk = mask ? VM(mask) : NULL;
    CHECK(to_dev(W));
    CHECK(to_dev(U));
    if (Mk) CHECK(to_dev(Mk));
    int info = grb_b200_daccum_mask(W->dev, U->dev, Mk ? Mk->dev : NULL, f.comp,
                                    f.strct, f.replace, accum ? accum->opcode : 0);
    if (info != 0) return (GrB_Info)info;
    host_free(W);
    return GrB_SUCCESS;
}

static GrB_Info reduce_any(void *s, int code, const GrB_BinaryOp accum,
                           const GrB_Monoid monoid, GrB_Matrix A)
{
    CHECK_INIT;
    if (!s || !monoid) return GrB_NULL_POINTER;
    if (!OBJ_OK(A)) return GrB_UNINITIALIZED_OBJECT;
    if (accum) return GrB_NOT_IMPLEMENTED;
    if (monoid->type->code != code || A->type->code != code) return GrB_DOMAIN_MISMATCH;
    CHECK(to_dev(A));
    int info = grb_b200_dreduce(s, A->dev, monoid->opcode);
    if (info == 1) return GrB_NOT_IMPLEMENTED;
    return (GrB_Info)info;
}

#define REDUCE(T, CT, CODE) \
GrB_Info GrB_Matrix_reduce_##T(CT *s, const GrB_BinaryOp accum, \
    const GrB_Monoid monoid, const GrB_Matrix A, const GrB_Descriptor d) \
{ (void)d; return reduce_any(s, CODE, accum, monoid, A); } \
GrB_Info GrB_Vector_reduce_##T(CT *s, const GrB_BinaryOp accum, \
    const GrB_Monoid monoid, const GrB_Vector u, const GrB_Descriptor d) \
{ (void)d; if (!VOK(u)) return GrB_UNINITIALIZED_OBJECT; \
  return reduce_any(s, CODE, accum, monoid, VM(u)); }
REDUCE(BOOL, bool, 1)
REDUCE(INT32, int32_t, 6)
REDUCE(INT64, int64_t, 8)
REDUCE(FP32, float, 10)
REDUCE(FP64, double, 11)
#undef REDUCE
