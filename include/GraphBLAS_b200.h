/* GraphBLAS_b200.h: the GrB_mxm / GrB_vxm / GrB_mxv path of the GraphBLAS C
 * API (as SuiteSparse:GraphBLAS v9.3.1 defines it in Include/GraphBLAS.h),
 * served by the B200 kernels of libgrb_b200.so.
 *
 * Names, argument meaning, enum values and GrB_Info error codes follow the
 * reference header line for line where they exist there:
 *   GrB_Info                      Include/GraphBLAS.h:358-381
 *   GrB_Desc_Field / _Value       Include/GraphBLAS.h:500-540
 *   predefined descriptors        Include/GraphBLAS.h:555-600
 *   GrB_mxm / GrB_vxm / GrB_mxv   Include/GraphBLAS.h:5749 / 5760 / 5771
 *   GxB_Matrix_pack_CSR / unpack  Include/GraphBLAS.h:9449 / 9976
 *   GxB_Vector_pack_CSC / unpack  Include/GraphBLAS.h:9840 / 10206
 * Only the objects this path needs exist: matrices are by-row (CSR),
 * vectors are sparse, semirings are the built-in ones the device kernels are
 * compiled for (any other built-in combination returns GrB_NOT_IMPLEMENTED).
 *
 * Matrices live in device memory (HBM) once an operation has used them; the
 * host copy is refreshed lazily by GrB_Matrix_wait, extractTuples or unpack.
 * Results of a masked dot product keep their zombies (empty entries) until a
 * wait, exactly as the reference does (Source/wait/GB_wait.c:62).
 */
#ifndef GRAPHBLAS_B200_H
#define GRAPHBLAS_B200_H

#include <stdint.h>
#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint64_t GrB_Index;

typedef enum
{
    GrB_SUCCESS = 0,
    GrB_NO_VALUE = 1,
    GrB_UNINITIALIZED_OBJECT = -1,
    GrB_NULL_POINTER = -2,
    GrB_INVALID_VALUE = -3,
    GrB_INVALID_INDEX = -4,
    GrB_DOMAIN_MISMATCH = -5,
    GrB_DIMENSION_MISMATCH = -6,
    GrB_OUTPUT_NOT_EMPTY = -7,
    GrB_NOT_IMPLEMENTED = -8,
    GrB_ALREADY_SET = -9,
    GrB_PANIC = -101,
    GrB_OUT_OF_MEMORY = -102,
    GrB_INSUFFICIENT_SPACE = -103,
    GrB_INVALID_OBJECT = -104,
    GrB_INDEX_OUT_OF_BOUNDS = -105,
    GrB_EMPTY_OBJECT = -106
}
GrB_Info;

typedef enum { GrB_NONBLOCKING = 0, GrB_BLOCKING = 1 } GrB_Mode;
typedef enum { GrB_COMPLETE = 0, GrB_MATERIALIZE = 1 } GrB_WaitMode;

typedef enum
{
    GrB_OUTP = 0, GrB_MASK = 1, GrB_INP0 = 2, GrB_INP1 = 3,
    GxB_AxB_METHOD = 7090, GxB_SORT = 7091
}
GrB_Desc_Field;

typedef enum
{
    GrB_DEFAULT = 0, GxB_DEFAULT = 0,
    GrB_REPLACE = 1,
    GrB_COMP = 2, GrB_STRUCTURE = 4, GrB_COMP_STRUCTURE = 6,
    GrB_TRAN = 3,
    GxB_AxB_GUSTAVSON = 7081, GxB_AxB_DOT = 7083, GxB_AxB_HASH = 7084,
    GxB_AxB_SAXPY = 7085
}
GrB_Desc_Value;

typedef struct GB_Type_opaque *GrB_Type;
typedef struct GB_BinaryOp_opaque *GrB_BinaryOp;
typedef struct GB_Monoid_opaque *GrB_Monoid;
typedef struct GB_Semiring_opaque *GrB_Semiring;
typedef struct GB_Descriptor_opaque *GrB_Descriptor;
typedef struct GB_Matrix_opaque *GrB_Matrix;
typedef struct GB_Vector_opaque *GrB_Vector;

/* built-in types */
extern GrB_Type GrB_BOOL, GrB_INT32, GrB_UINT32, GrB_INT64, GrB_UINT64,
    GrB_FP32, GrB_FP64;

/* binary operators (accumulators and multipliers) */
#define GRB_B200_OPS_OF(T) \
    GrB_FIRST_##T, GrB_SECOND_##T, GrB_PLUS_##T, GrB_MINUS_##T, \
    GrB_TIMES_##T, GrB_MIN_##T, GrB_MAX_##T, GxB_PAIR_##T, GxB_ANY_##T
extern GrB_BinaryOp GRB_B200_OPS_OF(BOOL), GRB_B200_OPS_OF(INT32),
    GRB_B200_OPS_OF(INT64), GRB_B200_OPS_OF(FP32), GRB_B200_OPS_OF(FP64),
    GrB_LOR, GrB_LAND, GrB_LXOR,
    GxB_FIRSTI_INT32, GxB_FIRSTI_INT64, GxB_FIRSTJ_INT32, GxB_FIRSTJ_INT64,
    GxB_SECONDI_INT32, GxB_SECONDI_INT64, GxB_SECONDJ_INT32, GxB_SECONDJ_INT64;

/* monoids */
#define GRB_B200_MONOIDS_OF(T) \
    GrB_PLUS_MONOID_##T, GrB_TIMES_MONOID_##T, GrB_MIN_MONOID_##T, \
    GrB_MAX_MONOID_##T, GxB_ANY_##T##_MONOID
extern GrB_Monoid GRB_B200_MONOIDS_OF(INT32), GRB_B200_MONOIDS_OF(INT64),
    GRB_B200_MONOIDS_OF(FP32), GRB_B200_MONOIDS_OF(FP64),
    GrB_LOR_MONOID_BOOL, GrB_LAND_MONOID_BOOL, GxB_ANY_BOOL_MONOID;

/* built-in semirings compiled for the device (Include/GraphBLAS.h:2037-2545
 * names) */
extern GrB_Semiring
    GrB_PLUS_TIMES_SEMIRING_FP64, GrB_PLUS_TIMES_SEMIRING_FP32,
    GrB_PLUS_TIMES_SEMIRING_INT64, GrB_PLUS_TIMES_SEMIRING_INT32,
    GxB_PLUS_PAIR_INT64, GxB_PLUS_PAIR_INT32, GxB_PLUS_PAIR_FP64,
    GrB_MIN_PLUS_SEMIRING_FP32, GrB_MIN_PLUS_SEMIRING_FP64,
    GrB_MIN_PLUS_SEMIRING_INT64, GrB_MIN_PLUS_SEMIRING_INT32,
    GrB_MAX_PLUS_SEMIRING_FP64, GrB_MAX_PLUS_SEMIRING_FP32,
    GrB_MIN_TIMES_SEMIRING_FP64, GrB_MAX_TIMES_SEMIRING_FP64,
    GrB_MIN_SECOND_SEMIRING_FP32, GrB_MIN_SECOND_SEMIRING_FP64,
    GrB_MIN_FIRST_SEMIRING_FP32, GrB_MIN_FIRST_SEMIRING_FP64,
    GxB_PLUS_FIRST_FP64, GxB_PLUS_SECOND_FP64,
    GxB_ANY_SECONDI_INT64, GxB_ANY_FIRSTJ_INT64, GxB_ANY_FIRSTI_INT64,
    GxB_ANY_SECONDJ_INT64, GxB_ANY_SECONDI_INT32, GxB_ANY_FIRSTJ_INT32,
    GxB_MIN_SECONDI_INT64, GxB_MIN_FIRSTJ_INT64, GxB_MIN_FIRSTI_INT64,
    GxB_MIN_SECONDJ_INT64, GxB_MAX_SECONDI_INT64, GxB_MAX_FIRSTJ_INT64,
    GxB_ANY_PAIR_BOOL, GrB_LOR_LAND_SEMIRING_BOOL, GxB_ANY_PAIR_INT64,
    GxB_ANY_TIMES_FP64;

/* predefined descriptors (Include/GraphBLAS.h:555-600) */
extern GrB_Descriptor
    GrB_DESC_T1, GrB_DESC_T0, GrB_DESC_T0T1,
    GrB_DESC_C, GrB_DESC_CT1, GrB_DESC_CT0, GrB_DESC_CT0T1,
    GrB_DESC_S, GrB_DESC_ST1, GrB_DESC_ST0, GrB_DESC_ST0T1,
    GrB_DESC_SC, GrB_DESC_SCT1, GrB_DESC_SCT0, GrB_DESC_SCT0T1,
    GrB_DESC_R, GrB_DESC_RT1, GrB_DESC_RT0, GrB_DESC_RT0T1,
    GrB_DESC_RC, GrB_DESC_RCT1, GrB_DESC_RCT0, GrB_DESC_RCT0T1,
    GrB_DESC_RS, GrB_DESC_RST1, GrB_DESC_RST0, GrB_DESC_RST0T1,
    GrB_DESC_RSC, GrB_DESC_RSCT1, GrB_DESC_RSCT0, GrB_DESC_RSCT0T1;

/* "all indices" for GrB_assign */
extern const GrB_Index *GrB_ALL;

/* ---- context ---- */
GrB_Info GrB_init(GrB_Mode mode);
GrB_Info GrB_finalize(void);

/* ---- algebra ---- */
GrB_Info GrB_Semiring_new(GrB_Semiring *semiring, GrB_Monoid add,
                          GrB_BinaryOp multiply);
GrB_Info GrB_Semiring_free(GrB_Semiring *semiring);
GrB_Info GrB_Descriptor_new(GrB_Descriptor *desc);
GrB_Info GrB_Descriptor_set(GrB_Descriptor desc, GrB_Desc_Field field,
                            GrB_Desc_Value val);
GrB_Info GrB_Descriptor_free(GrB_Descriptor *desc);

/* ---- matrices (by row) ---- */
GrB_Info GrB_Matrix_new(GrB_Matrix *A, GrB_Type type, GrB_Index nrows,
                        GrB_Index ncols);
GrB_Info GrB_Matrix_free(GrB_Matrix *A);
GrB_Info GrB_Matrix_dup(GrB_Matrix *C, const GrB_Matrix A);
GrB_Info GrB_Matrix_clear(GrB_Matrix A);
GrB_Info GrB_Matrix_nrows(GrB_Index *nrows, const GrB_Matrix A);
GrB_Info GrB_Matrix_ncols(GrB_Index *ncols, const GrB_Matrix A);
GrB_Info GrB_Matrix_nvals(GrB_Index *nvals, const GrB_Matrix A);
GrB_Info GrB_Matrix_wait(GrB_Matrix A, GrB_WaitMode mode);
GrB_Info GxB_Matrix_pack_CSR(GrB_Matrix A, GrB_Index **Ap, GrB_Index **Aj,
                             void **Ax, GrB_Index Ap_size, GrB_Index Aj_size,
                             GrB_Index Ax_size, bool iso, bool jumbled,
                             const GrB_Descriptor desc);
GrB_Info GxB_Matrix_unpack_CSR(GrB_Matrix A, GrB_Index **Ap, GrB_Index **Aj,
                               void **Ax, GrB_Index *Ap_size,
                               GrB_Index *Aj_size, GrB_Index *Ax_size,
                               bool *iso, bool *jumbled,
                               const GrB_Descriptor desc);
#define GRB_B200_EXTRACT(T, CT) \
    GrB_Info GrB_Matrix_extractTuples_##T(GrB_Index *I, GrB_Index *J, CT *X, \
                                          GrB_Index *nvals, const GrB_Matrix A);
GRB_B200_EXTRACT(BOOL, bool)
GRB_B200_EXTRACT(INT32, int32_t)
GRB_B200_EXTRACT(INT64, int64_t)
GRB_B200_EXTRACT(FP32, float)
GRB_B200_EXTRACT(FP64, double)
#undef GRB_B200_EXTRACT

/* ---- import / export (copies; GrB_CSR_FORMAT) ---- */
typedef enum { GrB_CSR_FORMAT = 0, GrB_CSC_FORMAT = 1, GrB_COO_FORMAT = 2 } GrB_Format;
#define GRB_B200_IMPORT(T, CT) \
    GrB_Info GrB_Matrix_import_##T(GrB_Matrix *A, GrB_Type type, GrB_Index nrows, \
        GrB_Index ncols, const GrB_Index *Ap, const GrB_Index *Ai, const CT *Ax, \
        GrB_Index Ap_len, GrB_Index Ai_len, GrB_Index Ax_len, GrB_Format format); \
    GrB_Info GrB_Matrix_export_##T(GrB_Index *Ap, GrB_Index *Ai, CT *Ax, \
        GrB_Index *Ap_len, GrB_Index *Ai_len, GrB_Index *Ax_len, GrB_Format format, \
        GrB_Matrix A);
GRB_B200_IMPORT(BOOL, bool)
GRB_B200_IMPORT(INT32, int32_t)
GRB_B200_IMPORT(UINT32, uint32_t)
GRB_B200_IMPORT(INT64, int64_t)
GRB_B200_IMPORT(UINT64, uint64_t)
GRB_B200_IMPORT(FP32, float)
GRB_B200_IMPORT(FP64, double)
#undef GRB_B200_IMPORT
GrB_Info GrB_Matrix_exportSize(GrB_Index *Ap_len, GrB_Index *Ai_len,
                               GrB_Index *Ax_len, GrB_Format format, GrB_Matrix A);

/* ---- serialize / deserialize (the reference's blob format) ----
 * Blobs written here are uncompressed (GxB_COMPRESSION_NONE); blobs read may
 * also be LZ4 / LZ4HC compressed.  ZSTD blobs give GrB_NOT_IMPLEMENTED.  The
 * descriptor arguments are accepted and ignored. */
GrB_Info GrB_Matrix_serializeSize(GrB_Index *blob_size_handle, GrB_Matrix A);
GrB_Info GrB_Matrix_serialize(void *blob, GrB_Index *blob_size_handle, GrB_Matrix A);
GrB_Info GxB_Matrix_serialize(void **blob_handle, GrB_Index *blob_size_handle,
                              GrB_Matrix A, const GrB_Descriptor desc);
GrB_Info GrB_Matrix_deserialize(GrB_Matrix *C, GrB_Type type, const void *blob,
                                GrB_Index blob_size);
GrB_Info GxB_Matrix_deserialize(GrB_Matrix *C, GrB_Type type, const void *blob,
                                GrB_Index blob_size, const GrB_Descriptor desc);
GrB_Info GxB_Vector_serialize(void **blob_handle, GrB_Index *blob_size_handle,
                              GrB_Vector u, const GrB_Descriptor desc);
GrB_Info GxB_Vector_deserialize(GrB_Vector *w, GrB_Type type, const void *blob,
                                GrB_Index blob_size, const GrB_Descriptor desc);

/* ---- vectors (sparse) ---- */
GrB_Info GrB_Vector_new(GrB_Vector *v, GrB_Type type, GrB_Index n);
GrB_Info GrB_Vector_free(GrB_Vector *v);
GrB_Info GrB_Vector_dup(GrB_Vector *w, const GrB_Vector u);
GrB_Info GrB_Vector_clear(GrB_Vector v);
GrB_Info GrB_Vector_size(GrB_Index *n, const GrB_Vector v);
GrB_Info GrB_Vector_nvals(GrB_Index *nvals, const GrB_Vector v);
GrB_Info GrB_Vector_wait(GrB_Vector v, GrB_WaitMode mode);
GrB_Info GrB_Vector_setElement_BOOL(GrB_Vector w, bool x, GrB_Index i);
GrB_Info GrB_Vector_setElement_INT32(GrB_Vector w, int32_t x, GrB_Index i);
GrB_Info GrB_Vector_setElement_INT64(GrB_Vector w, int64_t x, GrB_Index i);
GrB_Info GrB_Vector_setElement_FP32(GrB_Vector w, float x, GrB_Index i);
GrB_Info GrB_Vector_setElement_FP64(GrB_Vector w, double x, GrB_Index i);
GrB_Info GxB_Vector_pack_CSC(GrB_Vector v, GrB_Index **vi, void **vx,
                             GrB_Index vi_size, GrB_Index vx_size, bool iso,
                             GrB_Index nvals, bool jumbled,
                             const GrB_Descriptor desc);
GrB_Info GxB_Vector_unpack_CSC(GrB_Vector v, GrB_Index **vi, void **vx,
                               GrB_Index *vi_size, GrB_Index *vx_size,
                               bool *iso, GrB_Index *nvals, bool *jumbled,
                               const GrB_Descriptor desc);
#define GRB_B200_VEXTRACT(T, CT) \
    GrB_Info GrB_Vector_extractTuples_##T(GrB_Index *I, CT *X, \
                                          GrB_Index *nvals, const GrB_Vector v);
GRB_B200_VEXTRACT(BOOL, bool)
GRB_B200_VEXTRACT(INT32, int32_t)
GRB_B200_VEXTRACT(INT64, int64_t)
GRB_B200_VEXTRACT(FP32, float)
GRB_B200_VEXTRACT(FP64, double)
#undef GRB_B200_VEXTRACT

/* ---- the multiply path ---- */
GrB_Info GrB_mxm(GrB_Matrix C, const GrB_Matrix Mask, const GrB_BinaryOp accum,
                 const GrB_Semiring semiring, const GrB_Matrix A,
                 const GrB_Matrix B, const GrB_Descriptor desc);
GrB_Info GrB_vxm(GrB_Vector w, const GrB_Vector mask, const GrB_BinaryOp accum,
                 const GrB_Semiring semiring, const GrB_Vector u,
                 const GrB_Matrix A, const GrB_Descriptor desc);
GrB_Info GrB_mxv(GrB_Vector w, const GrB_Vector mask, const GrB_BinaryOp accum,
                 const GrB_Semiring semiring, const GrB_Matrix A,
                 const GrB_Vector u, const GrB_Descriptor desc);

/* ---- the callers on either side of it ---- */
/* w<mask> = accum (w, u) over all indices (GrB_Vector_assign with GrB_ALL) */
GrB_Info GrB_Vector_assign(GrB_Vector w, const GrB_Vector mask,
                           const GrB_BinaryOp accum, const GrB_Vector u,
                           const GrB_Index *I, GrB_Index ni,
                           const GrB_Descriptor desc);
/* s = accum (s, reduce (A)) with a monoid; accum must be NULL here */
#define GRB_B200_REDUCE(T, CT) \
    GrB_Info GrB_Matrix_reduce_##T(CT *s, const GrB_BinaryOp accum, \
        const GrB_Monoid monoid, const GrB_Matrix A, const GrB_Descriptor d); \
    GrB_Info GrB_Vector_reduce_##T(CT *s, const GrB_BinaryOp accum, \
        const GrB_Monoid monoid, const GrB_Vector u, const GrB_Descriptor d);
GRB_B200_REDUCE(BOOL, bool)
GRB_B200_REDUCE(INT32, int32_t)
GRB_B200_REDUCE(INT64, int64_t)
GRB_B200_REDUCE(FP32, float)
GRB_B200_REDUCE(FP64, double)
#undef GRB_B200_REDUCE

#ifdef __cplusplus
}
#endif

#endif
