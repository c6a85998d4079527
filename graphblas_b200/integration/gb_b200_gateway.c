// gb_b200_gateway.c: the binding a SuiteSparse:GraphBLAS maintainer adds to
// route the library's own GB_AxB_dot3 and GB_AxB_saxpy3 to the B200 kernels
// of libgrb_b200.so.  It is compiled with the library's internal headers
// (GB.h) and linked into the library with
//
//     -Wl,--wrap=GB_AxB_dot3 -Wl,--wrap=GB_AxB_saxpy3 -lgrb_b200
//
// so the calls from GB_AxB_dot.c:200 and GB_AxB_saxpy.c:208 land here; the
// same two functions can instead be called from the existing
// `#if GRAPHBLAS_HAS_CUDA` branch of GB_AxB_dot.c:189-197 and a new branch in
// GB_AxB_saxpy.c.  Anything the GPU does not take (hypersparse, bitmap or
// full operands, iso outputs, user types, semirings outside the compiled
// list) is declined with GrB_NO_VALUE and runs on the CPU as before.
//
// The GPU result is copied into a C built exactly as the CPU kernels build
// it (GB_new_bix with the same sizes, GB_AxB_dot3.c:172-176 and
// GB_AxB_saxpy3.c:242-244), so every later step of the library (GB_wait's
// zombie removal, GB_accum_mask, reductions) sees the same object.

#include "GB.h"
#include "mxm/GB_mxm.h"
#include "mxm/GB_AxB_saxpy3.h"
#include "grb_b200.h"

GrB_Info __real_GB_AxB_dot3 (GrB_Matrix C, const bool C_iso,
    const GB_void *cscalar, const GrB_Matrix M, const bool Mask_struct,
    const GrB_Matrix A, const GrB_Matrix B, const GrB_Semiring semiring,
    const bool flipxy, GB_Werk Werk) ;

GrB_Info __real_GB_AxB_saxpy3 (GrB_Matrix C, const bool C_iso,
    const GB_void *cscalar, int C_sparsity, const GrB_Matrix M,
    const bool Mask_comp, const bool Mask_struct, const GrB_Matrix A,
    const GrB_Matrix B, const GrB_Semiring semiring, const bool flipxy,
    bool *mask_applied, const GrB_Desc_Value AxB_method, const int do_sort,
    GB_Werk Werk) ;

// counters a test can read: how many calls the GPU took and declined
int64_t gb_b200_gateway_taken = 0, gb_b200_gateway_declined = 0 ;

static bool gb_b200_enabled (void)
{
    static int state = -1 ;
    if (state < 0)
    {
        const char *e = getenv ("GB_B200") ;
        state = (e != NULL && e [0] == '1') && (grb_b200_init ( ) == 0) ;
    }
    return state == 1 ;
}

// view a sparse, non-hypersparse GrB_Matrix with a built-in real type
static bool gb_b200_view (grb_b200_matrix *X, const GrB_Matrix A)
{
    if (A == NULL) return true ;
    if (A->h != NULL || A->b != NULL || A->p == NULL) return false ;
    if (A->nvec != A->vdim) return false ;
    int code = A->type->code ;
    if (!(code == GB_BOOL_code || code == GB_INT32_code || code == GB_UINT32_code
       || code == GB_INT64_code || code == GB_UINT64_code || code == GB_FP32_code
       || code == GB_FP64_code)) return false ;
    X->vlen = A->vlen ;
    X->vdim = A->vdim ;
    X->p = A->p ;
    X->i = A->i ;
    X->x = A->x ;
    X->type = code ;
    X->iso = A->iso ;
    X->jumbled = A->jumbled ;
    X->nzombies = A->nzombies ;
    return true ;
}

static bool gb_b200_semiring (grb_b200_semiring *s, const GrB_Semiring S)
{
    s->add_opcode = (int) S->add->op->opcode ;
    s->mult_opcode = (int) S->multiply->opcode ;
    s->type = (int) S->add->op->ztype->code ;
    // user-defined operators are not compiled for the device
    return s->add_opcode < GB_USER_binop_code && s->mult_opcode < GB_USER_binop_code ;
}

// build C like the CPU kernel does and copy the device result into it
static GrB_Info gb_b200_adopt (GrB_Matrix C, GrB_Type ctype, int64_t vlen,
    int64_t vdim, const GrB_Matrix like, grb_b200_matrix *R)
{
    GrB_Info info ;
    int64_t cnz = R->p [vdim] ;
    info = GB_new_bix (&C, ctype, vlen, vdim, GB_Ap_malloc, like->is_csc,
        GxB_SPARSE, true, like->hyper_switch, vdim, GB_IMAX (cnz, 1), true,
        false) ;
    if (info == GrB_SUCCESS)
    {
        memcpy (C->p, R->p, (vdim + 1) * sizeof (int64_t)) ;
        memcpy (C->i, R->i, cnz * sizeof (int64_t)) ;
        memcpy (C->x, R->x, cnz * ctype->size) ;
        C->nvec = vdim ;
        C->nvec_nonempty = -1 ;
        C->nvals = cnz ;
        C->nzombies = R->nzombies ;
        C->jumbled = R->jumbled ;
        C->magic = GB_MAGIC ;
    }
    free (R->p) ; free (R->i) ; free (R->x) ;
    return info ;
}

GrB_Info __wrap_GB_AxB_dot3 (GrB_Matrix C, const bool C_iso,
    const GB_void *cscalar, const GrB_Matrix M, const bool Mask_struct,
    const GrB_Matrix A, const GrB_Matrix B, const GrB_Semiring semiring,
    const bool flipxy, GB_Werk Werk)
{
    grb_b200_matrix m, a, b, r ;
    grb_b200_semiring s ;
    memset (&r, 0, sizeof (r)) ;
    if (gb_b200_enabled ( ) && !C_iso && gb_b200_view (&m, M)
        && gb_b200_view (&a, A) && gb_b200_view (&b, B)
        && M->nzombies == 0 && gb_b200_semiring (&s, semiring)
        && grb_b200_AxB_dot3_branch (&m, &a, &b, &s, flipxy))
    {
        int info = grb_b200_AxB_dot3 (&r, &m, Mask_struct, &a, &b, &s, flipxy) ;
        if (info == 0)
        {
            gb_b200_gateway_taken++ ;
            return gb_b200_adopt (C, semiring->add->op->ztype, M->vlen, M->vdim,
                M, &r) ;
        }
        if (info != GrB_NO_VALUE) return (GrB_Info) info ;
    }
    gb_b200_gateway_declined++ ;
    return __real_GB_AxB_dot3 (C, C_iso, cscalar, M, Mask_struct, A, B,
        semiring, flipxy, Werk) ;
}

GrB_Info __wrap_GB_AxB_saxpy3 (GrB_Matrix C, const bool C_iso,
    const GB_void *cscalar, int C_sparsity, const GrB_Matrix M,
    const bool Mask_comp, const bool Mask_struct, const GrB_Matrix A,
    const GrB_Matrix B, const GrB_Semiring semiring, const bool flipxy,
    bool *mask_applied, const GrB_Desc_Value AxB_method, const int do_sort,
    GB_Werk Werk)
{
    grb_b200_matrix m, a, b, r ;
    grb_b200_semiring s ;
    memset (&r, 0, sizeof (r)) ;
    if (gb_b200_enabled ( ) && !C_iso && C_sparsity == GxB_SPARSE
        && gb_b200_view (&m, M) && gb_b200_view (&a, A) && gb_b200_view (&b, B)
        && (M == NULL || M->nzombies == 0) && gb_b200_semiring (&s, semiring))
    {
        int info = grb_b200_AxB_saxpy3 (&r, M ? &m : NULL, Mask_comp, Mask_struct,
            &a, &b, &s, flipxy, mask_applied, do_sort) ;
        if (info == 0)
        {
            gb_b200_gateway_taken++ ;
            return gb_b200_adopt (C, semiring->add->op->ztype, A->vlen, B->vdim,
                B, &r) ;
        }
        if (info != GrB_NO_VALUE) return (GrB_Info) info ;
    }
    gb_b200_gateway_declined++ ;
    return __real_GB_AxB_saxpy3 (C, C_iso, cscalar, C_sparsity, M, Mask_comp,
        Mask_struct, A, B, semiring, flipxy, mask_applied, AxB_method, do_sort,
        Werk) ;
}
