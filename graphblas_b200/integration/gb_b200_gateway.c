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
// full operands, user types, semirings outside the compiled list) is
// declined with GrB_NO_VALUE and runs on the CPU as before.
//
// The product stays on the device until C has been built exactly as the CPU
// kernels build it (GB_new_bix with the same sizes, GB_AxB_dot3.c:172-176
// and GB_AxB_saxpy3.c:242-244); the device result is then copied straight
// into C's arrays, which belong to the library's allocator from the start,
// so every later step of the library (GB_wait's zombie removal,
// GB_accum_mask, reductions, GrB_free) sees its own kind of object.  An iso
// result (GB_AxB_iso.c:79: every entry the same value, cscalar) is computed
// as a pattern with the ANY_PAIR semiring - the pattern of a product does
// not depend on values - and C gets the one value.

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
    int64_t vdim, const GrB_Matrix like, grb_b200_dmatrix *R, bool C_iso,
    const GB_void *cscalar)
{
    GrB_Info info ;
    int64_t cnz = 0, nzombies = 0 ;
    grb_b200_dmatrix_info (*R, NULL, NULL, &cnz, &nzombies, NULL, NULL) ;
    info = GB_new_bix (&C, ctype, vlen, vdim, GB_Ap_malloc, like->is_csc,
        GxB_SPARSE, true, like->hyper_switch, vdim, GB_IMAX (cnz, 1), true,
        C_iso) ;
    if (info == GrB_SUCCESS)
    {
        int gi = grb_b200_dmatrix_copy_out (*R, C->p, C->i, C_iso ? NULL : C->x) ;
        if (gi != 0)
        {
            GB_phybix_free (C) ;
            info = (GrB_Info) gi ;
        }
        else
        {
            if (C_iso) memcpy (C->x, cscalar, ctype->size) ;
            C->nvec = vdim ;
            C->nvec_nonempty = -1 ;
            C->nvals = cnz ;
            C->nzombies = nzombies ;
            C->iso = C_iso ;
            C->magic = GB_MAGIC ;
        }
    }
    grb_b200_dmatrix_free (R) ;
    return info ;
}

// the semiring the device runs: the caller's, or ANY_PAIR (bool) for an iso
// result, whose pattern is all the device needs to find
static bool gb_b200_device_semiring (grb_b200_semiring *s,
    const GrB_Semiring S, bool C_iso)
{
    if (!C_iso) return gb_b200_semiring (s, S) ;
    s->add_opcode = (int) GB_ANY_binop_code ;
    s->mult_opcode = (int) GB_PAIR_binop_code ;
    s->type = (int) GB_BOOL_code ;
    return true ;
}

GrB_Info __wrap_GB_AxB_dot3 (GrB_Matrix C, const bool C_iso,
    const GB_void *cscalar, const GrB_Matrix M, const bool Mask_struct,
    const GrB_Matrix A, const GrB_Matrix B, const GrB_Semiring semiring,
    const bool flipxy, GB_Werk Werk)
{
    grb_b200_matrix m, a, b ;
    grb_b200_semiring s ;
    if (gb_b200_enabled ( ) && gb_b200_view (&m, M)
        && gb_b200_view (&a, A) && gb_b200_view (&b, B)
        && M->nzombies == 0 && gb_b200_device_semiring (&s, semiring, C_iso)
        && grb_b200_AxB_dot3_branch (&m, &a, &b, &s, flipxy))
    {
        grb_b200_dmatrix R = NULL ;
        int info = grb_b200_AxB_dot3_device (&R, &m, Mask_struct, &a, &b, &s,
            flipxy) ;
        if (info == 0)
        {
            // C keeps M's vector pointers, its zombies and M's order
            info = gb_b200_adopt (C, semiring->add->op->ztype, M->vlen,
                M->vdim, M, &R, C_iso, cscalar) ;
            if (info == GrB_SUCCESS)
            {
                C->jumbled = M->jumbled ;
                gb_b200_gateway_taken++ ;
            }
            return (GrB_Info) info ;
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
    grb_b200_matrix m, a, b ;
    grb_b200_semiring s ;
    if (gb_b200_enabled ( ) && C_sparsity == GxB_SPARSE
        && gb_b200_view (&m, M) && gb_b200_view (&a, A) && gb_b200_view (&b, B)
        && (M == NULL || M->nzombies == 0)
        && gb_b200_device_semiring (&s, semiring, C_iso))
    {
        grb_b200_dmatrix R = NULL ;
        int info = grb_b200_AxB_saxpy3_device (&R, M ? &m : NULL, Mask_comp,
            Mask_struct, &a, &b, &s, flipxy, mask_applied) ;
        if (info == 0)
        {
            // sorted, no zombies
            info = gb_b200_adopt (C, semiring->add->op->ztype, A->vlen,
                B->vdim, B, &R, C_iso, cscalar) ;
            if (info == GrB_SUCCESS)
            {
                C->jumbled = false ;
                gb_b200_gateway_taken++ ;
            }
            return (GrB_Info) info ;
        }
        if (info != GrB_NO_VALUE) return (GrB_Info) info ;
    }
    gb_b200_gateway_declined++ ;
    return __real_GB_AxB_saxpy3 (C, C_iso, cscalar, C_sparsity, M, Mask_comp,
        Mask_struct, A, B, semiring, flipxy, mask_applied, AxB_method, do_sort,
        Werk) ;
}
