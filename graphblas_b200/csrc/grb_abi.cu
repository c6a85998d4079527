// grb_abi.cu: the extern "C" entry points declared in include/grb_b200.h.
//
// The drop-in calls take matrices in the reference's internal orientation: a
// matrix is a set of vectors (columns of a CSC matrix inside the library).
// The device kernels work on rows, so each call maps the reference's problem
// onto row form:
//   dot3   C(i,j) = A(:,i)'*B(:,j) for i in M(:,j)  ->  row j of B . row i of A
//          for entry i of mask row j: kernel A := ref B, kernel B := ref A;
//   saxpy3 C(:,j) = sum_k A(:,k) B(k,j)             ->  row j of C = sum over
//          entries k of row j of B of B(k,j) * row k of A: kernel A := ref B,
//          kernel B := ref A.
// Both swap the operands of the multiplier, so a non-commutative multiplier
// is flipped (FIRST <-> SECOND, MINUS <-> RMINUS) unless the caller already
// asked for flipxy, and the positional multipliers exchange their row/column
// meaning (FIRSTI <-> SECONDJ; FIRSTJ and SECONDI both give k), the same
// rewrite GB_flip_binop performs (Source/binaryop/GB_flip_binop.c:13).

#include <cstdlib>
#include <cstring>
#include "../../include/grb_b200.h"
#include "grb_runtime.h"

using namespace grb;

static grb_b200_malloc_fn g_malloc = malloc;
static grb_b200_free_fn g_free = free;

// A device matrix.  sum_ok: `sum` is the PLUS reduction of its live entries,
// computed by the kernels that produced it (the counting dot3 path); every
// entry point that changes the matrix in place clears it.
struct grb_b200_dmatrix_s { DevCSR A; bool sum_ok = false; int64_t sum = 0; };

namespace {

// the caller's stream for this thread if one was set, else a pooled stream
struct StreamGuard {
    cudaStream_t s;
    bool pooled;
    StreamGuard() {
        s = thread_stream();
        pooled = (s == nullptr);
        if (pooled) s = stream_acquire();
    }
    ~StreamGuard() {
        if (prof_on()) { cudaStreamSynchronize(s); prof_flush(); }
        if (pooled) stream_release(s);
    }
};

// multiplier opcode after swapping the operands (a, b) -> (b, a)
int swap_mult(int op, bool flipxy, bool *ok)
{
    *ok = true;
    const bool positional = (op >= OP_FIRSTI && op <= OP_SECONDJ1);
    if (positional) {
        if (flipxy) { *ok = false; return op; }   // the library pre-flips these
        switch (op) {
            case OP_FIRSTI: return OP_SECONDJ;
            case OP_SECONDJ: return OP_FIRSTI;
            case OP_FIRSTJ: return OP_SECONDI;
            case OP_SECONDI: return OP_FIRSTJ;
            default: *ok = false; return op;      // the 1-based variants
        }
    }
    const bool flip = !flipxy;            // the swap flips; flipxy flips back
    if (!flip) return op;
    switch (op) {
        case OP_FIRST: return OP_SECOND;
        case OP_SECOND: return OP_FIRST;
        case OP_MINUS: return OP_RMINUS;
        case OP_RMINUS: return OP_MINUS;
        case OP_DIV: *ok = false; return op;
        default: return op;                // commutative
    }
}

int upload(DevCSR &D, const grb_b200_matrix *A, cudaStream_t s)
{
    if (!A || !A->p) return NULL_POINTER;
    if (A->jumbled) return NO_VALUE;
    return dev_upload(D, A->vdim, A->vlen, A->p, A->i, A->x, A->type,
                      A->iso || A->x == nullptr, s);
}

// pattern-only uploads get an iso value of one of their type
int ensure_values(DevCSR &D, cudaStream_t s)
{
    if (D.x) return SUCCESS;
    size_t ts = type_size(D.type);
    if (ts == 0) return NO_VALUE;
    D.x = dalloc(ts, s);
    if (!D.x) return OUT_OF_MEMORY;
    unsigned char one[8] = {0};
    switch (D.type) {
        case T_FP32: { float f = 1.0f; memcpy(one, &f, 4); break; }
        case T_FP64: { double d = 1.0; memcpy(one, &d, 8); break; }
        default: one[0] = 1; break;      // little-endian integer / bool one
    }
    cudaMemcpyAsync(D.x, one, ts, cudaMemcpyHostToDevice, s);
    D.iso = true;
    return SUCCESS;
}

bool types_ok(const grb_b200_matrix *A, const grb_b200_semiring *sr, int op_pos)
{
    // operands must have the monoid's type unless their values are not read
    const int m = sr->mult_opcode;
    const bool positional = (m >= OP_FIRSTI && m <= OP_SECONDJ1);
    if (positional || m == OP_PAIR) return true;
    if (m == OP_FIRST && op_pos == 1) return true;
    if (m == OP_SECOND && op_pos == 0) return true;
    return A->type == sr->type;
}

}  // namespace

extern "C" {

int grb_b200_init(void) { return init_device(); }

int grb_b200_finalize(void)
{
    cudaDeviceSynchronize();
    int dev = runtime().device;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
        cudaMemPoolTrimTo(pool, 0);
    return SUCCESS;
}

void grb_b200_set_allocator(grb_b200_malloc_fn m, grb_b200_free_fn f)
{
    g_malloc = m ? m : malloc;
    g_free = f ? f : free;
}

void grb_b200_debug_fail_alloc(int64_t n) { set_alloc_fail_countdown(n); }

void grb_b200_set_stream(void *stream) { set_thread_stream((cudaStream_t)stream); }

int grb_b200_stream_keep_scratch(void *stream, bool keep)
{
    if (!stream) return NULL_POINTER;
    if (keep) stream_scratch_enable((cudaStream_t)stream);
    else stream_scratch_release((cudaStream_t)stream);
    return SUCCESS;
}

void grb_b200_profile_enable(bool on) { prof_enable(on); }

int grb_b200_profile_select(const char *kernel, int every)
{
    if (every < 1) return INVALID_VALUE;
    prof_select(kernel, every);
    return SUCCESS;
}

void grb_b200_profile_reset(void) { prof_reset(); }

int grb_b200_profile(const char *kernel, double *total_ms, int64_t *launches)
{
    if (!kernel || !total_ms || !launches) return NULL_POINTER;
    return prof_read(kernel, total_ms, launches) ? SUCCESS : NO_VALUE;
}

bool grb_b200_AxB_dot3_branch(const grb_b200_matrix *M, const grb_b200_matrix *A,
                              const grb_b200_matrix *B,
                              const grb_b200_semiring *semiring, bool flipxy)
{
    if (!M || !A || !B || !semiring) return false;
    if (A->jumbled || B->jumbled) return false;
    bool ok;
    int mult = swap_mult(semiring->mult_opcode, flipxy, &ok);
    if (!ok) return false;
    SemiringCode sc{semiring->add_opcode, mult, semiring->type};
    if (!semiring_supported(sc)) return false;
    if (!types_ok(A, semiring, 0) || !types_ok(B, semiring, 1)) return false;
    const int64_t lim = INT32_MAX;
    if (A->vdim >= lim || B->vdim >= lim || M->vdim >= lim || A->vlen >= lim ||
        A->p[A->vdim] >= lim || B->p[B->vdim] >= lim || M->p[M->vdim] >= lim)
        return false;
    return true;
}

int grb_b200_AxB_dot3_device(grb_b200_dmatrix *C, const grb_b200_matrix *M,
                             bool Mask_struct, const grb_b200_matrix *A,
                             const grb_b200_matrix *B,
                             const grb_b200_semiring *semiring, bool flipxy)
{
    if (!C || !M || !A || !B || !semiring) return NULL_POINTER;
    int info = init_device();
    if (info != SUCCESS) return info;
    if (!grb_b200_AxB_dot3_branch(M, A, B, semiring, flipxy)) return NO_VALUE;
    if (A->vlen != B->vlen || M->vlen != A->vdim || M->vdim != B->vdim)
        return DIMENSION_MISMATCH;
    bool ok;
    SemiringCode sc{semiring->add_opcode,
                    swap_mult(semiring->mult_opcode, flipxy, &ok), semiring->type};
    StreamGuard g;
    cudaStream_t s = g.s;
    DevCSR dM, dA, dB;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    // kernel rows: mask row j, kernel A := reference B, kernel B := reference A
    grb_b200_matrix Mu = *M;
    Mu.jumbled = false;                 // the dot3 kernel reads M in any order
    if ((info = upload(dM, &Mu, s)) == SUCCESS &&
        (info = upload(dA, B, s)) == SUCCESS &&
        (info = upload(dB, A, s)) == SUCCESS &&
        (info = ensure_values(dA, s)) == SUCCESS &&
        (info = ensure_values(dB, s)) == SUCCESS) {
        bool mstruct = Mask_struct || M->x == nullptr;
        info = dot3(h->A, dM, mstruct, dA, dB, sc, s);
    }
    dev_free(dM, s); dev_free(dA, s); dev_free(dB, s);
    cudaStreamSynchronize(s);
    if (info != SUCCESS) { delete h; return info; }
    *C = h;
    return SUCCESS;
}

int grb_b200_dmatrix_copy_out(grb_b200_dmatrix D, int64_t *p, int64_t *i, void *x)
{
    if (!D || !p || !i) return NULL_POINTER;
    StreamGuard g;
    return dev_copy_out(D->A, p, i, x, g.s);
}

int grb_b200_AxB_dot3(grb_b200_matrix *C, const grb_b200_matrix *M,
                      bool Mask_struct, const grb_b200_matrix *A,
                      const grb_b200_matrix *B,
                      const grb_b200_semiring *semiring, bool flipxy)
{
    if (!C) return NULL_POINTER;
    grb_b200_dmatrix D = nullptr;
    int info = grb_b200_AxB_dot3_device(&D, M, Mask_struct, A, B, semiring, flipxy);
    if (info != SUCCESS) return info;
    const int64_t n = D->A.nrows, nnz = D->A.nnz;
    const size_t ts = type_size(D->A.type);
    int64_t *p = (int64_t *)g_malloc((size_t)(n + 1) * 8);
    int64_t *i = (int64_t *)g_malloc((size_t)(nnz ? nnz : 1) * 8);
    void *x = g_malloc((size_t)(nnz ? nnz : 1) * ts);
    info = (p && i && x) ? grb_b200_dmatrix_copy_out(D, p, i, x) : OUT_OF_MEMORY;
    const int64_t nz = D->A.nzombies;
    grb_b200_dmatrix_free(&D);
    if (info != SUCCESS) {
        if (p) g_free(p);
        if (i) g_free(i);
        if (x) g_free(x);
        return info;
    }
    // C keeps M's vector pointers (the kernel copied them) and M's order
    C->vlen = M->vlen; C->vdim = M->vdim;
    C->p = p; C->i = i; C->x = x;
    C->type = semiring->type; C->iso = false;
    C->jumbled = M->jumbled; C->nzombies = nz;
    return SUCCESS;
}

int grb_b200_AxB_saxpy3_device(grb_b200_dmatrix *C, const grb_b200_matrix *M,
                               bool Mask_comp, bool Mask_struct,
                               const grb_b200_matrix *A, const grb_b200_matrix *B,
                               const grb_b200_semiring *semiring, bool flipxy,
                               bool *mask_applied)
{
    if (!C || !A || !B || !semiring) return NULL_POINTER;
    int info = init_device();
    if (info != SUCCESS) return info;
    bool ok;
    SemiringCode sc{semiring->add_opcode,
                    swap_mult(semiring->mult_opcode, flipxy, &ok), semiring->type};
    if (!ok || !semiring_supported(sc)) return NO_VALUE;
    if (!types_ok(A, semiring, 0) || !types_ok(B, semiring, 1)) return NO_VALUE;
    if (A->jumbled || B->jumbled) return NO_VALUE;
    // reference: A is vlen-by-vdim(A), B is vdim(A)-by-vdim(B) (vectors = columns)
    if (A->vdim != B->vlen) return DIMENSION_MISMATCH;
    if (M && (M->vlen != A->vlen || M->vdim != B->vdim)) return DIMENSION_MISMATCH;
    StreamGuard g;
    cudaStream_t s = g.s;
    DevCSR dM, dA, dB;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    info = upload(dA, B, s);                       // kernel rows: vectors of B
    if (info == SUCCESS) info = upload(dB, A, s);  // gathered rows: vectors of A
    if (info == SUCCESS && M) {
        grb_b200_matrix Mu = *M;
        Mu.jumbled = false;           // mask rows are scattered, order is free
        info = upload(dM, &Mu, s);
    }
    if (info == SUCCESS) info = ensure_values(dA, s);
    if (info == SUCCESS) info = ensure_values(dB, s);
    if (info == SUCCESS) {
        bool mstruct = Mask_struct || (M && M->x == nullptr);
        info = saxpy3(h->A, M ? &dM : nullptr, Mask_comp, mstruct, dA, dB, sc, s);
    }
    dev_free(dM, s); dev_free(dA, s); dev_free(dB, s);
    cudaStreamSynchronize(s);
    if (info != SUCCESS) { dev_free(h->A, s); delete h; return info; }
    if (mask_applied) *mask_applied = (M != nullptr);
    *C = h;
    return SUCCESS;
}

int grb_b200_AxB_saxpy3(grb_b200_matrix *C, const grb_b200_matrix *M,
                        bool Mask_comp, bool Mask_struct,
                        const grb_b200_matrix *A, const grb_b200_matrix *B,
                        const grb_b200_semiring *semiring, bool flipxy,
                        bool *mask_applied, int do_sort)
{
    (void)do_sort;
    if (!C) return NULL_POINTER;
    grb_b200_dmatrix D = nullptr;
    int info = grb_b200_AxB_saxpy3_device(&D, M, Mask_comp, Mask_struct, A, B, semiring,
                                          flipxy, mask_applied);
    if (info != SUCCESS) return info;
    const int64_t n = D->A.nrows, nnz = D->A.nnz;
    const size_t ts = type_size(D->A.type);
    int64_t *p = (int64_t *)g_malloc((size_t)(n + 1) * 8);
    int64_t *i = (int64_t *)g_malloc((size_t)(nnz ? nnz : 1) * 8);
    void *x = g_malloc((size_t)(nnz ? nnz : 1) * ts);
    info = (p && i && x) ? grb_b200_dmatrix_copy_out(D, p, i, x) : OUT_OF_MEMORY;
    grb_b200_dmatrix_free(&D);
    if (info != SUCCESS) {
        if (p) g_free(p);
        if (i) g_free(i);
        if (x) g_free(x);
        return info;
    }
    C->vlen = A->vlen; C->vdim = B->vdim;
    C->p = p; C->i = i; C->x = x;
    C->type = semiring->type; C->iso = false; C->jumbled = false;
    C->nzombies = 0;
    return SUCCESS;
}

int grb_b200_reduce_to_scalar(void *out, const grb_b200_matrix *A, int monoid_opcode)
{
    if (!out || !A) return NULL_POINTER;
    int info = init_device();
    if (info != SUCCESS) return info;
    StreamGuard g;
    cudaStream_t s = g.s;
    DevCSR dA;
    grb_b200_matrix Au = *A;
    Au.jumbled = false;                  // order does not matter for a reduce
    info = upload(dA, &Au, s);
    if (info == SUCCESS) info = ensure_values(dA, s);
    if (info == SUCCESS) info = reduce_scalar(out, dA, monoid_opcode, s);
    dev_free(dA, s);
    cudaStreamSynchronize(s);
    return info;
}

// ---------------------------------------------------------------------------
// device-resident matrices
// ---------------------------------------------------------------------------

int grb_b200_dmatrix_upload(grb_b200_dmatrix *D, int64_t nrows, int64_t ncols,
                            const int64_t *p, const int64_t *i, const void *x,
                            int type, bool iso)
{
    if (!D || !p) return NULL_POINTER;
    int info = init_device();
    if (info != SUCCESS) return info;
    if (type_size(type) == 0) return INVALID_VALUE;
    StreamGuard g;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    info = dev_upload(h->A, nrows, ncols, p, i, x, type, iso || x == nullptr, g.s);
    if (info == SUCCESS) info = ensure_values(h->A, g.s);
    cudaError_t e = cudaStreamSynchronize(g.s);
    if (info == SUCCESS && e != cudaSuccess) info = cuda_to_info(e);
    if (info != SUCCESS) { dev_free(h->A, g.s); delete h; return info; }
    *D = h;
    return SUCCESS;
}

int grb_b200_dmatrix_download(grb_b200_dmatrix D, int64_t **p, int64_t **i,
                              void **x, bool prune)
{
    if (!D || !p || !i || !x) return NULL_POINTER;
    StreamGuard g;
    return dev_download(D->A, p, i, x, !prune, g_malloc, g.s);
}

int grb_b200_dmatrix_import(grb_b200_dmatrix *D, int64_t nrows, int64_t ncols,
                            const int64_t *p, const int64_t *i, const void *x, int type)
{
    if (!D || !p || !i || !x) return NULL_POINTER;
    *D = nullptr;
    int info = init_device();
    if (info != SUCCESS) return info;
    if (type_size(type) == 0) return INVALID_VALUE;
    StreamGuard g;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    info = dev_import(h->A, nrows, ncols, p, i, x, type, g.s);
    if (info != SUCCESS) { delete h; return info; }
    *D = h;
    return SUCCESS;
}

int grb_b200_dmatrix_export(grb_b200_dmatrix D, int64_t *p, int64_t *i, void *x)
{
    if (!D || !p || !i) return NULL_POINTER;
    StreamGuard g;
    return dev_download_to(D->A, p, i, x, g.s);
}

int grb_b200_dmatrix_free(grb_b200_dmatrix *D)
{
    if (!D || !*D) return SUCCESS;
    StreamGuard g;
    dev_free((*D)->A, g.s);
    cudaStreamSynchronize(g.s);
    delete *D;
    *D = nullptr;
    return SUCCESS;
}

int grb_b200_dmatrix_info(grb_b200_dmatrix D, int64_t *nrows, int64_t *ncols,
                          int64_t *nnz, int64_t *nzombies, int *type, bool *iso)
{
    if (!D) return NULL_POINTER;
    if (nrows) *nrows = D->A.nrows;
    if (ncols) *ncols = D->A.ncols;
    if (nnz) *nnz = D->A.nnz;
    if (nzombies) *nzombies = D->A.nzombies;
    if (type) *type = D->A.type;
    if (iso) *iso = D->A.iso;
    return SUCCESS;
}

int grb_b200_dmxm_dot3(grb_b200_dmatrix *C, grb_b200_dmatrix M, bool mask_struct,
                       grb_b200_dmatrix A, grb_b200_dmatrix B,
                       const grb_b200_semiring *sr)
{
    if (!C || !M || !A || !B || !sr) return NULL_POINTER;
    StreamGuard g;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    SemiringCode sc{sr->add_opcode, sr->mult_opcode, sr->type};
    int64_t live = 0;
    int info = dot3(h->A, M->A, mask_struct, A->A, B->A, sc, g.s, &live);
    if (info != SUCCESS) { delete h; return info; }
    // the counting semirings (PLUS_PAIR on integers) bring C's sum along
    const bool counting = sr->add_opcode == OP_PLUS && sr->mult_opcode == OP_PAIR &&
        (sr->type == T_INT32 || sr->type == T_UINT32 || sr->type == T_INT64 ||
         sr->type == T_UINT64);
    h->sum_ok = counting;
    h->sum = live;
    *C = h;
    return SUCCESS;
}

int grb_b200_dmxm_saxpy3(grb_b200_dmatrix *C, grb_b200_dmatrix M, bool mask_comp,
                         bool mask_struct, grb_b200_dmatrix A, grb_b200_dmatrix B,
                         const grb_b200_semiring *sr)
{
    if (!C || !A || !B || !sr) return NULL_POINTER;
    StreamGuard g;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    SemiringCode sc{sr->add_opcode, sr->mult_opcode, sr->type};
    int info = saxpy3(h->A, M ? &M->A : nullptr, mask_comp, mask_struct, A->A,
                      B->A, sc, g.s);
    if (info != SUCCESS) { delete h; return info; }
    *C = h;
    return SUCCESS;
}

int grb_b200_dreduce(void *out, grb_b200_dmatrix D, int monoid_opcode)
{
    if (!out || !D) return NULL_POINTER;
    if (D->sum_ok && monoid_opcode == OP_PLUS) {
        // the sum the producing kernels accumulated, wrapped to the type as
        // the reduction's own integer adds would wrap
        switch (D->A.type) {
            case T_INT64: case T_UINT64: memcpy(out, &D->sum, 8); return SUCCESS;
            case T_INT32: case T_UINT32: {
                const uint32_t v = (uint32_t)(uint64_t)D->sum;
                memcpy(out, &v, 4);
                return SUCCESS;
            }
            default: break;
        }
    }
    StreamGuard g;
    return reduce_scalar(out, D->A, monoid_opcode, g.s);
}

int grb_b200_dmatrix_empty(grb_b200_dmatrix *D, int64_t nrows, int64_t ncols,
                           int type)
{
    if (!D) return NULL_POINTER;
    int info = init_device();
    if (info != SUCCESS) return info;
    if (type_size(type) == 0) return INVALID_VALUE;
    if (nrows >= INT32_MAX || ncols >= INT32_MAX) return NO_VALUE;
    StreamGuard g;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    h->A.nrows = nrows; h->A.ncols = ncols; h->A.nnz = 0; h->A.type = type;
    h->A.p = (int32_t *)dalloc((size_t)(nrows + 1) * 4, g.s);
    h->A.j = (int32_t *)dalloc(4, g.s);
    h->A.x = dalloc(type_size(type), g.s);
    if (!h->A.p || !h->A.j || !h->A.x) { dev_free(h->A, g.s); delete h; return OUT_OF_MEMORY; }
    cudaMemsetAsync(h->A.p, 0, (size_t)(nrows + 1) * 4, g.s);
    cudaError_t e = cudaStreamSynchronize(g.s);
    if (e != cudaSuccess) { dev_free(h->A, g.s); delete h; return cuda_to_info(e); }
    *D = h;
    return SUCCESS;
}

int grb_b200_dmatrix_dup(grb_b200_dmatrix *D, grb_b200_dmatrix A)
{
    if (!D || !A) return NULL_POINTER;
    StreamGuard g;
    cudaStream_t s = g.s;
    const DevCSR &X = A->A;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    h->A = X;
    size_t ts = type_size(X.type);
    h->A.p = (int32_t *)dalloc((size_t)(X.nrows + 1) * 4, s);
    h->A.j = (int32_t *)dalloc((size_t)(X.nnz ? X.nnz : 1) * 4, s);
    h->A.x = X.x ? dalloc(X.iso ? ts : (size_t)(X.nnz ? X.nnz : 1) * ts, s) : nullptr;
    if (!h->A.p || !h->A.j || (X.x && !h->A.x)) { dev_free(h->A, s); delete h; return OUT_OF_MEMORY; }
    cudaMemcpyAsync(h->A.p, X.p, (size_t)(X.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(h->A.j, X.j, (size_t)X.nnz * 4, cudaMemcpyDeviceToDevice, s);
    if (X.x) cudaMemcpyAsync(h->A.x, X.x, X.iso ? ts : (size_t)X.nnz * ts, cudaMemcpyDeviceToDevice, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { dev_free(h->A, s); delete h; return cuda_to_info(e); }
    *D = h;
    return SUCCESS;
}

int grb_b200_daccum_mask(grb_b200_dmatrix C, grb_b200_dmatrix T, grb_b200_dmatrix M,
                         bool mask_comp, bool mask_struct, bool replace,
                         int accum_opcode)
{
    if (!C || !T) return NULL_POINTER;
    StreamGuard g;
    C->sum_ok = false;
    int info = accum_mask(C->A, T->A, M ? &M->A : nullptr, mask_comp, mask_struct,
                          replace, accum_opcode, g.s);
    cudaError_t e = cudaStreamSynchronize(g.s);
    return info != SUCCESS ? info : cuda_to_info(e);
}

int grb_b200_dtranspose(grb_b200_dmatrix *B, grb_b200_dmatrix A)
{
    if (!B || !A) return NULL_POINTER;
    StreamGuard g;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    int info = transpose(h->A, A->A, g.s);
    if (info != SUCCESS) { delete h; return info; }
    *B = h;
    return SUCCESS;
}

int grb_b200_dmxv(grb_b200_dmatrix *w, grb_b200_dmatrix mask, bool mask_comp,
                  bool mask_struct, grb_b200_dmatrix A, grb_b200_dmatrix u,
                  const grb_b200_semiring *sr)
{
    if (!w || !A || !u || !sr) return NULL_POINTER;
    StreamGuard g;
    grb_b200_dmatrix h = new grb_b200_dmatrix_s();
    SemiringCode sc{sr->add_opcode, sr->mult_opcode, sr->type};
    int info = mxv(h->A, mask ? &mask->A : nullptr, mask_comp, mask_struct, A->A,
                   u->A, sc, g.s);
    if (info != SUCCESS) { delete h; return info; }
    *w = h;
    return SUCCESS;
}

int grb_b200_dwait(grb_b200_dmatrix D)
{
    if (!D) return NULL_POINTER;
    StreamGuard g;
    int info = dev_prune_zombies(D->A, g.s);
    cudaError_t e = cudaStreamSynchronize(g.s);
    return info != SUCCESS ? info : cuda_to_info(e);
}

}  // extern "C"
