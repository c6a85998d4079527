// grb_reduce.cu: reduce a matrix to a scalar with a built-in monoid, skipping
// zombies; the B200 replacement of GB_reduce_to_scalar
// (Source/reduce/GB_reduce_to_scalar.c:41) and of the draft GPU reduce
// (CUDA/template/GB_jit_kernel_cuda_reduce.cu:44).  Two passes: per-block
// partials (grid = a multiple of the SM count), then one block folds them.
// An empty matrix (or one with only zombies) reduces to the identity.

#include "grb_runtime.h"

namespace grb {

template <int ADD, typename Z>
__device__ __forceinline__ Z mono_id() { return Monoid<ADD, Z>::identity(); }

template <int ADD, typename Z>
__device__ __forceinline__ void warp_fold(Z &v, bool &has)
{
    for (int o = 16; o > 0; o >>= 1) {
        Z ov = shfl_down<Z>(v, o);
        bool oh = shfl_down<bool>(has, o);
        if (oh) { v = has ? Monoid<ADD, Z>::add(v, ov) : ov; has = true; }
    }
}

template <int ADD, typename Z>
__global__ void k_reduce_partial(const int32_t *__restrict__ Aj,
                                 const Z *__restrict__ Ax, bool iso,
                                 int64_t nnz, Z *__restrict__ part_v,
                                 int *__restrict__ part_h)
{
    __shared__ Z sv[32];
    __shared__ bool sh[32];
    Z v = Z();
    bool has = false;
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < nnz; t += stride) {
        if (Aj[t] < 0) continue;                      // zombie
        Z a = Ax[iso ? 0 : t];
        v = has ? Monoid<ADD, Z>::add(v, a) : a;
        has = true;
    }
    warp_fold<ADD, Z>(v, has);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sv[w] = v; sh[w] = has; }
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        v = lane < nw ? sv[lane] : Z();
        has = lane < nw ? sh[lane] : false;
        warp_fold<ADD, Z>(v, has);
        if (lane == 0) { part_v[blockIdx.x] = v; part_h[blockIdx.x] = has; }
    }
}

template <int ADD, typename Z>
__global__ void k_reduce_final(const Z *__restrict__ part_v,
                               const int *__restrict__ part_h, int n,
                               Z *__restrict__ out)
{
    Z v = Z();
    bool has = false;
    // one warp folds the partials in block order
    for (int b = threadIdx.x; b < n; b += 32) {
        if (part_h[b]) { v = has ? Monoid<ADD, Z>::add(v, part_v[b]) : part_v[b]; has = true; }
    }
    warp_fold<ADD, Z>(v, has);
    if (threadIdx.x == 0) *out = has ? v : mono_id<ADD, Z>();
}

template <int ADD, typename Z>
static int reduce_t(void *out, const DevCSR &A, cudaStream_t s)
{
    int blocks = runtime().num_sms * 4;
    Z *pv = (Z *)dalloc(sizeof(Z) * (blocks + 1), s);
    int *ph = (int *)dalloc(sizeof(int) * blocks, s);
    if (!pv || !ph) { dfree(pv, s); dfree(ph, s); return OUT_OF_MEMORY; }
    if (A.nnz > 0 && A.x) {
        k_reduce_partial<ADD, Z><<<blocks, 256, 0, s>>>(A.j, (const Z *)A.x, A.iso,
                                                        A.nnz, pv, ph);
        k_reduce_final<ADD, Z><<<1, 32, 0, s>>>(pv, ph, blocks, pv + blocks);
    } else {
        cudaMemsetAsync(ph, 0, sizeof(int) * blocks, s);
        k_reduce_final<ADD, Z><<<1, 32, 0, s>>>(pv, ph, blocks, pv + blocks);
    }
    cudaError_t e = readback(out, pv + blocks, sizeof(Z), s);
    dfree(pv, s); dfree(ph, s);
    return cuda_to_info(e);
}

int reduce_scalar(void *out, const DevCSR &A, int monoid, cudaStream_t s)
{
    int t = A.type;
#define R_CASE(ADD, TC, CT) if (monoid == ADD && t == TC) return reduce_t<ADD, CT>(out, A, s);
#define R_TYPES(ADD) R_CASE(ADD, T_INT64, int64_t) R_CASE(ADD, T_INT32, int32_t) \
    R_CASE(ADD, T_FP64, double) R_CASE(ADD, T_FP32, float)
    R_TYPES(OP_PLUS)
    R_TYPES(OP_MIN)
    R_TYPES(OP_MAX)
    R_TYPES(OP_TIMES)
    R_TYPES(OP_ANY)
    R_CASE(OP_LOR, T_BOOL, bool)
    R_CASE(OP_LAND, T_BOOL, bool)
    R_CASE(OP_ANY, T_BOOL, bool)
#undef R_TYPES
#undef R_CASE
    return NO_VALUE;
}

}  // namespace grb
