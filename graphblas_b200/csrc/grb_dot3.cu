// grb_dot3.cu: masked dot-product SpGEMM, C<M> = A*B' (C(i,j) = A(i,:).B(j,:)
// for every (i,j) in the pattern of M), the B200 replacement of the
// reference's GB_AxB_dot3 (Source/mxm/GB_AxB_dot3.c:37) and of its draft GPU
// kernels (CUDA/template/GB_cuda_jit_AxB_dot3_phase{1,2,3_vsvs,3_mp}.cuh).
//
// Design (one launch, no host round trip):
//   * A warp owns one mask row i at a time, taken from a global work counter
//     (rows are uneven: R-MAT degrees span 1..65k).  A(i,:) is staged once in
//     the warp's shared-memory slice and reused by every entry of M(i,:).
//   * Each lane takes one entry (i,j) of the row and trims both lists to their
//     overlap [max(first), min(last)] with binary searches (the reference's
//     dot3 trims when one list is much longer, GB_AxB_dot_cij.c:538-617).
//     Empty overlaps become zombies at once; short overlaps are merged by the
//     lane itself (the reference's VSVS bucket, phase3_vsvs.cuh:133).
//   * Long overlaps are queued and taken by the whole warp, one at a time:
//     lanes walk 32 consecutive elements of one list (coalesced) and locate
//     each in the other list by binary search, advancing the search window
//     chunk by chunk (a merge-path partition of the two lists).  The list that
//     is scanned is the shorter one in cost: B when it is at most 8x longer
//     than A (A is in shared memory), otherwise A, searched in global B.
//   * Matches come out of __ballot_sync in ascending k, so order-dependent
//     monoids (floating PLUS/TIMES, ANY) fold them in exactly the reference's
//     sequential order, first match assigned and later ones added
//     (GB_AxB_dot_cij.c:516-652); order-free monoids keep per-lane partials
//     and finish with a warp reduction.
//   * ANY is terminal: the first match ends the dot product.
//   * Empty results are zombies, Cj[p] = flip(j) (GB_zombie.h:37), counted in
//     C.nzombies; C keeps M's row pointers, as the reference's dot3 does
//     (GB_AxB_dot3.c:172-197).

#include <cstdio>
#include <cstring>
#include "grb_runtime.h"
#include "grb_semirings.h"

namespace grb {

static constexpr int D3_WARPS = 8;        // warps per block
static constexpr int D3_CAP = 1024;       // A(i,:) entries staged per warp
static constexpr int D3_SMALL = 48;       // per-lane merge threshold (nA+nB)

__device__ __forceinline__ bool mask_value_true(const void *Mx, int mtype,
                                                int64_t p)
{
    switch (mtype) {
        case T_BOOL: return ((const uint8_t *)Mx)[p] != 0;
        case T_INT32: case T_UINT32: return ((const uint32_t *)Mx)[p] != 0;
        case T_FP32: return ((const float *)Mx)[p] != 0.0f;
        case T_FP64: return ((const double *)Mx)[p] != 0.0;
        default: return ((const uint64_t *)Mx)[p] != 0;
    }
}

// partial result of a dot product: value plus "exists" flag
template <typename Z> struct Part { Z v; bool has; };

template <class SR>
__device__ __forceinline__ Part<typename SR::z_t>
combine(Part<typename SR::z_t> a, Part<typename SR::z_t> b)
{
    if (!a.has) return b;
    if (!b.has) return a;
    return {SR::M::add(a.v, b.v), true};
}

template <class SR, int WARPS, int CAP>
__global__ void __launch_bounds__(WARPS * 32)
k_dot3(const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
       const void *__restrict__ Mx, int mtype, bool mask_struct,
       const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
       const void *__restrict__ Ax, bool a_iso,
       const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
       const void *__restrict__ Bx, bool b_iso,
       int32_t *__restrict__ Cj, typename SR::z_t *__restrict__ Cx,
       int64_t nrows, int *__restrict__ row_counter,
       unsigned long long *__restrict__ nzombies)
{
    using Z = typename SR::z_t;
    __shared__ int32_t sA_all[WARPS][CAP];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    int32_t *sA = sA_all[warp];
    unsigned long long zcount = 0;

    while (true) {
        int r = 0;
        if (lane == 0) r = atomicAdd(row_counter, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= nrows) break;
        const int64_t i = r;
        const int32_t mp0 = Mp[i], mp1 = Mp[i + 1];
        if (mp0 == mp1) continue;
        const int32_t pa0 = Ap[i];
        const int32_t na = Ap[i + 1] - pa0;
        const int32_t *a_idx;
        if (na <= CAP) {
            for (int32_t t = lane; t < na; t += 32) sA[t] = Aj[pa0 + t];
            __syncwarp();
            a_idx = sA;
        } else {
            a_idx = Aj + pa0;
        }

        for (int32_t cb = mp0; cb < mp1; cb += 32) {
            const int32_t pm = cb + lane;
            const bool valid = pm < mp1;
            int32_t j = 0, ia0 = 0, ia1 = 0, ib0 = 0, ib1 = 0;
            bool coop = false, exists = false;
            Z cij = Z();
            if (valid) {
                j = Mj[pm];
                bool mval = mask_struct || Mx == nullptr || mask_value_true(Mx, mtype, pm);
                if (mval && na > 0) {
                    const int32_t pb0 = Bp[j], pb1 = Bp[j + 1];
                    if (pb1 > pb0) {
                        const int32_t blo = Bj[pb0], bhi = Bj[pb1 - 1];
                        ia0 = lower_bound(a_idx, 0, na, blo);
                        ia1 = upper_bound(a_idx, ia0, na, bhi);
                        if (ia1 > ia0) {
                            const int32_t alo = a_idx[ia0], ahi = a_idx[ia1 - 1];
                            ib0 = lower_bound(Bj, pb0, pb1, alo);
                            ib1 = upper_bound(Bj, ib0, pb1, ahi);
                            if (ib1 > ib0) {
                                if ((ia1 - ia0) + (ib1 - ib0) <= D3_SMALL) {
                                    // per-lane two-pointer merge
                                    int32_t a = ia0, b = ib0;
                                    while (a < ia1 && b < ib1) {
                                        const int32_t ka = a_idx[a], kb = Bj[b];
                                        if (ka < kb) a++;
                                        else if (kb < ka) b++;
                                        else {
                                            Z av = Z(), bv = Z();
                                            if (SR::needs_a) av = ld_val<Z>(Ax, pa0 + a, a_iso);
                                            if (SR::needs_b) bv = ld_val<Z>(Bx, b, b_iso);
                                            Z t = SR::F::f(av, bv, i, ka, j);
                                            if (!exists) { cij = t; exists = true; }
                                            else cij = SR::M::add(cij, t);
                                            if (SR::M::any) break;
                                            a++; b++;
                                        }
                                    }
                                } else {
                                    coop = true;
                                }
                            }
                        }
                    }
                }
            }
            if (valid && !coop) {
                if (exists) { Cj[pm] = j; Cx[pm] = cij; }
                else { Cj[pm] = flip(j); zcount++; }
            }

            // warp-cooperative intersections, one queued entry at a time
            unsigned q = __ballot_sync(0xffffffffu, coop);
            while (q) {
                const int src = __ffs(q) - 1;
                q &= q - 1;
                const int32_t qpm = __shfl_sync(0xffffffffu, pm, src);
                const int32_t qj = __shfl_sync(0xffffffffu, j, src);
                const int32_t qa0 = __shfl_sync(0xffffffffu, ia0, src);
                const int32_t qa1 = __shfl_sync(0xffffffffu, ia1, src);
                const int32_t qb0 = __shfl_sync(0xffffffffu, ib0, src);
                const int32_t qb1 = __shfl_sync(0xffffffffu, ib1, src);
                const int32_t nA = qa1 - qa0, nB = qb1 - qb0;
                Part<Z> part{Z(), false};      // order-free partial (per lane)
                Z acc = Z();                   // in-order fold (uniform)
                bool acc_has = false;
                const bool scanB = (nB <= 8 * nA);
                const int32_t s0 = scanB ? qb0 : qa0;     // scanned list range
                const int32_t s1 = scanB ? qb1 : qa1;
                int32_t lo = scanB ? qa0 : qb0;           // searched list window
                const int32_t hi = scanB ? qa1 : qb1;
                for (int32_t c0 = s0; c0 < s1; c0 += 32) {
                    const int32_t sp = c0 + lane;
                    const bool has = sp < s1;
                    int32_t key = INT32_MAX, pos;
                    if (scanB) {
                        if (has) key = Bj[sp];
                        pos = lower_bound(a_idx, lo, hi, key);
                    } else {
                        if (has) key = a_idx[sp];
                        pos = lower_bound(Bj, lo, hi, key);
                    }
                    bool match = false;
                    if (has && pos < hi)
                        match = scanB ? (a_idx[pos] == key) : (Bj[pos] == key);
                    Z t = Z();
                    if (match) {
                        const int32_t apos = scanB ? pos : sp;
                        const int32_t bpos = scanB ? sp : pos;
                        Z av = Z(), bv = Z();
                        if (SR::needs_a) av = ld_val<Z>(Ax, pa0 + apos, a_iso);
                        if (SR::needs_b) bv = ld_val<Z>(Bx, bpos, b_iso);
                        t = SR::F::f(av, bv, i, key, qj);
                    }
                    const unsigned mm = __ballot_sync(0xffffffffu, match);
                    if (SR::order_free && !SR::M::any) {
                        if (match) part = combine<SR>(part, Part<Z>{t, true});
                    } else {
                        // fold in ascending k, exactly as the sequential merge
                        unsigned m2 = mm;
                        while (m2) {
                            const int b = __ffs(m2) - 1;
                            m2 &= m2 - 1;
                            const Z tv = shfl<Z>(t, b);
                            if (!acc_has) { acc = tv; acc_has = true; }
                            else acc = SR::M::add(acc, tv);
                            if (SR::M::any) break;
                        }
                        if (SR::M::any && acc_has) break;
                    }
                    lo = __shfl_sync(0xffffffffu, pos, 31);
                    if (lo >= hi) break;
                }
                if (SR::order_free && !SR::M::any) {
                    // warp reduction of the per-lane partials
                    for (int o = 16; o > 0; o >>= 1) {
                        Part<Z> other;
                        other.v = shfl_down<Z>(part.v, o);
                        other.has = shfl_down<bool>(part.has, o);
                        part = combine<SR>(part, other);
                    }
                    acc = part.v; acc_has = part.has;
                }
                if (lane == 0) {
                    if (acc_has) { Cj[qpm] = qj; Cx[qpm] = acc; }
                    else { Cj[qpm] = flip(qj); zcount++; }
                }
            }
        }
        __syncwarp();
    }
    if (zcount) atomicAdd(nzombies, zcount);
}

template <class SR>
static int dot3_launch(DevCSR &C, const DevCSR &M, bool mask_struct,
                       const DevCSR &A, const DevCSR &B, cudaStream_t s)
{
    using Z = typename SR::z_t;
    int64_t mnz = M.nnz;
    C.nrows = M.nrows; C.ncols = M.ncols; C.nnz = mnz; C.type = 0; C.iso = false;
    C.p = (int32_t *)dalloc((size_t)(M.nrows + 1) * 4, s);
    C.j = (int32_t *)dalloc((size_t)(mnz ? mnz : 1) * 4, s);
    C.x = dalloc((size_t)(mnz ? mnz : 1) * sizeof(Z), s);
    int *counter = (int *)dalloc(64, s);
    if (!C.p || !C.j || !C.x || !counter) {
        dev_free(C, s); dfree(counter, s); return OUT_OF_MEMORY;
    }
    cudaMemcpyAsync(C.p, M.p, (size_t)(M.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(counter, 0, 64, s);
    unsigned long long *zc = (unsigned long long *)((char *)counter + 32);
    if (mnz > 0 && M.nrows > 0) {
        int blocks = runtime().num_sms * 6;
        int ps = prof_begin("dot3", s);
        k_dot3<SR, D3_WARPS, D3_CAP><<<blocks, D3_WARPS * 32, 0, s>>>(
            M.p, M.j, mask_struct ? nullptr : M.x, M.type, mask_struct,
            A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso,
            C.j, (Z *)C.x, M.nrows, counter, zc);
        prof_end(ps, s);
    }
    unsigned long long hz = 0;
    cudaMemcpyAsync(&hz, zc, 8, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    dfree(counter, s);
    if (e != cudaSuccess) { dev_free(C, s); return cuda_to_info(e); }
    C.nzombies = (int64_t)hz;
    return SUCCESS;
}

__global__ void k_flip_all(const int32_t *__restrict__ Mj, int32_t *__restrict__ Cj,
                           int64_t n)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < n; t += stride) Cj[t] = flip(Mj[t]);
}

static int dot3_all_zombies(DevCSR &C, const DevCSR &M, SemiringCode sr,
                            cudaStream_t s)
{
    if (!semiring_supported(sr)) return NO_VALUE;
    int64_t mnz = M.nnz;
    C.nrows = M.nrows; C.ncols = M.ncols; C.nnz = mnz; C.type = sr.type;
    C.iso = false;
    C.p = (int32_t *)dalloc((size_t)(M.nrows + 1) * 4, s);
    C.j = (int32_t *)dalloc((size_t)(mnz ? mnz : 1) * 4, s);
    C.x = dalloc((size_t)(mnz ? mnz : 1) * type_size(sr.type), s);
    if (!C.p || !C.j || !C.x) { dev_free(C, s); return OUT_OF_MEMORY; }
    cudaMemcpyAsync(C.p, M.p, (size_t)(M.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
    if (mnz > 0) k_flip_all<<<runtime().num_sms * 4, 256, 0, s>>>(M.j, C.j, mnz);
    C.nzombies = mnz;
    return cuda_to_info(cudaStreamSynchronize(s));
}

int dot3(DevCSR &C, const DevCSR &M, bool mask_struct, const DevCSR &A,
         const DevCSR &B, SemiringCode sr, cudaStream_t s)
{
    if (A.ncols != B.ncols || M.nrows != A.nrows || M.ncols != B.nrows)
        return DIMENSION_MISMATCH;
    // an iso valued mask is all-true (structural) or all-false (every entry
    // of C is a zombie)
    bool all_false = false;
    if (!mask_struct && M.iso && M.x) {
        uint64_t v = 0;
        size_t ts = type_size(M.type);
        cudaMemcpyAsync(&v, M.x, ts, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        if (M.type == T_FP32) { float f; memcpy(&f, &v, 4); all_false = (f == 0.0f); }
        else if (M.type == T_FP64) { double d; memcpy(&d, &v, 8); all_false = (d == 0.0); }
        else all_false = (v == 0);
        mask_struct = true;
    }
    if (!M.x) mask_struct = true;
    if (all_false) return dot3_all_zombies(C, M, sr, s);
#define GRB_DOT3_CASE(ADD, MULT, TC, CT)                                       \
    if (sr.add == ADD && sr.mult == MULT && sr.type == TC) {                   \
        int info = dot3_launch<Semiring<ADD, MULT, CT>>(C, M, mask_struct, A, B, s); \
        if (info == SUCCESS) C.type = TC;                                      \
        return info;                                                           \
    }
    GRB_FOR_EACH_SEMIRING(GRB_DOT3_CASE)
#undef GRB_DOT3_CASE
    return NO_VALUE;
}

bool semiring_supported(SemiringCode sr)
{
#define GRB_SUP_CASE(ADD, MULT, TC, CT) \
    if (sr.add == ADD && sr.mult == MULT && sr.type == TC) return true;
    GRB_FOR_EACH_SEMIRING(GRB_SUP_CASE)
#undef GRB_SUP_CASE
    return false;
}

}  // namespace grb
