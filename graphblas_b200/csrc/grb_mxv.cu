// grb_mxv.cu: w<m> = A*u for a sparse vector u (GrB_mxv, Source/mxm/
// GrB_mxv.c:18), w(i) = sum over k of A(i,k) (x) u(k).  u is scattered into
// a dense value array plus a presence bitmap over its length; one warp per
// row of A then walks A(i,:) (coalesced) and folds the products of the
// present k in ascending k (ballot order), so floating PLUS is bit-exact with
// the reference's sequential dot products (GB_AxB_dot_cij.c:516-652).  The
// mask m on w is scattered the same way; rows the mask rejects are skipped.
// Results are compacted into a sorted sparse vector (a 1-by-nrows CSR row).
//
// MAX with a multiplier whose value is k (SECONDI, FIRSTJ: the parent in a
// pull BFS step) is the largest k that matches, so such a row is walked from
// its end and stops at its first match: an unvisited vertex usually finds a
// frontier neighbour within its last few entries.

#include "grb_runtime.h"
#include "grb_semirings.h"

namespace grb {

template <typename Z>
__global__ void k_scatter_vec(const int32_t *__restrict__ uj, const Z *__restrict__ ux,
                              bool iso, int64_t nu, Z *__restrict__ dense,
                              uint32_t *__restrict__ bits)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nu;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = uj[e];
        if (k < 0) continue;
        dense[k] = ux[iso ? 0 : e];
        atomicOr(&bits[k >> 5], 1u << (k & 31));
    }
}

__global__ void k_scatter_bits(const int32_t *__restrict__ mj, int64_t nm,
                               uint32_t *__restrict__ bits)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nm;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = mj[e];
        if (k >= 0) atomicOr(&bits[k >> 5], 1u << (k & 31));
    }
}

template <class SR>
__global__ void __launch_bounds__(256)
k_mxv_rows(int64_t m, const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
           const void *__restrict__ Ax, bool a_iso,
           const typename SR::z_t *__restrict__ ud, const uint32_t *__restrict__ ubits,
           const uint32_t *__restrict__ mbits, bool has_mask, bool comp,
           typename SR::z_t *__restrict__ wd, int32_t *__restrict__ wflag)
{
    using Z = typename SR::z_t;
    const int lane = threadIdx.x & 31;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        bool ok = true;
        if (has_mask) {
            const bool present = (mbits[i >> 5] >> (i & 31)) & 1u;
            ok = comp ? !present : present;
        } else if (comp) {
            ok = false;
        }
        if (!ok) { if (lane == 0) wflag[i] = 0; continue; }
        Z acc = Z();
        bool has = false;
        const int32_t lo = Ap[i], hi = Ap[i + 1];
        if constexpr (SR::add_op == OP_MAX && (SR::mult_op == OP_SECONDI ||
                                                SR::mult_op == OP_FIRSTJ)) {
            // the largest matching k: 32 entries at a time from the end
            for (int32_t c1 = hi; c1 > lo; c1 -= 32) {
                const int32_t p = c1 - 32 + lane;
                bool match = false;
                int32_t k = 0;
                if (p >= lo) {
                    k = Aj[p];
                    match = (ubits[k >> 5] >> (k & 31)) & 1u;
                }
                const unsigned mm = __ballot_sync(0xffffffffu, match);
                if (mm) {
                    const int b = 31 - __clz(mm);
                    const int32_t kb = __shfl_sync(0xffffffffu, k, b);
                    acc = (Z)kb;
                    has = true;
                    break;
                }
            }
            if (lane == 0) { wflag[i] = has ? 1 : 0; if (has) wd[i] = acc; }
            continue;
        }
        for (int32_t c0 = lo; c0 < hi; c0 += 32) {
            const int32_t p = c0 + lane;
            bool match = false;
            Z t = Z();
            int32_t k = 0;
            if (p < hi) {
                k = Aj[p];
                match = (ubits[k >> 5] >> (k & 31)) & 1u;
                if (match) {
                    Z av = Z();
                    if (SR::needs_a) av = ld_val<Z>(Ax, p, a_iso);
                    t = SR::F::f(av, ud[k], i, k, 0);
                }
            }
            unsigned mm = __ballot_sync(0xffffffffu, match);
            while (mm) {
                const int b = __ffs(mm) - 1;
                mm &= mm - 1;
                const Z tv = shfl<Z>(t, b);
                if (!has) { acc = tv; has = true; }
                else acc = SR::M::add(acc, tv);
                if (SR::M::any) break;
            }
            if (SR::M::any && has) break;
        }
        if (lane == 0) { wflag[i] = has ? 1 : 0; if (has) wd[i] = acc; }
    }
}

template <typename Z>
__global__ void k_compact_dense(int64_t m, const int32_t *__restrict__ flag,
                                const int64_t *__restrict__ pos, const Z *__restrict__ wd,
                                int32_t *__restrict__ wj, Z *__restrict__ wx)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (flag[i]) { wj[pos[i]] = (int32_t)i; wx[pos[i]] = wd[i]; }
    }
}

static inline int grid_v(int64_t n, int threads = 256)
{
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)runtime().num_sms * 16;
    if (b > cap) b = cap;
    return b < 1 ? 1 : (int)b;
}

template <class SR>
static int mxv_t(DevCSR &w, const DevCSR *mask, bool comp, const DevCSR &A,
                 const DevCSR &u, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t m = A.nrows, n = A.ncols;
    Scratch ws(s);
    Z *ud = ws.get<Z>(n + 1);
    uint32_t *ubits = ws.get<uint32_t>(n / 32 + 2);
    uint32_t *mbits = ws.get<uint32_t>(m / 32 + 2);
    Z *wd = ws.get<Z>(m + 1);
    int32_t *wflag = ws.get<int32_t>(m + 1);
    int64_t *pos = ws.get<int64_t>(m + 1);
    if (ws.failed) return OUT_OF_MEMORY;
    cudaMemsetAsync(ubits, 0, (size_t)(n / 32 + 2) * 4, s);
    cudaMemsetAsync(mbits, 0, (size_t)(m / 32 + 2) * 4, s);
    if (u.nnz > 0)
        k_scatter_vec<Z><<<grid_v(u.nnz), 256, 0, s>>>(u.j, (const Z *)u.x, u.iso, u.nnz,
                                                       ud, ubits);
    if (mask && mask->nnz > 0)
        k_scatter_bits<<<grid_v(mask->nnz), 256, 0, s>>>(mask->j, mask->nnz, mbits);
    const int ps = prof_begin("mxv", s);
    if (m > 0)
        k_mxv_rows<SR><<<grid_v(m * 32), 256, 0, s>>>(m, A.p, A.j, A.x, A.iso, ud, ubits,
            mbits, mask != nullptr, comp, wd, wflag);
    prof_end(ps, s);
    cudaMemsetAsync(wflag + m, 0, 4, s);
    int info = scan_exclusive_i32_to_i64(wflag, pos, m + 1, s);
    if (info != SUCCESS) return info;
    int64_t nw = 0;
    cudaError_t e = readback(&nw, pos + m, 8, s);
    if (e != cudaSuccess) return cuda_to_info(e);
    w = DevCSR();
    w.nrows = 1; w.ncols = m; w.nnz = nw; w.iso = false;
    w.p = (int32_t *)dalloc(8, s);
    w.j = (int32_t *)dalloc((size_t)(nw ? nw : 1) * 4, s);
    w.x = dalloc((size_t)(nw ? nw : 1) * sizeof(Z), s);
    if (!w.p || !w.j || !w.x) { dev_free(w, s); return OUT_OF_MEMORY; }
    int32_t hp[2] = {0, (int32_t)nw};
    cudaMemcpyAsync(w.p, hp, 8, cudaMemcpyHostToDevice, s);
    if (m > 0) k_compact_dense<Z><<<grid_v(m), 256, 0, s>>>(m, wflag, pos, wd, w.j, (Z *)w.x);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { dev_free(w, s); return cuda_to_info(e); }
    return SUCCESS;
}

int mxv(DevCSR &w, const DevCSR *mask, bool mask_comp, bool mask_struct,
        const DevCSR &A, const DevCSR &u, SemiringCode sr, cudaStream_t s)
{
    if (u.ncols != A.ncols || u.nrows != 1) return DIMENSION_MISMATCH;
    if (mask && (mask->ncols != A.nrows || mask->nrows != 1)) return DIMENSION_MISMATCH;
    DevCSR Ms;
    bool own = false;
    if (mask && !mask_struct && mask->x) {
        int info = dev_mask_to_struct(Ms, *mask, s);
        if (info != SUCCESS) return info;
        mask = &Ms;
        own = true;
    }
    int info = NO_VALUE;
#define GRB_MXV_CASE(ADD, MULT, TC, CT)                                        \
    if (sr.add == ADD && sr.mult == MULT && sr.type == TC) {                   \
        info = mxv_t<Semiring<ADD, MULT, CT>>(w, mask, mask_comp, A, u, s);    \
        if (info == SUCCESS) w.type = TC;                                      \
    } else
    GRB_FOR_EACH_SEMIRING(GRB_MXV_CASE) { info = NO_VALUE; }
#undef GRB_MXV_CASE
    if (own) dev_free(Ms, s);
    return info;
}

}  // namespace grb
