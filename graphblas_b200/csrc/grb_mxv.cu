// grb_mxv.cu: w<m> = A*u for a sparse vector u (GrB_mxv, Source/mxm/
// GrB_mxv.c:18), w(i) = sum over k of A(i,k) (x) u(k).  u is scattered into
// a dense value array plus a presence bitmap over its length; one warp per
// row of A then walks A(i,:) (coalesced) and folds the products of the
// present k in ascending k (ballot order), so floating PLUS is bit-exact with
// the reference's sequential dot products (GB_AxB_dot_cij.c:516-652).  The
// mask m on w is scattered the same way; rows the mask rejects are skipped.
// Results are compacted into a sorted sparse vector (a 1-by-nrows CSR row)
// with one host read per call.
//
// MAX with a multiplier whose value is k (SECONDI, FIRSTJ: the parent in a
// pull BFS step) is the largest k that matches, so such a row is walked from
// its end and stops at its first match: an unvisited vertex usually finds a
// frontier neighbour within its last few entries.  Those rows are taken one
// per lane (most rows of a graph are short), and a row longer than
// MAXK_SHORT by the whole warp, 32 entries a step.

#include "grb_runtime.h"
#include "grb_semirings.h"
#include "grb_lookback.cuh"

namespace grb {

// set bit k of `bits` for the indices of a sorted list (zombies, k < 0,
// skipped): the lanes of a warp that fall in the same 32-bit word combine
// their bits first, so a word takes one atomic per warp
__device__ __forceinline__ void warp_set_bit(uint32_t *__restrict__ bits, int32_t k, bool on)
{
    const unsigned act = __ballot_sync(0xffffffffu, on);
    if (!on) return;
    const int32_t word = k >> 5;
    const unsigned same = __match_any_sync(act, word);
    const unsigned v = __reduce_or_sync(same, 1u << (k & 31));
    if ((int)(__ffs(same) - 1) == (int)(threadIdx.x & 31)) atomicOr(&bits[word], v);
}

template <typename Z>
__global__ void k_scatter_vec(const int32_t *__restrict__ uj, const Z *__restrict__ ux,
                              bool iso, int64_t nu, Z *__restrict__ dense,
                              uint32_t *__restrict__ bits)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); e0 < nu;
         e0 += stride) {
        const int64_t e = e0 + (threadIdx.x & 31);
        const int32_t k = e < nu ? uj[e] : -1;
        if (k >= 0) dense[k] = ux[iso ? 0 : e];
        warp_set_bit(bits, k, k >= 0);
    }
}

__global__ void k_scatter_bits(const int32_t *__restrict__ mj, int64_t nm,
                               uint32_t *__restrict__ bits)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); e0 < nm;
         e0 += stride) {
        const int64_t e = e0 + (threadIdx.x & 31);
        const int32_t k = e < nm ? mj[e] : -1;
        warp_set_bit(bits, k, k >= 0);
    }
}

template <class SR>
__global__ void __launch_bounds__(256)
k_mxv_rows(int64_t m, const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
           const void *__restrict__ Ax, bool a_iso,
           const typename SR::z_t *__restrict__ ud, const uint32_t *__restrict__ ubits,
           const uint32_t *__restrict__ mbits, bool has_mask, bool comp,
           typename SR::z_t *__restrict__ wd, uint32_t *__restrict__ gbits)
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
        if (!ok) continue;
        Z acc = Z();
        bool has = false;
        const int32_t lo = Ap[i], hi = Ap[i + 1];
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
        if (lane == 0 && has) {
            wd[i] = acc;
            atomicOr(&gbits[i >> 5], 1u << (i & 31));
        }
    }
}

static constexpr int MAXK_SHORT = 64;

template <class SR>
__global__ void __launch_bounds__(256)
k_mxv_rows_maxk(int64_t m, const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
                const uint32_t *__restrict__ ubits, const uint32_t *__restrict__ mbits,
                bool has_mask, bool comp, typename SR::z_t *__restrict__ wd,
                uint32_t *__restrict__ gbits)
{
    using Z = typename SR::z_t;
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < m;
         base += nw * 32) {
        const int64_t i = base + lane;
        bool ok = i < m;
        if (ok) {
            if (has_mask) {
                const bool present = (mbits[i >> 5] >> (i & 31)) & 1u;
                ok = comp ? !present : present;
            } else if (comp) {
                ok = false;
            }
        }
        int32_t lo = 0, hi = 0;
        if (ok) { lo = Ap[i]; hi = Ap[i + 1]; }
        const bool lng = ok && hi - lo > MAXK_SHORT;
        bool found = false;
        int32_t kf = 0;
        if (ok && !lng) {
            // four entries a step, from the end
            for (int32_t p = hi; p > lo && !found; p -= 4) {
                int32_t k[4];
                bool hit[4];
                #pragma unroll
                for (int t = 0; t < 4; t++) {
                    const int32_t q = p - 1 - t;
                    k[t] = q >= lo ? Aj[q] : 0;
                    hit[t] = q >= lo && ((ubits[k[t] >> 5] >> (k[t] & 31)) & 1u);
                }
                // the largest match is the one nearest the end (smallest t)
                #pragma unroll
                for (int t = 3; t >= 0; t--)
                    if (hit[t]) { found = true; kf = k[t]; }
            }
        }
        // long rows: the whole warp, one row at a time
        unsigned lm = __ballot_sync(0xffffffffu, lng);
        while (lm) {
            const int b = __ffs(lm) - 1;
            lm &= lm - 1;
            const int32_t blo = __shfl_sync(0xffffffffu, lo, b);
            const int32_t bhi = __shfl_sync(0xffffffffu, hi, b);
            bool bf = false;
            int32_t bk = 0;
            for (int32_t c1 = bhi; c1 > blo; c1 -= 32) {
                const int32_t q = c1 - 32 + lane;
                int32_t k = 0;
                bool match = false;
                if (q >= blo) {
                    k = Aj[q];
                    match = (ubits[k >> 5] >> (k & 31)) & 1u;
                }
                const unsigned mm = __ballot_sync(0xffffffffu, match);
                if (mm) {
                    bk = __shfl_sync(0xffffffffu, k, 31 - __clz(mm));
                    bf = true;
                    break;
                }
            }
            if (lane == b) { found = bf; kf = bk; }
        }
        if (found) wd[i] = (Z)kf;
        // the warp owns the 32 rows of its group: their bits in one word
        const unsigned fb = __ballot_sync(0xffffffffu, found);
        if (lane == 0) gbits[base >> 5] = fb;
    }
}

// rows with a result are marked in gbits (bit i & 31 of word i >> 5); gpos[g]
// is the number of marked rows before group g
template <typename Z>
__global__ void k_compact_dense(int64_t m, const uint32_t *__restrict__ gbits,
                                const int64_t *__restrict__ gpos, const Z *__restrict__ wd,
                                int32_t *__restrict__ wp, int32_t *__restrict__ wj,
                                Z *__restrict__ wx)
{
    const int64_t ng = (m + 31) / 32;
    if (blockIdx.x == 0 && threadIdx.x == 0) { wp[0] = 0; wp[1] = (int32_t)gpos[ng]; }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t b = gbits[i >> 5];
        const int r = (int)(i & 31);
        if ((b >> r) & 1u) {
            const int64_t q = gpos[i >> 5] + __popc(b & ((1u << r) - 1u));
            wj[q] = (int32_t)i;
            wx[q] = wd[i];
        }
    }
}

// value g of the output-position scan: the marked rows of group g
struct MxvLoadGroup {
    const uint32_t *gbits;
    int64_t ng;
    __device__ int64_t operator()(int64_t g) const { return g < ng ? __popc(gbits[g]) : 0; }
};

static inline int grid_v(int64_t n, int threads = 256)
{
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)runtime().num_sms * 16;
    if (b > cap) b = cap;
    return b < 1 ? 1 : (int)b;
}

// One host read per call: the scratch in one block (the stream's scratch
// buffer when the library owns the stream; the totals, the two bitmaps and
// the scan's workspace adjacent, cleared by one memset), the output
// positions by a single-launch scan, then the result at its exact size.
template <class SR>
static int mxv_t(DevCSR &w, const DevCSR *mask, bool comp, const DevCSR &A,
                 const DevCSR &u, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t m = A.nrows, n = A.ncols;
    Carve cv(s);
    uint32_t *ubits = nullptr, *mbits = nullptr;
    unsigned long long *lbws = nullptr;
    const int64_t ng = (m + 31) / 32;
    int64_t *tot = nullptr, *pos = nullptr;
    Z *ud = nullptr, *wd = nullptr;
    uint32_t *gbits = nullptr;
    auto layout = [&]() {
        tot = cv.take<int64_t>(2);
        ubits = cv.take<uint32_t>(n / 32 + 2);
        mbits = cv.take<uint32_t>(m / 32 + 2);
        gbits = cv.take<uint32_t>(ng + 1);
        lbws = cv.take<unsigned long long>(lb_ws_elems(ng + 1));
        ud = cv.take<Z>(n + 1);
        wd = cv.take<Z>(m + 1);
        pos = cv.take<int64_t>(ng + 1);
    };
    layout();
    CallBlock blk(s);
    if (!blk.get(cv.off)) return OUT_OF_MEMORY;
    cv.base = blk.base;
    cv.off = 0;
    layout();
    cudaMemsetAsync(tot, 0, (size_t)((char *)(lbws + lb_ws_elems(ng + 1)) - (char *)tot), s);
    if (u.nnz > 0)
        k_scatter_vec<Z><<<grid_v(u.nnz), 256, 0, s>>>(u.j, (const Z *)u.x, u.iso, u.nnz,
                                                       ud, ubits);
    if (mask && mask->nnz > 0)
        k_scatter_bits<<<grid_v(mask->nnz), 256, 0, s>>>(mask->j, mask->nnz, mbits);
    const int ps = prof_begin("mxv", s);
    constexpr bool maxk = SR::add_op == OP_MAX &&
                          (SR::mult_op == OP_SECONDI || SR::mult_op == OP_FIRSTJ);
    if (m > 0 && maxk)
        k_mxv_rows_maxk<SR><<<grid_v(m), 256, 0, s>>>(m, A.p, A.j, ubits, mbits,
            mask != nullptr, comp, wd, gbits);
    else if (m > 0)
        k_mxv_rows<SR><<<grid_v(m * 32), 256, 0, s>>>(m, A.p, A.j, A.x, A.iso, ud, ubits,
            mbits, mask != nullptr, comp, wd, gbits);
    prof_end(ps, s);
    // tot[0]: the result's size; tot[1]: the scan's error word
    lb_scan(MxvLoadGroup{gbits, ng}, pos, ng + 1, lbws, s, tot, nullptr, (int *)(tot + 1));
    int64_t hv[2] = {0, 0};
    cudaError_t e = readback(hv, tot, 16, s);
    if (e != cudaSuccess) return cuda_to_info(e);
    if ((int)hv[1]) return PANIC;
    const int64_t nw = hv[0];
    w = DevCSR();
    w.nrows = 1; w.ncols = m; w.iso = false; w.nnz = nw;
    w.p = (int32_t *)dalloc(8, s);
    w.j = (int32_t *)dalloc((size_t)(nw ? nw : 1) * 4, s);
    w.x = dalloc((size_t)(nw ? nw : 1) * sizeof(Z), s);
    if (!w.p || !w.j || !w.x) { dev_free(w, s); return OUT_OF_MEMORY; }
    k_compact_dense<Z><<<grid_v(m > 0 ? m : 1), 256, 0, s>>>(m, gbits, pos, wd, w.p, w.j,
                                                             (Z *)w.x);
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
