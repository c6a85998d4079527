// grb_ewise.cu: the write-back and layout kernels around the multiply:
//
//   accum_mask   C<M,replace> = accum(C,T), the B200 replacement of
//                GB_accum_mask (Source/mask/GB_accum_mask.c:126) for sparse
//                C, T and M.  Flat over entries (no row is too long): every
//                entry of T and of C decides, by binary searches in its row of
//                C/T and M, whether it survives; two single-launch scans give
//                each survivor its rank inside its row (the union of two
//                sorted lists), and a scatter writes the sorted result into
//                arrays sized for every entry of T and C, so the result's
//                size comes back with the call's one host read.
//   transpose    B = A' (Source/transpose/GB_transpose_cast.c:18): column
//                counts, scan, atomic scatter, then each row of B is sorted
//                by its (unique) indices with a bitonic network.
//
// Semantics (GraphBLAS C API, as the reference implements them):
//   Z = accum(C,T) on the union of the patterns (or Z = T without accum);
//   where the mask allows (i,j): C(i,j) = Z(i,j) if present, else deleted;
//   elsewhere C(i,j) keeps its old value unless replace is set.  A valued
//   mask is reduced to its true entries first; "no mask" allows everything,
//   and its complement allows nothing.

#include <cstring>
#include <vector>
#include "grb_runtime.h"
#include "grb_lookback.cuh"

namespace grb {

template <typename Z>
__device__ __forceinline__ Z apply_accum(int op, Z c, Z t)
{
    switch (op) {
        case OP_PLUS: return rn_add<Z>(c, t);
        case OP_TIMES: return rn_mul<Z>(c, t);
        case OP_MIN: return op_min<Z>(c, t);
        case OP_MAX: return op_max<Z>(c, t);
        case OP_MINUS: return (Z)(c - t);
        case OP_RMINUS: return (Z)(t - c);
        case OP_FIRST: return c;
        case OP_LOR: return (Z)((c != (Z)0) || (t != (Z)0));
        case OP_LAND: return (Z)((c != (Z)0) && (t != (Z)0));
        case OP_PAIR: return (Z)1;
        default: return t;                // SECOND, ANY
    }
}
template <> __device__ __forceinline__ bool apply_accum(int op, bool c, bool t)
{
    switch (op) {
        case OP_PLUS: case OP_LOR: case OP_MAX: return c || t;
        case OP_TIMES: case OP_LAND: case OP_MIN: return c && t;
        case OP_MINUS: case OP_RMINUS: case OP_LXOR: return c != t;
        case OP_FIRST: return c;
        case OP_PAIR: return true;
        default: return t;
    }
}

__device__ __forceinline__ int32_t row_of(const int32_t *__restrict__ p,
                                          int64_t nrows, int64_t e)
{
    return upper_bound(p, 0, (int32_t)nrows + 1, (int32_t)e) - 1;
}

__device__ __forceinline__ bool mask_allows(const int32_t *__restrict__ Mp,
                                            const int32_t *__restrict__ Mj,
                                            bool comp, int32_t i, int32_t j)
{
    if (Mp == nullptr) return !comp;
    const int32_t lo = Mp[i], hi = Mp[i + 1];
    const int32_t q = lower_bound(Mj, lo, hi, j);
    const bool present = q < hi && Mj[q] == j;
    return comp ? !present : present;
}

template <typename Z>
__global__ void k_am_tside(int64_t m, const int32_t *__restrict__ Tp,
                           const int32_t *__restrict__ Tj, const Z *__restrict__ Tx,
                           bool t_iso, int64_t nT,
                           const int32_t *__restrict__ Cp, const int32_t *__restrict__ Cj,
                           const Z *__restrict__ Cx, bool c_iso,
                           const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
                           bool comp, bool m_is_t, int accum, int64_t *__restrict__ keepT,
                           Z *__restrict__ valT)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) keepT[nT] = 0;       // the scan's last input
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nT;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = row_of(Tp, m, e), j = Tj[e];
        const bool ok = m_is_t || mask_allows(Mp, Mj, comp, i, j);
        Z t = Tx[t_iso ? 0 : e];
        if (ok && accum) {
            const int32_t q = lower_bound(Cj, Cp[i], Cp[i + 1], j);
            if (q < Cp[i + 1] && Cj[q] == j) t = apply_accum<Z>(accum, Cx[c_iso ? 0 : q], t);
        }
        keepT[e] = ok ? 1 : 0;
        valT[e] = t;
    }
}

template <typename Z>
__global__ void k_am_cside(int64_t m, const int32_t *__restrict__ Cp,
                           const int32_t *__restrict__ Cj, int64_t nC,
                           const int32_t *__restrict__ Tp, const int32_t *__restrict__ Tj,
                           const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
                           bool comp, bool m_is_t, bool replace, int accum,
                           int64_t *__restrict__ keepC)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) keepC[nC] = 0;       // the scan's last input
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nC;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = row_of(Cp, m, e), j = Cj[e];
        bool keep;
        if (m_is_t) {
            // the mask is T's own pattern: one search answers both questions
            const int32_t q = lower_bound(Tj, Tp[i], Tp[i + 1], j);
            const bool in_t = q < Tp[i + 1] && Tj[q] == j;
            keep = !in_t && !replace;
        } else if (mask_allows(Mp, Mj, comp, i, j)) {
            const int32_t q = lower_bound(Tj, Tp[i], Tp[i + 1], j);
            const bool in_t = q < Tp[i + 1] && Tj[q] == j;
            keep = !in_t && accum != 0;       // Z(i,j) = C(i,j) when only C has it
        } else {
            keep = !replace;
        }
        keepC[e] = keep ? 1 : 0;
    }
}

__global__ void k_am_rowptr(int64_t m, const int32_t *__restrict__ Cp,
                            const int32_t *__restrict__ Tp,
                            const int64_t *__restrict__ sC, const int64_t *__restrict__ sT,
                            int32_t *__restrict__ Rp)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m;
         i += (int64_t)gridDim.x * blockDim.x)
        Rp[i] = (int32_t)(sC[Cp[i]] + sT[Tp[i]]);
}

// scatter the survivors of one side; `other` is the opposite side's list
template <typename Z>
__global__ void k_am_write(int64_t m, const int32_t *__restrict__ Xp,
                           const int32_t *__restrict__ Xj, const Z *__restrict__ Xv,
                           bool x_iso, int64_t nX, const int64_t *__restrict__ sX,
                           const int32_t *__restrict__ Yp, const int32_t *__restrict__ Yj,
                           const int64_t *__restrict__ sY,
                           const int32_t *__restrict__ Rp, int32_t *__restrict__ Rj,
                           Z *__restrict__ Rx)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nX;
         e += (int64_t)gridDim.x * blockDim.x) {
        if (sX[e + 1] == sX[e]) continue;           // not kept
        const int32_t i = row_of(Xp, m, e), j = Xj[e];
        const int32_t q = lower_bound(Yj, Yp[i], Yp[i + 1], j);
        const int64_t rank = (sX[e] - sX[Xp[i]]) + (sY[q] - sY[Yp[i]]);
        const int64_t pos = Rp[i] + rank;
        Rj[pos] = j;
        Rx[pos] = Xv[x_iso ? 0 : e];
    }
}

static inline int grid_n(int64_t n, int threads = 256)
{
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)runtime().num_sms * 16;
    if (b > cap) b = cap;
    return b < 1 ? 1 : (int)b;
}

// ---------------------------------------------------------------------------
// one-row union: w<u> = u with u's pattern as the structural mask, no
// accumulator, no replace (the BFS parent update) on row vectors.  The
// result is the merge of two sorted index lists in which u's entry wins a
// tie.  One launch: tiles of UN_TILE merged positions (from a ticket); a
// tile finds where its positions start in each list (merge path: a
// warp-cooperative search over the diagonal), stages both ranges in shared
// memory, each thread merges UN_ITEMS positions, the tile's kept count gets
// its offset by decoupled look-back, and the tile's output is written from
// shared memory by consecutive threads.
// ---------------------------------------------------------------------------

static constexpr int UN_THREADS = 256, UN_ITEMS = 12, UN_TILE = UN_THREADS * UN_ITEMS;

// T before C on equal keys: C[i-1] precedes T[d-i] iff C[i-1] < T[d-i].
// The number of C entries among the first d merged positions: the largest
// i in [max(0, d - nT), min(d, nC)] with i == 0, d - i >= nT or
// C[i-1] < T[d-i]; all lanes of the warp search together, 32 candidates a
// step.
__device__ __forceinline__ int64_t union_split(const int32_t *__restrict__ C, int64_t nC,
                                               const int32_t *__restrict__ T, int64_t nT,
                                               int64_t d, int lane)
{
    int64_t lo = d - nT > 0 ? d - nT : 0;
    int64_t hi = d < nC ? d : nC;
    while (lo < hi) {
        const int64_t step = (hi - lo + 31) / 32;
        const int64_t c = lo + 1 + (int64_t)lane * step;
        bool q = false;
        if (c <= hi) q = (d - c >= nT) || (C[c - 1] < T[d - c]);
        const unsigned m = __ballot_sync(0xffffffffu, q);
        if (m == 0) { hi = lo; break; }
        const int k = 31 - __clz(m);
        lo = lo + 1 + (int64_t)k * step;
        const int64_t h2 = lo + step - 1;
        hi = h2 < hi ? h2 : hi;
    }
    return lo;
}

template <typename Z>
__global__ void __launch_bounds__(UN_THREADS)
k_union_row(const int32_t *__restrict__ Cj, const Z *__restrict__ Cx, bool c_iso, int64_t nC,
            const int32_t *__restrict__ Tj, const Z *__restrict__ Tx, bool t_iso, int64_t nT,
            int32_t *__restrict__ Rp, int32_t *__restrict__ Rj, Z *__restrict__ Rx,
            int64_t *__restrict__ total, int64_t ntiles, unsigned long long *__restrict__ ws,
            int *__restrict__ err)
{
    __shared__ int s_tile, s_last, s_agg;
    __shared__ long long s_ex;
    __shared__ int64_t s_i0, s_i1;
    __shared__ int s_w[UN_THREADS / 32];
    // the staged input indices, then (after the merge) the staged output:
    // its indices and the source of each (a position in C, or in T with the
    // top bit set); the values are gathered while the output is written
    __shared__ __align__(16) int32_t s_buf[2 * UN_TILE];
    int32_t *s_c = s_buf, *s_t = s_buf + UN_TILE;
    int32_t *s_oj = s_buf, *s_os = s_buf + UN_TILE;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    unsigned long long *status = ws + 2;
    if (tid == 0) s_tile = (int)atomicAdd(&ws[0], 1ull);
    __syncthreads();
    const int64_t tile = s_tile;
    const int64_t nd = nC + nT;
    const int64_t d0 = tile * UN_TILE;
    const int64_t d1 = d0 + UN_TILE < nd ? d0 + UN_TILE : nd;
    if (w == 0) {
        const int64_t a = union_split(Cj, nC, Tj, nT, d0, lane);
        if (lane == 0) s_i0 = a;
    } else if (w == 1) {
        const int64_t b = union_split(Cj, nC, Tj, nT, d1, lane);
        if (lane == 0) s_i1 = b;
    }
    __syncthreads();
    const int64_t i0 = s_i0, i1 = s_i1, j0 = d0 - i0, j1 = d1 - i1;
    const int nc = (int)(i1 - i0), nt = (int)(j1 - j0);
    for (int k = tid; k < nc; k += UN_THREADS) s_c[k] = Cj[i0 + k];
    for (int k = tid; k < nt; k += UN_THREADS) s_t[k] = Tj[j0 + k];
    const int32_t tprev = j0 > 0 ? Tj[j0 - 1] : -1;     // the T entry before the tile's
    __syncthreads();
    // this thread's positions [dl, dl + UN_ITEMS) of the tile, merged locally
    const int dl = tid * UN_ITEMS;
    const int nl = (int)(d1 - d0);
    int ci = 0, tj = 0;
    if (dl < nl) {
        // the split of diagonal dl within the staged ranges
        int lo = dl - nt > 0 ? dl - nt : 0, hi = dl < nc ? dl : nc;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if ((dl - mid >= nt) || (s_c[mid - 1] < s_t[dl - mid])) lo = mid; else hi = mid - 1;
        }
        ci = lo;
        tj = dl - lo;
    }
    int32_t oj[UN_ITEMS], os[UN_ITEMS];
    int kept = 0;
    for (int k = 0; k < UN_ITEMS && dl + k < nl; k++) {
        if (tj < nt && (ci >= nc || s_t[tj] <= s_c[ci])) {
            oj[kept] = s_t[tj];
            os[kept] = (int32_t)(0x80000000u | (uint32_t)tj);
            kept++;
            tj++;
        } else {
            const int32_t key = s_c[ci];
            const int32_t before = tj > 0 ? s_t[tj - 1] : tprev;
            if (before != key) {
                oj[kept] = key;
                os[kept] = ci;
                kept++;
            }
            ci++;
        }
    }
    int x = kept;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
        int v = lane < UN_THREADS / 32 ? s_w[lane] : 0;
        const int ownv = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        const long long agg = __shfl_sync(0xffffffffu, v, 31);
        if (lane < UN_THREADS / 32) s_w[lane] = v - ownv;
        long long ex = 0;
        if (tile == 0) {
            if (lane == 0) atomicExch(&status[0], LB_INC | ((unsigned long long)agg & LB_VAL));
        } else {
            if (lane == 0) atomicExch(&status[tile], LB_AGG | ((unsigned long long)agg & LB_VAL));
            ex = lb_lookback(status, tile, lane, err);
            if (lane == 0)
                atomicExch(&status[tile], LB_INC | ((unsigned long long)(ex + agg) & LB_VAL));
        }
        if (lane == 0) {
            s_ex = ex;
            s_agg = (int)agg;
            if (tile == 0) Rp[0] = 0;
            if (tile == ntiles - 1) { Rp[1] = (int32_t)(ex + agg); *total = ex + agg; }
        }
    }
    // (the block barrier above also ends every read of the staged inputs)
    __syncthreads();
    int loc = s_w[w] + (x - kept);
    for (int k = 0; k < kept; k++) { s_oj[loc + k] = oj[k]; s_os[loc + k] = os[k]; }
    __syncthreads();
    const int64_t base = s_ex;
    const int agg = s_agg;
    // all of a thread's value loads first (independent, so they overlap),
    // then its stores
    Z v[UN_ITEMS];
    #pragma unroll
    for (int r = 0; r < UN_ITEMS; r++) {
        const int k = tid + r * UN_THREADS;
        if (k < agg) {
            const int32_t src = s_os[k];
            v[r] = src < 0 ? Tx[t_iso ? 0 : j0 + (src & 0x7fffffff)] : Cx[c_iso ? 0 : i0 + src];
        }
    }
    #pragma unroll
    for (int r = 0; r < UN_ITEMS; r++) {
        const int k = tid + r * UN_THREADS;
        if (k < agg) {
            Rj[base + k] = s_oj[k];
            Rx[base + k] = v[r];
        }
    }
    // the last tile to finish clears the workspace
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(&ws[1], 1ull) == (unsigned long long)(ntiles - 1);
    }
    __syncthreads();
    if (s_last) {
        for (int64_t t = tid; t < ntiles; t += UN_THREADS) status[t] = 0;
        if (tid == 0) { ws[0] = 0; ws[1] = 0; }
    }
}

// C = C union T on one row, T's entries winning ties (w<u> = u)
template <typename Z>
static int union_row_t(DevCSR &C, const DevCSR &T, cudaStream_t s)
{
    const int64_t nC = C.nnz, nT = T.nnz, nd = nC + nT;
    if (nd >= INT32_MAX) return OUT_OF_MEMORY;
    const int64_t ntiles = nd > 0 ? (nd + UN_TILE - 1) / UN_TILE : 0;
    Carve cv(s);
    int64_t *tot_d = nullptr;
    unsigned long long *ws = nullptr;
    auto layout = [&]() {
        tot_d = cv.take<int64_t>(2);
        ws = cv.take<unsigned long long>(ntiles + 2);
    };
    layout();
    if (!cv.alloc()) return OUT_OF_MEMORY;
    layout();
    struct Release { Carve &c; ~Release() { dfree(c.base, c.s); } } release{cv};
    DevCSR R;
    R.nrows = 1; R.ncols = T.ncols; R.type = T.type; R.iso = false;
    R.p = (int32_t *)dalloc(2 * 4, s);
    R.j = (int32_t *)dalloc((size_t)(nd ? nd : 1) * 4, s);
    R.x = dalloc((size_t)(nd ? nd : 1) * sizeof(Z), s);
    if (!R.p || !R.j || !R.x) { dev_free(R, s); return OUT_OF_MEMORY; }
    int64_t tot[2] = {0, 0};
    if (ntiles > 0) {
        cudaMemsetAsync(tot_d, 0, (size_t)((char *)(ws + ntiles + 2) - (char *)tot_d), s);
        k_union_row<Z><<<(unsigned)ntiles, UN_THREADS, 0, s>>>(C.j, (const Z *)C.x, C.iso, nC,
            T.j, (const Z *)T.x, T.iso, nT, R.p, R.j, (Z *)R.x, tot_d, ntiles, ws,
            (int *)(tot_d + 1));
        cudaError_t e = readback(tot, tot_d, 16, s);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) { dev_free(R, s); return cuda_to_info(e); }
        if ((int)tot[1] != 0) { dev_free(R, s); return PANIC; }
    } else {
        cudaMemsetAsync(R.p, 0, 2 * 4, s);
    }
    R.nnz = tot[0];
    dev_free(C, s);
    C = R;
    return SUCCESS;
}

template <typename Z>
static int accum_mask_t(DevCSR &C, const DevCSR &T, const DevCSR *M, bool comp,
                        bool replace, int accum, cudaStream_t s)
{
    const int64_t m = T.nrows, nT = T.nnz, nC = C.nnz;
    if (m == 1 && M && !comp && !replace && !accum && M->p == T.p && M->j == T.j)
        return union_row_t<Z>(C, T, s);
    // the totals and error word, the two scans' workspaces, the keep flags /
    // offsets of both sides and T's values in one allocation; the first three
    // are cleared by one memset
    Carve cv(s);
    int64_t *keepT = nullptr, *keepC = nullptr, *tot_d = nullptr;
    unsigned long long *lbT = nullptr, *lbC = nullptr;
    Z *valT = nullptr;
    auto layout = [&]() {
        tot_d = cv.take<int64_t>(4);
        lbT = cv.take<unsigned long long>(scan_lb_ws_elems(nT + 1));
        lbC = cv.take<unsigned long long>(scan_lb_ws_elems(nC + 1));
        keepT = cv.take<int64_t>(nT + 1);
        keepC = cv.take<int64_t>(nC + 1);
        valT = cv.take<Z>(nT + 1);
    };
    layout();
    if (!cv.alloc()) return OUT_OF_MEMORY;
    layout();
    struct Release { Carve &c; ~Release() { dfree(c.base, c.s); } } release{cv};
    cudaMemsetAsync(tot_d, 0, (size_t)((char *)(lbC + scan_lb_ws_elems(nC + 1)) - (char *)tot_d),
                    s);
    int *err = (int *)(tot_d + 2);
    const int32_t *Mp = M ? M->p : nullptr, *Mj = M ? M->j : nullptr;
    // C<T> = T (a structural mask that is T itself, as in w<q> = q): every
    // entry of T is allowed, and an entry of C is under the mask exactly
    // when T holds it
    const bool m_is_t = M && !comp && M->p == T.p && M->j == T.j;
    k_am_tside<Z><<<grid_n(nT), 256, 0, s>>>(m, T.p, T.j, (const Z *)T.x, T.iso, nT,
        C.p, C.j, (const Z *)C.x, C.iso, Mp, Mj, comp, m_is_t, accum, keepT, valT);
    k_am_cside<Z><<<grid_n(nC), 256, 0, s>>>(m, C.p, C.j, nC, T.p, T.j, Mp, Mj,
        comp, m_is_t, replace, accum, keepC);
    scan_exclusive_lb(keepT, keepT, nT + 1, lbT, s, tot_d, nullptr, err);
    scan_exclusive_lb(keepC, keepC, nC + 1, lbC, s, tot_d + 1, nullptr, err);
    // the result is written before its size comes back, into arrays that
    // hold every entry of T and C; they are trimmed afterwards if the result
    // is much smaller
    const int64_t cap = nT + nC;
    if (cap >= INT32_MAX) return OUT_OF_MEMORY;
    DevCSR R;
    R.nrows = m; R.ncols = T.ncols; R.type = T.type; R.iso = false;
    R.p = (int32_t *)dalloc((size_t)(m + 1) * 4, s);
    R.j = (int32_t *)dalloc((size_t)(cap ? cap : 1) * 4, s);
    R.x = dalloc((size_t)(cap ? cap : 1) * sizeof(Z), s);
    if (!R.p || !R.j || !R.x) { dev_free(R, s); return OUT_OF_MEMORY; }
    k_am_rowptr<<<grid_n(m + 1), 256, 0, s>>>(m, C.p, T.p, keepC, keepT, R.p);
    if (nT > 0)
        k_am_write<Z><<<grid_n(nT), 256, 0, s>>>(m, T.p, T.j, valT, false, nT, keepT,
            C.p, C.j, keepC, R.p, R.j, (Z *)R.x);
    if (nC > 0)
        k_am_write<Z><<<grid_n(nC), 256, 0, s>>>(m, C.p, C.j, (const Z *)C.x, C.iso, nC,
            keepC, T.p, T.j, keepT, R.p, R.j, (Z *)R.x);
    int64_t tot[3] = {0, 0, 0};
    cudaError_t e = readback(tot, tot_d, 24, s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) { dev_free(R, s); return cuda_to_info(e); }
    if ((int)tot[2] != 0) { dev_free(R, s); return PANIC; }
    const int64_t nR = tot[0] + tot[1];
    R.nnz = nR;
    if (cap > 2 * nR + 4096) {
        int32_t *j2 = (int32_t *)dalloc((size_t)(nR ? nR : 1) * 4, s);
        void *x2 = dalloc((size_t)(nR ? nR : 1) * sizeof(Z), s);
        if (j2 && x2) {
            cudaMemcpyAsync(j2, R.j, (size_t)nR * 4, cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(x2, R.x, (size_t)nR * sizeof(Z), cudaMemcpyDeviceToDevice, s);
            dfree(R.j, s); dfree(R.x, s);
            R.j = j2; R.x = x2;
        } else {
            dfree(j2, s); dfree(x2, s);
        }
    }
    dev_free(C, s);
    C = R;
    return SUCCESS;
}

int accum_mask(DevCSR &C, const DevCSR &T0, const DevCSR *M0, bool mask_comp,
               bool mask_struct, bool replace, int accum, cudaStream_t s)
{
    if (C.nrows != T0.nrows || C.ncols != T0.ncols) return DIMENSION_MISMATCH;
    if (M0 && (M0->nrows != C.nrows || M0->ncols != C.ncols)) return DIMENSION_MISMATCH;
    if (C.nnz > 0 && C.type != T0.type) return DOMAIN_MISMATCH;
    // zombie-free operands with sorted rows
    DevCSR T = T0, Ms;
    bool ownT = false, ownM = false;
    int info = SUCCESS;
    if (T0.nzombies > 0) {
        T = DevCSR();
        T.nrows = T0.nrows; T.ncols = T0.ncols; T.nnz = T0.nnz; T.type = T0.type;
        T.iso = T0.iso; T.nzombies = T0.nzombies;
        size_t ts = type_size(T0.type);
        T.p = (int32_t *)dalloc((size_t)(T0.nrows + 1) * 4, s);
        T.j = (int32_t *)dalloc((size_t)(T0.nnz ? T0.nnz : 1) * 4, s);
        T.x = dalloc(T0.iso ? ts : (size_t)(T0.nnz ? T0.nnz : 1) * ts, s);
        if (!T.p || !T.j || !T.x) { dev_free(T, s); return OUT_OF_MEMORY; }
        cudaMemcpyAsync(T.p, T0.p, (size_t)(T0.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(T.j, T0.j, (size_t)T0.nnz * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(T.x, T0.x, T0.iso ? ts : (size_t)T0.nnz * ts, cudaMemcpyDeviceToDevice, s);
        info = dev_prune_zombies(T, s);
        ownT = true;
    }
    if (info == SUCCESS && C.nzombies > 0) info = dev_prune_zombies(C, s);
    const DevCSR *M = M0;
    if (info == SUCCESS && M0 && (!mask_struct && M0->x)) {
        info = dev_mask_to_struct(Ms, *M0, s);
        M = &Ms; ownM = true;
    } else if (info == SUCCESS && M0 && M0->nzombies > 0) {
        info = NO_VALUE;
    }
    if (info == SUCCESS) {
        if (C.nnz == 0 && C.type != T.type) C.type = T.type;
        switch (T.type) {
            case T_BOOL:   info = accum_mask_t<bool>(C, T, M, mask_comp, replace, accum, s); break;
            case T_INT32:  info = accum_mask_t<int32_t>(C, T, M, mask_comp, replace, accum, s); break;
            case T_UINT32: info = accum_mask_t<uint32_t>(C, T, M, mask_comp, replace, accum, s); break;
            case T_INT64:  info = accum_mask_t<int64_t>(C, T, M, mask_comp, replace, accum, s); break;
            case T_UINT64: info = accum_mask_t<uint64_t>(C, T, M, mask_comp, replace, accum, s); break;
            case T_FP32:   info = accum_mask_t<float>(C, T, M, mask_comp, replace, accum, s); break;
            case T_FP64:   info = accum_mask_t<double>(C, T, M, mask_comp, replace, accum, s); break;
            default: info = NO_VALUE;
        }
    }
    if (ownT) dev_free(T, s);
    if (ownM) dev_free(Ms, s);
    return info;
}

// ---------------------------------------------------------------------------
// transpose
// ---------------------------------------------------------------------------

__global__ void k_col_count(const int32_t *__restrict__ Aj, int64_t nnz,
                            int32_t *__restrict__ cnt)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[Aj[e]], 1);
}

template <typename Z>
__global__ void k_tr_scatter(int64_t m, const int32_t *__restrict__ Ap,
                             const int32_t *__restrict__ Aj, const Z *__restrict__ Ax,
                             bool iso, int64_t nnz, const int64_t *__restrict__ Bp,
                             int32_t *__restrict__ fill, int32_t *__restrict__ Bj,
                             Z *__restrict__ Bx)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = row_of(Ap, m, e), j = Aj[e];
        const int64_t pos = Bp[j] + atomicAdd(&fill[j], 1);
        Bj[pos] = i;
        if (Bx) Bx[pos] = Ax[iso ? 0 : e];
    }
}

// sort every row by index: one warp per row of up to SORT_W entries in shared
// memory; longer rows are sorted by a whole block in global memory
template <typename Z, int SORT_W>
__global__ void __launch_bounds__(128)
k_sort_rows_warp(int64_t m, const int64_t *__restrict__ Bp, int32_t *__restrict__ Bj,
                 Z *__restrict__ Bx)
{
    __shared__ int32_t sk[4][SORT_W];
    __shared__ Z sv[4][SORT_W];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m;
         r += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t lo = Bp[r];
        const int n = (int)(Bp[r + 1] - lo);
        if (n <= 1 || n > SORT_W) continue;
        int n2 = 1;
        while (n2 < n) n2 <<= 1;
        for (int q = lane; q < n2; q += 32) {
            if (q < n) { sk[w][q] = Bj[lo + q]; if (Bx) sv[w][q] = Bx[lo + q]; }
            else sk[w][q] = INT32_MAX;
        }
        __syncwarp();
        for (int size = 2; size <= n2; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int q = lane; q < n2; q += 32) {
                    const int pq = q ^ stride;
                    if (pq > q) {
                        const bool up = (q & size) == 0;
                        const int32_t a = sk[w][q], b = sk[w][pq];
                        if ((a > b) == up) {
                            sk[w][q] = b; sk[w][pq] = a;
                            if (Bx) { Z t = sv[w][q]; sv[w][q] = sv[w][pq]; sv[w][pq] = t; }
                        }
                    }
                }
                __syncwarp();
            }
        for (int q = lane; q < n; q += 32) { Bj[lo + q] = sk[w][q]; if (Bx) Bx[lo + q] = sv[w][q]; }
        __syncwarp();
    }
}

// one block per long row: bitonic sort over a padded scratch copy
template <typename Z>
__global__ void __launch_bounds__(512)
k_sort_rows_block(const int32_t *__restrict__ rows, int nrows_long,
                  const int64_t *__restrict__ Bp, int32_t *__restrict__ Bj,
                  Z *__restrict__ Bx, int32_t *__restrict__ sk_all, Z *__restrict__ sv_all,
                  const int64_t *__restrict__ soff)
{
    for (int t = blockIdx.x; t < nrows_long; t += gridDim.x) {
        const int32_t r = rows[t];
        const int64_t lo = Bp[r];
        const int64_t n = Bp[r + 1] - lo;
        int64_t n2 = 1;
        while (n2 < n) n2 <<= 1;
        int32_t *sk = sk_all + soff[t];
        Z *sv = sv_all + soff[t];
        for (int64_t q = threadIdx.x; q < n2; q += blockDim.x) {
            if (q < n) { sk[q] = Bj[lo + q]; if (Bx) sv[q] = Bx[lo + q]; }
            else sk[q] = INT32_MAX;
        }
        __syncthreads();
        for (int64_t size = 2; size <= n2; size <<= 1)
            for (int64_t stride = size >> 1; stride > 0; stride >>= 1) {
                for (int64_t q = threadIdx.x; q < n2; q += blockDim.x) {
                    const int64_t pq = q ^ stride;
                    if (pq > q) {
                        const bool up = (q & size) == 0;
                        const int32_t a = sk[q], b = sk[pq];
                        if ((a > b) == up) {
                            sk[q] = b; sk[pq] = a;
                            if (Bx) { Z tv = sv[q]; sv[q] = sv[pq]; sv[pq] = tv; }
                        }
                    }
                }
                __syncthreads();
            }
        for (int64_t q = threadIdx.x; q < n; q += blockDim.x) {
            Bj[lo + q] = sk[q];
            if (Bx) Bx[lo + q] = sv[q];
        }
        __syncthreads();
    }
}

__global__ void k_i64_to_i32_e(const int64_t *__restrict__ in, int32_t *__restrict__ out,
                               int64_t n)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        out[t] = (int32_t)in[t];
}

template <typename Z>
static int transpose_t(DevCSR &B, const DevCSR &A, cudaStream_t s)
{
    const int64_t m = A.nrows, n = A.ncols, nnz = A.nnz;
    constexpr int SORT_W = 512;
    Scratch ws(s);
    int32_t *cnt = ws.get<int32_t>(n + 1);
    int64_t *Bp64 = ws.get<int64_t>(n + 1);
    int32_t *fill = ws.get<int32_t>(n + 1);
    if (ws.failed) return OUT_OF_MEMORY;
    cudaMemsetAsync(cnt, 0, (size_t)(n + 1) * 4, s);
    cudaMemsetAsync(fill, 0, (size_t)(n + 1) * 4, s);
    if (nnz > 0) k_col_count<<<grid_n(nnz), 256, 0, s>>>(A.j, nnz, cnt);
    int info = scan_exclusive_i32_to_i64(cnt, Bp64, n + 1, s);
    if (info != SUCCESS) return info;
    B = DevCSR();
    B.nrows = n; B.ncols = m; B.nnz = nnz; B.type = A.type; B.iso = A.iso;
    size_t ts = type_size(A.type);
    B.p = (int32_t *)dalloc((size_t)(n + 1) * 4, s);
    B.j = (int32_t *)dalloc((size_t)(nnz ? nnz : 1) * 4, s);
    B.x = A.x ? dalloc(A.iso ? ts : (size_t)(nnz ? nnz : 1) * ts, s) : nullptr;
    if (!B.p || !B.j || (A.x && !B.x)) { dev_free(B, s); return OUT_OF_MEMORY; }
    k_i64_to_i32_e<<<grid_n(n + 1), 256, 0, s>>>(Bp64, B.p, n + 1);
    Z *Bx = (A.x && !A.iso) ? (Z *)B.x : nullptr;
    if (A.x && A.iso) cudaMemcpyAsync(B.x, A.x, ts, cudaMemcpyDeviceToDevice, s);
    if (nnz > 0) {
        k_tr_scatter<Z><<<grid_n(nnz), 256, 0, s>>>(m, A.p, A.j, (const Z *)A.x, A.iso,
            nnz, Bp64, fill, B.j, Bx);
        k_sort_rows_warp<Z, SORT_W><<<grid_n(n * 32, 128), 128, 0, s>>>(n, Bp64, B.j, Bx);
        // long rows: gather their ids and sort each with a block
        std::vector<int64_t> hp((size_t)n + 1);
        cudaMemcpyAsync(hp.data(), Bp64, (size_t)(n + 1) * 8, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { dev_free(B, s); return cuda_to_info(e); }
        std::vector<int32_t> longr;
        std::vector<int64_t> off;
        int64_t tot = 0;
        for (int64_t r = 0; r < n; r++) {
            int64_t len = hp[r + 1] - hp[r];
            if (len > SORT_W) {
                int64_t n2 = 1;
                while (n2 < len) n2 <<= 1;
                longr.push_back((int32_t)r);
                off.push_back(tot);
                tot += n2;
            }
        }
        if (!longr.empty()) {
            int32_t *drows = ws.get<int32_t>(longr.size());
            int64_t *doff = ws.get<int64_t>(off.size());
            int32_t *sk = ws.get<int32_t>(tot);
            Z *sv = ws.get<Z>(tot);
            if (ws.failed) { dev_free(B, s); return OUT_OF_MEMORY; }
            cudaMemcpyAsync(drows, longr.data(), longr.size() * 4, cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(doff, off.data(), off.size() * 8, cudaMemcpyHostToDevice, s);
            int nb = (int)longr.size();
            k_sort_rows_block<Z><<<nb < 1024 ? nb : 1024, 512, 0, s>>>(drows, nb, Bp64,
                B.j, Bx, sk, sv, doff);
        }
    }
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { dev_free(B, s); return cuda_to_info(e); }
    return SUCCESS;
}

int transpose(DevCSR &B, const DevCSR &A0, cudaStream_t s)
{
    DevCSR A = A0;
    DevCSR P;
    bool own = false;
    if (A0.nzombies > 0) {
        // transpose the live entries only
        P = DevCSR();
        P.nrows = A0.nrows; P.ncols = A0.ncols; P.nnz = A0.nnz; P.type = A0.type;
        P.iso = A0.iso; P.nzombies = A0.nzombies;
        size_t ts = type_size(A0.type);
        P.p = (int32_t *)dalloc((size_t)(A0.nrows + 1) * 4, s);
        P.j = (int32_t *)dalloc((size_t)(A0.nnz ? A0.nnz : 1) * 4, s);
        P.x = A0.x ? dalloc(A0.iso ? ts : (size_t)(A0.nnz ? A0.nnz : 1) * ts, s) : nullptr;
        if (!P.p || !P.j || (A0.x && !P.x)) { dev_free(P, s); return OUT_OF_MEMORY; }
        cudaMemcpyAsync(P.p, A0.p, (size_t)(A0.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(P.j, A0.j, (size_t)A0.nnz * 4, cudaMemcpyDeviceToDevice, s);
        if (A0.x) cudaMemcpyAsync(P.x, A0.x, A0.iso ? ts : (size_t)A0.nnz * ts,
                                  cudaMemcpyDeviceToDevice, s);
        int info = dev_prune_zombies(P, s);
        if (info != SUCCESS) { dev_free(P, s); return info; }
        A = P; own = true;
    }
    int info;
    switch (type_size(A.type)) {
        case 1: info = transpose_t<uint8_t>(B, A, s); break;
        case 4: info = transpose_t<uint32_t>(B, A, s); break;
        case 8: info = transpose_t<uint64_t>(B, A, s); break;
        default: info = NO_VALUE;
    }
    if (own) dev_free(P, s);
    return info;
}

}  // namespace grb
