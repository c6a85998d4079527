// grb_saxpy3.cu: row-wise (Gustavson) semiring SpGEMM, C<M> = A*B with
// C(i,:) = sum over k in A(i,:) of A(i,k) (x) B(k,:); the B200 replacement of
// GB_AxB_saxpy3 (Source/mxm/GB_AxB_saxpy3.c:119).  The reference has no GPU
// saxpy3; this is new.
//
// Phases (all on one stream, no host round trip until the output size):
//   1. flop count per row, flops[i] = sum_k nnz(B(k,:)) (the reference's
//      GB_AxB_saxpy3_flopcount, Source/mxm/GB_AxB_saxpy3_flopcount.c:81),
//      capped by nnz(M(i,:)) when a plain mask bounds the row, and bin
//      assignment by size class.
//   2. device exclusive scan of the row capacities -> offsets of each row's
//      slot in a temporary output (capacity = min(flops, ncols, |M(i,:)|)).
//   3. numeric, one kernel per bin:
//        short rows (<= 256 products by default): one warp expands the row's
//        products into shared memory, sorts them by (column, position) and
//        folds equal columns in ascending k (expand-sort-compress);
//        medium rows: a group of TPR threads owns one row and a
//        shared-memory open-addressing hash table of CAP slots (the
//        reference's coarse hash task, GB_AxB_saxpy3_coarseHash_phase5.c,
//        with linear probing on GB_HASHF-style keys, math/include/GB_hash.h);
//        heavy rows: a dense accumulator in global memory (Gustavson,
//        GB_AxB_saxpy3_coarseGus_*_phase5.c) with block-cooperative, ordered
//        compaction.
//      In every bin the row's k loop runs in ascending k and the threads of
//      the group split B(k,:), whose column indices are distinct, so every
//      C(i,j) sees its terms in the reference's order: first term written,
//      later terms folded with the monoid's UPDATE.  This makes floating
//      PLUS bit-exact as well.  Order-free monoids on heavy rows instead
//      spread all products over the grid (a flat product index: the heavy
//      rows' A entries and each one's B-row length, scanned) with atomic
//      updates into a dense row of byte flags and values, skipping the atomic
//      when an idempotent monoid's value cannot change.
//   4. each row's entries are sorted by column in shared memory (bitonic) and
//      written to its slot; a compaction kernel packs the slots into CSR.
//
// Masks: in the hash bins M (or !M) is scattered into the row's table first
// (the reference's "scatter M" step, GB_AxB_saxpy3_symbolic.c), with a state
// per slot: allowed-unset, set, or forbidden; the expand-sort-compress bin
// checks each product's column against M(i,:) by binary search; heavy rows
// mark the dense row's flags.

#include <atomic>
#include <functional>
#include <mutex>
#include <vector>
#include <cstdio>
#include <cstring>
#include "grb_saxpy3.h"
#include "grb_semirings.h"
#include "grb_lookback.cuh"

namespace grb {

static constexpr int MAX_SMEM_BINS = 6;

// slot states
static constexpr uint8_t S_EMPTY = 0, S_ALLOWED = 1, S_SET = 2, S_FORBID = 3;

// The rows of one shared-memory bin, read on the device: the bins' row lists
// lie end to end in `list` in bin order, count[b] rows in bin b (count[0],
// the rows without products, is 0).  When `need` is set the kernel first
// checks that the slots it writes fit: *need (the slot total) <= avail, else
// it does nothing and the host, which reads the total, runs it again with
// more slots.
struct BinRows {
    const int32_t *list;
    const int *count;
    int b;
    const int64_t *need;
    int64_t avail;
    __device__ int get(const int32_t *&rows) const
    {
        if (need && *need > avail) { rows = list; return 0; }
        int start = 0;
        for (int q = 0; q < b; q++) start += count[q];
        rows = list + start;
        return count[b];
    }
};

// ---------------------------------------------------------------------------
// phase 1: flops and capacity per row
// ---------------------------------------------------------------------------

// Flat over A's entries, so a row of any length is spread over the whole
// grid (a one-row A, as in vxm, would otherwise run on one warp): each lane
// takes one entry A(i,k) and adds nnz(B(k,:)); a segmented scan over the
// warp's lanes (rows are contiguous in lane order) gives each row segment its
// sum, and the segment that runs on into the next 32 entries is carried
// instead of added, so a warp adds once per row it touches in its span (a
// single long row takes one atomic per span, not one per 32 entries).
// flops[] must be zero on entry.
__global__ void __launch_bounds__(256)
k_flops_flat(const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
             const int32_t *__restrict__ Bp, int64_t nrows, int64_t nnz, int span,
             unsigned long long *__restrict__ flops)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // each warp owns spans of `span` consecutive entries (a multiple of 32):
    // one warp-cooperative search per span, then the row carries over from
    // one 32-entry step to the next
    for (int64_t s0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * span;
         s0 < nnz; s0 += nw * span) {
        int32_t r0 = warp_last_le<int32_t, int32_t>(Ap, (int32_t)nrows, (int32_t)s0, lane);
        const int64_t s1 = s0 + span < nnz ? s0 + span : nnz;
        // the open segment of the previous step: its row and its sum so far
        int32_t crow = -1;
        unsigned long long carry = 0;
        for (int64_t base = s0; base < s1; base += 32) {
            const int64_t e = base + lane;
            int32_t r = -1;
            unsigned long long f = 0;
            if (e < s1) {
                r = r0;
                while (Ap[r + 1] <= e) r++;
                const int32_t k = Aj[e];
                f = (unsigned long long)(Bp[k + 1] - Bp[k]);
            }
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, f, o);
                const int32_t ry = __shfl_up_sync(0xffffffffu, r, o);
                if (lane >= o && ry == r) f += y;
            }
            // rows only grow along the span: only this step's first segment
            // can continue the open one
            if (r >= 0 && r == crow) f += carry;
            const int32_t first = __shfl_sync(0xffffffffu, r, 0);
            if (crow >= 0 && first != crow && lane == 0) atomicAdd(&flops[crow], carry);
            const int32_t rn = __shfl_down_sync(0xffffffffu, r, 1);
            const bool end = r >= 0 && (lane == 31 || rn != r);
            if (end && lane != 31) atomicAdd(&flops[r], f);
            // lane 31's segment stays open (flushed when its row ends)
            crow = __shfl_sync(0xffffffffu, r, 31);
            carry = __shfl_sync(0xffffffffu, f, 31);
            // the next step starts in the row of this step's last entry
            r0 = crow >= 0 ? crow : r0;
        }
        if (crow >= 0 && lane == 0) atomicAdd(&flops[crow], carry);
    }
}

// bin of a row: 0 empty, 1..nb shared-memory hash bins (by the config's
// limits on flops + mask entries), nb+1 heavy (dense accumulator)
struct BinLimits { int nb; int64_t limit[MAX_SMEM_BINS]; };

// The same pass writes each row's slot capacity, min(flops, ncols,
// |M(i,:)| when a plain mask bounds the row), 0 for an empty row.
__global__ void k_bin_rows(const int64_t *__restrict__ flops,
                           const int32_t *__restrict__ Mp, bool has_mask,
                           bool mask_bounds, int64_t ncols,
                           int64_t nrows, BinLimits lim, int *__restrict__ bin_count,
                           int8_t *__restrict__ row_bin, int64_t *__restrict__ cap,
                           const int32_t *__restrict__ Ap,
                           unsigned long long *__restrict__ heavy_alen)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // warp-uniform loop: the bin counters take one atomic per bin per warp
    for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); r0 < nrows;
         r0 += stride) {
        const int64_t r = r0 + lane;
        int b = -1;
        if (r < nrows) {
            const int64_t f = flops[r];
            int64_t c = f < ncols ? f : ncols;
            if (mask_bounds) {
                const int64_t mc = Mp[r + 1] - Mp[r];
                if (mc < c) c = mc;
            }
            cap[r] = f == 0 ? 0 : c;
            if (f == 0) b = 0;
            else {
                const int64_t need = f + (has_mask ? (int64_t)(Mp[r + 1] - Mp[r]) : 0);
                b = lim.nb + 1;
                for (int q = 0; q < lim.nb; q++)
                    if (need <= lim.limit[q]) { b = q + 1; break; }
            }
            row_bin[r] = (int8_t)b;
            // entries of A in the heavy rows (sizes the flat product index)
            if (b == lim.nb + 1) atomicAdd(heavy_alen, (unsigned long long)(Ap[r + 1] - Ap[r]));
        }
        const unsigned counted = __ballot_sync(0xffffffffu, b > 0);
        if (b > 0) {
            const unsigned same = __match_any_sync(counted, b);
            if ((int)(__ffs(same) - 1) == lane) atomicAdd(&bin_count[b], __popc(same));
        }
    }
}

// scatter rows into per-bin lists (order within a bin does not matter); a
// bin's list starts after the rows of the bins before it
__global__ void k_fill_bins(const int8_t *__restrict__ row_bin, int64_t nrows,
                            int *__restrict__ bin_fill,
                            const int *__restrict__ bin_count, int nbins,
                            int32_t *__restrict__ bin_rows)
{
    __shared__ int bin_start[16];
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int q = 0; q < 16; q++) {
            bin_start[q] = acc;
            if (q < nbins) acc += bin_count[q];
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); r0 < nrows;
         r0 += stride) {
        const int64_t r = r0 + lane;
        const int b = r < nrows ? row_bin[r] : 0;
        const unsigned placed = __ballot_sync(0xffffffffu, b > 0);
        if (b > 0) {
            const unsigned same = __match_any_sync(placed, b);
            const int leader = __ffs(same) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&bin_fill[b], __popc(same));
            base = __shfl_sync(same, base, leader);
            bin_rows[bin_start[b] + base + __popc(same & ((1u << lane) - 1))] = (int32_t)r;
        }
    }
}

// ---------------------------------------------------------------------------
// group synchronisation (TPR threads working on one row)
// ---------------------------------------------------------------------------

template <int TPR> __device__ __forceinline__ void group_sync()
{
    if (TPR <= 32) {
        const unsigned lane = threadIdx.x & 31;
        const unsigned base = (lane / TPR) * TPR;
        const unsigned m = (TPR == 32) ? 0xffffffffu : (((1u << TPR) - 1u) << base);
        __syncwarp(m);
    } else {
        __syncthreads();
    }
}

// hash of a column index (multiplicative, like GB_HASHF's spreading of keys)
__device__ __forceinline__ uint32_t hslot(int32_t j, uint32_t mask)
{
    return ((uint32_t)j * 0x9E3779B1u) >> 7 & mask;
}

// ---------------------------------------------------------------------------
// phase 3a: shared-memory hash rows
// ---------------------------------------------------------------------------

// shared memory of one row group: keys[cap] int32, vals[cap] Z, state[cap] u8
template <typename Z> __host__ __device__ inline size_t group_bytes(int cap)
{
    return ((size_t)cap * (4 + sizeof(Z) + 1) + 15) / 16 * 16;
}

// A group of TPR threads (TPR = 4..32 inside a 128-thread block, or the whole
// 256-thread block when BLOCK) owns one row and one hash table of cap slots.
template <class SR, bool BLOCK>
__global__ void __launch_bounds__(BLOCK ? 256 : 128, BLOCK ? 4 : 8)
k_saxpy_hash(BinRows br, int tpr_log2, int cap,
             const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
             const void *__restrict__ Ax, bool a_iso,
             const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
             const void *__restrict__ Bx, bool b_iso,
             const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
             bool has_mask, bool mask_comp,
             const int64_t *__restrict__ slot_off,
             int32_t *__restrict__ Tj, typename SR::z_t *__restrict__ Tx,
             int32_t *__restrict__ row_cnt)
{
    using Z = typename SR::z_t;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_cnt[32];
    const int TPR = BLOCK ? (int)blockDim.x : (1 << tpr_log2);
    const int G = BLOCK ? 1 : ((int)blockDim.x >> tpr_log2);
    const int g = BLOCK ? 0 : ((int)threadIdx.x >> tpr_log2);
    const int t = BLOCK ? (int)threadIdx.x : ((int)threadIdx.x & (TPR - 1));
    const unsigned lane = threadIdx.x & 31;
    const unsigned gmask = (TPR >= 32) ? 0xffffffffu
                         : (((1u << TPR) - 1u) << ((lane >> tpr_log2) << tpr_log2));
    auto gsync = [&]() { if (BLOCK) __syncthreads(); else __syncwarp(gmask); };
    unsigned char *base = smem + (size_t)g * group_bytes<Z>(cap);
    int32_t *keys = (int32_t *)base;
    Z *vals = (Z *)(base + (size_t)cap * 4);
    uint8_t *state = (uint8_t *)(base + (size_t)cap * (4 + sizeof(Z)));
    const uint32_t hmask = (uint32_t)cap - 1;
    const int32_t *rows;
    const int nrows_bin = br.get(rows);

    for (int64_t rb = (int64_t)blockIdx.x * G + g; rb < nrows_bin;
         rb += (int64_t)gridDim.x * G) {
        const int32_t i = rows[rb];
        for (int s = t; s < cap; s += TPR) { keys[s] = -1; state[s] = S_EMPTY; }
        gsync();
        // scatter the mask row
        if (has_mask) {
            const uint8_t st = mask_comp ? S_FORBID : S_ALLOWED;
            for (int32_t pm = Mp[i] + t; pm < Mp[i + 1]; pm += TPR) {
                const int32_t j = Mj[pm];
                uint32_t h = hslot(j, hmask);
                while (true) {
                    int32_t old = atomicCAS(&keys[h], -1, j);
                    if (old == -1 || old == j) { state[h] = st; break; }
                    h = (h + 1) & hmask;
                }
            }
            gsync();
        }
        // k loop in ascending order; threads split B(k,:)
        const int32_t pa0 = Ap[i], pa1 = Ap[i + 1];
        for (int32_t pa = pa0; pa < pa1; pa++) {
            const int32_t k = Aj[pa];
            Z a = Z();
            if (SR::needs_a) a = ld_val<Z>(Ax, pa, a_iso);
            const int32_t pb0 = Bp[k], pb1 = Bp[k + 1];
            for (int32_t pb = pb0 + t; pb < pb1; pb += TPR) {
                const int32_t j = Bj[pb];
                uint32_t h = hslot(j, hmask);
                int32_t found = -1;
                if (has_mask && !mask_comp) {
                    // only columns of M(i,:) are allowed
                    while (true) {
                        int32_t kk = keys[h];
                        if (kk == j) { found = (int32_t)h; break; }
                        if (kk == -1) break;
                        h = (h + 1) & hmask;
                    }
                    if (found < 0) continue;
                } else {
                    while (true) {
                        int32_t old = atomicCAS(&keys[h], -1, j);
                        if (old == -1 || old == j) { found = (int32_t)h; break; }
                        h = (h + 1) & hmask;
                    }
                }
                const uint8_t st = state[found];
                if (st == S_FORBID) continue;
                Z b = Z();
                if (SR::needs_b) b = ld_val<Z>(Bx, pb, b_iso);
                const Z tv = SR::F::f(a, b, i, k, j);
                if (st == S_SET) {
                    vals[found] = SR::M::update(vals[found], tv);
                } else {
                    vals[found] = tv;
                    state[found] = S_SET;
                }
            }
            gsync();
        }
        // gather the set slots into the row's output slot, then sort them by
        // column in the (now free) table memory with a bitonic network
        const int64_t off = slot_off[i];
        if (t == 0) s_cnt[g] = 0;
        gsync();
        for (int s = t; s < cap; s += TPR) {
            if (state[s] == S_SET) {
                int q = atomicAdd(&s_cnt[g], 1);
                Tj[off + q] = keys[s];
                Tx[off + q] = vals[s];
            }
        }
        gsync();
        const int cnt = s_cnt[g];
        int n2 = 1;
        while (n2 < cnt) n2 <<= 1;
        for (int q = t; q < n2; q += TPR) {
            if (q < cnt) { keys[q] = Tj[off + q]; vals[q] = Tx[off + q]; }
            else keys[q] = INT32_MAX;
        }
        gsync();
        for (int size = 2; size <= n2; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int q = t; q < n2; q += TPR) {
                    const int partner = q ^ stride;
                    if (partner > q) {
                        const bool up = ((q & size) == 0);
                        const int32_t ka = keys[q], kb = keys[partner];
                        if ((ka > kb) == up) {
                            keys[q] = kb; keys[partner] = ka;
                            const Z va = vals[q]; vals[q] = vals[partner]; vals[partner] = va;
                        }
                    }
                }
                gsync();
            }
        }
        for (int q = t; q < cnt; q += TPR) { Tj[off + q] = keys[q]; Tx[off + q] = vals[q]; }
        if (t == 0) row_cnt[i] = cnt;
        gsync();
    }
}

// ---------------------------------------------------------------------------
// phase 3a': expand-sort-compress rows, one warp per row
// ---------------------------------------------------------------------------

// For rows with at most `cap` products.  The warp expands the row's products
// in order (A(i,:) in ascending k, each B(k,:) in order) into shared memory,
// keyed by (column j, position): the loads of all of the row's products are
// issued at once, with no per-k synchronisation and no hash probing.  A
// bitonic sort by that key groups equal columns with their terms still in
// ascending k, and each group is folded in that order with the monoid's
// UPDATE (first term written, later terms folded), as in the hash kernels,
// so every semiring, floating PLUS included, gives the same bits.
static constexpr int ESC_WARPS = 8;

// Bitonic sort of a warp's n <= 32*R keys in registers: element e = 32*r +
// lane sits in k[r]; compare-exchanges with strides of 32 or more stay inside
// a lane, shorter ones go through shuffles.  Keys past n sort as all ones.
// The keys are read from and written back to key[0..n).
template <int R, typename KT>
__device__ __forceinline__ void warp_sort_regs(KT *key, int n, int lane)
{
    KT k[R];
    #pragma unroll
    for (int r = 0; r < R; r++) {
        const int e = r * 32 + lane;
        k[r] = e < n ? key[e] : ~(KT)0;
    }
    #pragma unroll
    for (int size = 2; size <= 32 * R; size <<= 1) {
        #pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= 32) {
                const int rs = stride >> 5;
                #pragma unroll
                for (int r = 0; r < R; r++) {
                    if (r & rs) continue;
                    const int r2 = r | rs;
                    const bool up = ((r * 32 + lane) & size) == 0;
                    const KT a = k[r], b = k[r2];
                    const KT lo = a < b ? a : b, hi = a < b ? b : a;
                    k[r] = up ? lo : hi;
                    k[r2] = up ? hi : lo;
                }
            } else {
                #pragma unroll
                for (int r = 0; r < R; r++) {
                    const KT other = __shfl_xor_sync(0xffffffffu, k[r], stride);
                    const bool up = ((r * 32 + lane) & size) == 0;
                    const bool lower = (lane & stride) == 0;
                    k[r] = (lower == up) ? (k[r] < other ? k[r] : other)
                                         : (k[r] < other ? other : k[r]);
                }
            }
        }
    }
    #pragma unroll
    for (int r = 0; r < R; r++) {
        const int e = r * 32 + lane;
        if (e < n) key[e] = k[r];
    }
}

// One row of the expand-sort-compress bin by one warp: the row's products
// (at most cap) expand into key[] / val[] (the warp's shared-memory arrays),
// the keys are sorted and each run of equal columns is folded into one entry
// of Tj / Tx from position off() on (read only when the row is written).
// Returns the row's entry count; with LIMIT, -1 (and nothing written) when
// the row keeps more than cap products.
// KT: 32-bit keys when (column << posb) fits, else 64-bit; posb = log2(cap)
// bits hold the product's position, so only the keys move in the sort and
// the values stay where the expansion wrote them.
template <class SR, typename KT, bool LIMIT = false, class Off>
__device__ __forceinline__ int esc_row(int32_t i, int cap, int posb, KT *key,
                                       typename SR::z_t *val,
                                       const int32_t *__restrict__ Ap,
                                       const int32_t *__restrict__ Aj,
                                       const void *__restrict__ Ax, bool a_iso,
                                       const int32_t *__restrict__ Bp,
                                       const int32_t *__restrict__ Bj,
                                       const void *__restrict__ Bx, bool b_iso,
                                       const int32_t *__restrict__ Mp,
                                       const int32_t *__restrict__ Mj,
                                       bool has_mask, bool mask_comp, const Off &off_of,
                                       int32_t *__restrict__ Tj, typename SR::z_t *__restrict__ Tx)
{
    using Z = typename SR::z_t;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const KT posmask = ((KT)1 << posb) - 1;
    const int32_t pa0 = Ap[i], pa1 = Ap[i + 1];
    int32_t m0 = 0, m1 = 0;
    if (has_mask) { m0 = Mp[i]; m1 = Mp[i + 1]; }
    int n = 0;                                   // products kept so far
    for (int32_t c0 = pa0; c0 < pa1; c0 += 32) {
        // 32 entries of A(i,:) at a time: lane l holds k and nnz(B(k,:))
        const int32_t pa = c0 + lane;
        int32_t k = 0, b0 = 0, len = 0;
        Z a = Z();
        if (pa < pa1) {
            k = Aj[pa];
            b0 = Bp[k];
            len = Bp[k + 1] - b0;
            if (SR::needs_a) a = ld_val<Z>(Ax, pa, a_iso);
        }
        int incl = len;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for (int q0 = 0; q0 < total; q0 += 32) {
            // product q of this chunk belongs to the first lane src whose
            // inclusive count exceeds q
            const int q = q0 + lane;
            int src = 0;
            #pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int v = __shfl_sync(0xffffffffu, incl, src + step - 1);
                if (v <= q) src += step;
            }
            const int excl = __shfl_sync(0xffffffffu, incl - len, src);
            const int32_t kk = __shfl_sync(0xffffffffu, k, src);
            const int32_t bb = __shfl_sync(0xffffffffu, b0, src);
            const Z aa = shfl<Z>(a, src);
            bool keep = q < total;
            int32_t j = 0, pb = 0;
            if (keep) {
                pb = bb + (q - excl);
                j = Bj[pb];
                if (has_mask) {
                    const int32_t f = lower_bound(Mj, m0, m1, j);
                    const bool present = f < m1 && Mj[f] == j;
                    keep = mask_comp ? !present : present;
                }
            }
            const unsigned km = __ballot_sync(0xffffffffu, keep);
            if (LIMIT && n + __popc(km) > cap) return -1;
            if (keep) {
                const int pos = n + __popc(km & below);
                Z b = Z();
                if (SR::needs_b) b = ld_val<Z>(Bx, pb, b_iso);
                key[pos] = ((KT)(uint32_t)j << posb) | (KT)pos;
                val[pos] = SR::F::f(aa, b, i, kk, j);
            }
            n += __popc(km);
        }
    }
    __syncwarp();
    int n2 = 1;
    while (n2 < n) n2 <<= 1;
    if (n <= 32) {
        // one key per lane: bitonic network over the lanes in registers
        KT kk = lane < n ? key[lane] : ~(KT)0;
        #pragma unroll
        for (int size = 2; size <= 32; size <<= 1) {
            #pragma unroll
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                const KT other = __shfl_xor_sync(0xffffffffu, kk, stride);
                const bool up = (lane & size) == 0;
                const bool lower = (lane & stride) == 0;
                kk = (lower == up) ? (kk < other ? kk : other) : (kk < other ? other : kk);
            }
        }
        if (lane < n) key[lane] = kk;
        n2 = 0;                                  // the shared-memory network is skipped
    } else if (n <= 64) {
        warp_sort_regs<2>(key, n, lane);
        n2 = 0;
    } else if (n <= 128) {
        warp_sort_regs<4>(key, n, lane);
        n2 = 0;
    } else if (n <= 256) {
        warp_sort_regs<8>(key, n, lane);
        n2 = 0;
    }
    for (int q = n + lane; q < n2; q += 32) key[q] = ~(KT)0;
    __syncwarp();
    // bitonic sort of the keys; a lane owns every 32nd compare-exchange
    for (int size = 2; size <= n2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int q = lane; q < (n2 >> 1); q += 32) {
                // q-th pair of this pass: lower index a, partner a + stride
                const int a = ((q & ~(stride - 1)) << 1) | (q & (stride - 1));
                const int b = a + stride;
                const bool up = ((a & size) == 0);
                const KT ka = key[a], kb = key[b];
                if ((ka > kb) == up) { key[a] = kb; key[b] = ka; }
            }
            __syncwarp();
        }
    }
    // the first entry of each run of equal columns folds the run in
    // ascending k (its positions ascend) and writes one output entry
    const int64_t off = off_of();
    int out = 0;
    for (int c0 = 0; c0 < n; c0 += 32) {
        const int p = c0 + lane;
        bool head = false;
        KT kp = 0;
        if (p < n) {
            kp = key[p];
            head = (p == 0) || ((key[p - 1] >> posb) != (kp >> posb));
        }
        const unsigned hm = __ballot_sync(0xffffffffu, head);
        if (head) {
            const KT jcol = kp >> posb;
            Z z = val[kp & posmask];
            for (int r = p + 1; r < n; r++) {
                const KT kr = key[r];
                if ((kr >> posb) != jcol) break;
                z = SR::M::update(z, val[kr & posmask]);
            }
            const int64_t dst = off + out + __popc(hm & below);
            Tj[dst] = (int32_t)jcol;
            Tx[dst] = z;
        }
        out += __popc(hm);
    }
    return out;
}

template <class SR, typename KT>
__global__ void __launch_bounds__(ESC_WARPS * 32, 6)
k_saxpy_esc(BinRows br, int cap, int posb,
            const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
            const void *__restrict__ Ax, bool a_iso,
            const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
            const void *__restrict__ Bx, bool b_iso,
            const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
            bool has_mask, bool mask_comp,
            const int64_t *__restrict__ slot_off,
            int32_t *__restrict__ Tj, typename SR::z_t *__restrict__ Tx,
            int32_t *__restrict__ row_cnt)
{
    using Z = typename SR::z_t;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    KT *key = (KT *)(smem + (size_t)w * cap * (sizeof(KT) + sizeof(Z)));
    Z *val = (Z *)((unsigned char *)key + (size_t)cap * sizeof(KT));
    const int32_t *rows;
    const int nrows_bin = br.get(rows);

    for (int64_t rb = (int64_t)blockIdx.x * ESC_WARPS + w; rb < nrows_bin;
         rb += (int64_t)gridDim.x * ESC_WARPS) {
        const int32_t i = rows[rb];
        const int out = esc_row<SR, KT>(i, cap, posb, key, val, Ap, Aj, Ax, a_iso, Bp, Bj, Bx,
                                        b_iso,
                                        Mp, Mj, has_mask, mask_comp,
                                        [&]() { return slot_off[i]; }, Tj, Tx);
        if (lane == 0) row_cnt[i] = out;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// small products in one launch
// ---------------------------------------------------------------------------

// C = A*B (masked or not) in one launch, for products whose rows all fit the
// expand-sort-compress bin.  Blocks take row ranges of `chunk` rows from a
// ticket in the order they start, and row i's slots are [i*SMALL_CAP,
// (i+1)*SMALL_CAP):
//
//   1. each row expands, sorts and compresses into its slots (esc_row); a
//      row that keeps more than SMALL_CAP products sets tot[1] instead
//   2. the block's entry count is posted, and a decoupled look-back over the
//      blocks before it (they started earlier, so they are running or done)
//      gives its offset among C's entries; the last block's inclusive sum is
//      nnz(C)
//   3. C's row offsets for the block's rows, and its entries copied from the
//      slots, flat over the block's threads
//
// No block waits for one that has not started, so the launch needs no
// co-residency and runs beside other kernels.  tot[0] = nnz(C), tot[1] = 0
// (done), SMALL_TOO_LONG or SMALL_NO_ROOM (C's arrays too small; the blocks
// past the capacity write nothing), tot[2] is set when a look-back gave up
// waiting (the results are void), tot[3] is the ticket counter; part[G] are
// the blocks' look-back words.  The host zeroes tot[] and part[] first.
static constexpr int SMALL_CAP = 256;              // products per row, at most
static constexpr int SMALL_POSB = 8;               // log2(SMALL_CAP)
static constexpr int SMALL_CHUNK = 128;            // rows per block, at most
enum { SMALL_DONE = 0, SMALL_TOO_LONG = 1, SMALL_NO_ROOM = 3 };

// exclusive scan of v[0..n) (n <= SMALL_CHUNK) in place by warp 0; returns
// the total to every lane of warp 0
template <typename T>
__device__ __forceinline__ T small_warp_scan(T *v, int n, int lane)
{
    constexpr int PER = SMALL_CHUNK / 32;
    T x[PER];
    T sum = 0;
    #pragma unroll
    for (int q = 0; q < PER; q++) {
        const int e = lane * PER + q;
        x[q] = e < n ? v[e] : (T)0;
        sum += x[q];
    }
    T incl = sum;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const T total = __shfl_sync(0xffffffffu, incl, 31);
    T run = incl - sum;
    #pragma unroll
    for (int q = 0; q < PER; q++) {
        const int e = lane * PER + q;
        if (e < n) v[e] = run;
        run += x[q];
    }
    return total;
}

template <class SR>
__global__ void __launch_bounds__(ESC_WARPS * 32, 6)
k_saxpy_small(int32_t m, int32_t chunk,
              const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
              const void *__restrict__ Ax, bool a_iso,
              const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
              const void *__restrict__ Bx, bool b_iso,
              const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
              bool has_mask, bool mask_comp, long long *__restrict__ part,
              int32_t *__restrict__ Tj, typename SR::z_t *__restrict__ Tx,
              int32_t *__restrict__ Cp, int32_t *__restrict__ Cj,
              typename SR::z_t *__restrict__ Cx, int64_t ccap, long long *__restrict__ tot)
{
    using Z = typename SR::z_t;
    using KT = uint32_t;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_cnt[SMALL_CHUNK];           // the rows' entry counts
    __shared__ int s_coff[SMALL_CHUNK];          // their offsets among the block's entries
    __shared__ long long s_ex;
    __shared__ int s_btot, s_long, s_tile;
    unsigned long long *status = (unsigned long long *)part;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int G = (int)gridDim.x;
    // blocks take their row ranges from a ticket, in the order they start,
    // so a block's predecessors are running or done when it looks back
    if (tid == 0) {
        s_long = 0;
        s_tile = (int)atomicAdd((unsigned long long *)tot + 3, 1ull);
    }
    __syncthreads();
    const int b = s_tile;
    const int32_t r0 = b * chunk;
    const int32_t r1 = r0 + chunk < m ? r0 + chunk : m;
    const int nr = r1 > r0 ? r1 - r0 : 0;

    // 1. expand-sort-compress each row into its slots
    {
        KT *key = (KT *)(smem + (size_t)w * SMALL_CAP * (sizeof(KT) + sizeof(Z)));
        Z *val = (Z *)((unsigned char *)key + (size_t)SMALL_CAP * sizeof(KT));
        for (int r = w; r < nr; r += ESC_WARPS) {
            const int32_t i = r0 + r;
            const int out = esc_row<SR, KT, true>(i, SMALL_CAP, SMALL_POSB, key, val, Ap, Aj, Ax,
                                                  a_iso, Bp, Bj, Bx, b_iso, Mp, Mj, has_mask,
                                                  mask_comp,
                                                  [&]() { return (int64_t)i * SMALL_CAP; },
                                                  Tj, Tx);
            if (lane == 0) {
                s_cnt[r] = out < 0 ? 0 : out;
                if (out < 0) s_long = 1;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (w == 0) {
        for (int r = lane; r < SMALL_CHUNK; r += 32) s_coff[r] = r < nr ? s_cnt[r] : 0;
        __syncwarp();
        const int total = small_warp_scan<int>(s_coff, nr, lane);
        // the block's offset among C's entries: decoupled look-back over the
        // blocks before it (bounded waits; a wait past the bound sets tot[2])
        long long ex = 0;
        if (b == 0) {
            if (lane == 0) atomicExch(&status[0], LB_INC | (unsigned long long)total);
        } else {
            if (lane == 0) atomicExch(&status[b], LB_AGG | (unsigned long long)total);
            ex = lb_lookback(status, b, lane, (int *)(tot + 2));
            if (lane == 0)
                atomicExch(&status[b], LB_INC | ((unsigned long long)(ex + total) & LB_VAL));
        }
        if (lane == 0) {
            s_ex = ex;
            s_btot = total;
            if (s_long) atomicExch((unsigned long long *)tot + 1, (unsigned long long)SMALL_TOO_LONG);
            if (b == G - 1) {
                tot[0] = ex + total;
                if (ex + total > ccap)
                    atomicCAS((unsigned long long *)tot + 1, 0ull,
                              (unsigned long long)SMALL_NO_ROOM);
            }
        }
    }
    __syncthreads();

    // 2. C's row offsets and entries (a block whose entries would pass C's
    //    capacity writes nothing: the call then runs the general path)
    const long long cbefore = s_ex;
    const long long nnz_end = cbefore + s_btot;
    if (nnz_end > ccap) return;
    for (int r = tid; r < nr; r += blockDim.x) Cp[r0 + r] = (int32_t)(cbefore + s_coff[r]);
    if (r1 == m && nr > 0 && tid == 0) Cp[m] = (int32_t)nnz_end;
    // the block's entries flat over its threads, four per thread in flight
    const int btot = s_btot;
    for (int e0 = tid; e0 < btot; e0 += 4 * (int)blockDim.x) {
        int32_t jv[4];
        Z xv[4];
        #pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = e0 + u * (int)blockDim.x;
            if (e < btot) {
                int lo = 0, hi = nr - 1;        // the last row starting at or before e
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (s_coff[mid] <= e) lo = mid; else hi = mid - 1;
                }
                const long long src = (long long)(r0 + lo) * SMALL_CAP + (e - s_coff[lo]);
                jv[u] = Tj[src];
                xv[u] = Tx[src];
            }
        }
        #pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = e0 + u * (int)blockDim.x;
            if (e < btot) {
                Cj[cbefore + e] = jv[u];
                Cx[cbefore + e] = xv[u];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// phase 3b: heavy rows, dense accumulator in global memory
// ---------------------------------------------------------------------------

// sequential-k, one block per row; flag[j] holds the row's mark when set,
// mark+1 when forbidden (complemented mask) or allowed (plain mask)
template <class SR>
__global__ void __launch_bounds__(256)
k_saxpy_dense_seq(const int32_t *__restrict__ rows, int nrows_bin,
                  const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
                  const void *__restrict__ Ax, bool a_iso,
                  const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
                  const void *__restrict__ Bx, bool b_iso,
                  const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
                  bool has_mask, bool mask_comp, int64_t ncols,
                  int64_t *__restrict__ flag_all, typename SR::z_t *__restrict__ val_all,
                  const int64_t *__restrict__ slot_off,
                  int32_t *__restrict__ Tj, typename SR::z_t *__restrict__ Tx,
                  int32_t *__restrict__ row_cnt)
{
    using Z = typename SR::z_t;
    int64_t *flag = flag_all + (int64_t)blockIdx.x * ncols;
    Z *val = val_all + (int64_t)blockIdx.x * ncols;
    __shared__ int s_warp[8];
    __shared__ int s_base;
    for (int64_t rb = blockIdx.x; rb < nrows_bin; rb += gridDim.x) {
        const int32_t i = rows[rb];
        // marks: 3*rb+1 set, 3*rb+2 allowed, 3*rb+3 forbidden (unique per row)
        const int64_t mk_set = 3 * (rb + 1), mk_ok = mk_set + 1, mk_no = mk_set + 2;
        if (has_mask) {
            const int64_t st = mask_comp ? mk_no : mk_ok;
            for (int32_t pm = Mp[i] + threadIdx.x; pm < Mp[i + 1]; pm += blockDim.x)
                flag[Mj[pm]] = st;
            __syncthreads();
        }
        const int32_t pa0 = Ap[i], pa1 = Ap[i + 1];
        for (int32_t pa = pa0; pa < pa1; pa++) {
            const int32_t k = Aj[pa];
            Z a = Z();
            if (SR::needs_a) a = ld_val<Z>(Ax, pa, a_iso);
            for (int32_t pb = Bp[k] + threadIdx.x; pb < Bp[k + 1]; pb += blockDim.x) {
                const int32_t j = Bj[pb];
                const int64_t f = flag[j];
                if (has_mask) {
                    if (!mask_comp && f != mk_ok && f != mk_set) continue;
                    if (mask_comp && f == mk_no) continue;
                }
                Z b = Z();
                if (SR::needs_b) b = ld_val<Z>(Bx, pb, b_iso);
                const Z tv = SR::F::f(a, b, i, k, j);
                if (f == mk_set) val[j] = SR::M::update(val[j], tv);
                else { val[j] = tv; flag[j] = mk_set; }
            }
            __syncthreads();
        }
        // ordered compaction over all columns
        const int64_t off = slot_off[i];
        int total = 0;
        for (int64_t c0 = 0; c0 < ncols; c0 += blockDim.x) {
            const int64_t j = c0 + threadIdx.x;
            const bool on = (j < ncols) && (flag[j] == mk_set);
            const unsigned m = __ballot_sync(0xffffffffu, on);
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            if (lane == 0) s_warp[w] = __popc(m);
            __syncthreads();
            if (threadIdx.x == 0) {
                int acc = 0;
                for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
                    int c = s_warp[q]; s_warp[q] = acc; acc += c;
                }
                s_base = acc;
            }
            __syncthreads();
            if (on) {
                const int64_t q = off + total + s_warp[w] + __popc(m & ((1u << lane) - 1));
                Tj[q] = (int32_t)j;
                Tx[q] = val[j];
            }
            total += s_base;
            __syncthreads();
        }
        // clear the marks of this row's mask (values need no clearing)
        if (threadIdx.x == 0) row_cnt[i] = total;
        __syncthreads();
    }
}

// order-free heavy rows: all products of all heavy rows spread over the grid
template <typename Z> __device__ __forceinline__ void atomic_store_first(Z *p, Z v) { *p = v; }

template <int ADD, typename Z> struct AtomicUpd;
template <typename Z> struct AtomicUpd<OP_PLUS, Z> {
    __device__ static void run(Z *p, Z v) {
        atomicAdd((unsigned long long *)p, (unsigned long long)v);
    }
};
template <> struct AtomicUpd<OP_PLUS, int32_t> {
    __device__ static void run(int32_t *p, int32_t v) { atomicAdd(p, v); }
};
template <typename Z> struct AtomicUpd<OP_MAX, Z> {
    __device__ static void run(Z *p, Z v) { atomicMax((long long *)p, (long long)v); }
};
template <> struct AtomicUpd<OP_MAX, int32_t> {
    __device__ static void run(int32_t *p, int32_t v) { atomicMax(p, v); }
};
template <typename Z> struct AtomicUpd<OP_MIN, Z> {
    __device__ static void run(Z *p, Z v) { atomicMin((long long *)p, (long long)v); }
};
template <> struct AtomicUpd<OP_MIN, int32_t> {
    __device__ static void run(int32_t *p, int32_t v) { atomicMin(p, v); }
};
// floating min/max with the reference's NaN rule (skip NaN terms) via CAS
template <> struct AtomicUpd<OP_MIN, float> {
    __device__ static void run(float *p, float v) {
        if (isnan(v)) return;
        unsigned int *u = (unsigned int *)p;
        unsigned int old = *u;
        while (true) {
            float cur = __uint_as_float(old);
            if (cur <= v) return;
            unsigned int prev = atomicCAS(u, old, __float_as_uint(v));
            if (prev == old) return;
            old = prev;
        }
    }
};
template <> struct AtomicUpd<OP_MIN, double> {
    __device__ static void run(double *p, double v) {
        if (isnan(v)) return;
        unsigned long long *u = (unsigned long long *)p;
        unsigned long long old = *u;
        while (true) {
            double cur = __longlong_as_double((long long)old);
            if (cur <= v) return;
            unsigned long long prev = atomicCAS(u, old, (unsigned long long)__double_as_longlong(v));
            if (prev == old) return;
            old = prev;
        }
    }
};
template <> struct AtomicUpd<OP_MAX, float> {
    __device__ static void run(float *p, float v) {
        if (isnan(v)) return;
        unsigned int *u = (unsigned int *)p;
        unsigned int old = *u;
        while (true) {
            float cur = __uint_as_float(old);
            if (cur >= v) return;
            unsigned int prev = atomicCAS(u, old, __float_as_uint(v));
            if (prev == old) return;
            old = prev;
        }
    }
};
template <> struct AtomicUpd<OP_MAX, double> {
    __device__ static void run(double *p, double v) {
        if (isnan(v)) return;
        unsigned long long *u = (unsigned long long *)p;
        unsigned long long old = *u;
        while (true) {
            double cur = __longlong_as_double((long long)old);
            if (cur >= v) return;
            unsigned long long prev = atomicCAS(u, old, (unsigned long long)__double_as_longlong(v));
            if (prev == old) return;
            old = prev;
        }
    }
};
template <typename Z> struct AtomicUpd<OP_LOR, Z> {
    __device__ static void run(Z *p, Z v) { if (v) *p = (Z)1; }
};
template <typename Z> struct AtomicUpd<OP_LAND, Z> {
    __device__ static void run(Z *p, Z v) { if (!v) *p = (Z)0; }
};
template <typename Z> struct AtomicUpd<OP_TIMES, Z> {
    __device__ static void run(Z *p, Z v) {
        unsigned long long *u = (unsigned long long *)p;
        unsigned long long old = *u, prev;
        do {
            prev = old;
            Z nv = rn_mul<Z>((Z)prev, v);
            old = atomicCAS(u, prev, (unsigned long long)nv);
        } while (old != prev);
    }
};
template <> struct AtomicUpd<OP_TIMES, int32_t> {
    __device__ static void run(int32_t *p, int32_t v) {
        int old = *p, prev;
        do { prev = old; old = atomicCAS(p, prev, rn_mul<int32_t>(prev, v)); } while (old != prev);
    }
};
// ANY with k-valued multiplier: last k wins = max k; constant multipliers:
// every term is equal, a plain store is exact
template <typename Z> struct AtomicUpd<OP_ANY, Z> {
    __device__ static void run(Z *p, Z v) { atomicMax((long long *)p, (long long)v); }
};
template <> struct AtomicUpd<OP_ANY, int32_t> {
    __device__ static void run(int32_t *p, int32_t v) { atomicMax(p, v); }
};
template <> struct AtomicUpd<OP_ANY, bool> {
    __device__ static void run(bool *p, bool v) { *p = v; }
};

// initial value of a dense slot for order-free accumulation
template <class SR> __device__ __forceinline__ typename SR::z_t dense_init()
{
    using Z = typename SR::z_t;
    if (SR::M::any) {
        // max-k accumulation starts below every k
        return std::is_same<Z, bool>::value ? (Z)0 : (Z)(-1);
    }
    return SR::M::identity();
}

// The dense row of a max-k ANY (any_secondi, any_firstj) on integer values:
// each column is one 64-bit word, state << 32 | k (state 0 empty, 1 allowed
// by a mask, 2 forbidden by a complemented mask, 3 holding k; every k is a
// row or column index, below 2^31).  A product reads one word instead of a
// flag and a value, and atomicMax on the word keeps the largest k, because
// every word holding a value has the same state bits and is above every
// word that does not.  The byte flags then only mark, for the compaction,
// the columns that received a value.
template <class SR> struct PackedDense {
    using Z = typename SR::z_t;
    static constexpr bool on = SR::any_max_k && std::is_integral<Z>::value && sizeof(Z) >= 4;
};
template <class SR>
using dense_val_t = typename std::conditional<PackedDense<SR>::on, unsigned long long,
                                              typename SR::z_t>::type;
static constexpr unsigned long long PK_SET = 3ull << 32;

// the first p in [lo, hi) with a[p] >= key (hi if none), a nondecreasing,
// found by the 32 lanes of a warp together (32 probes a step)
__device__ __forceinline__ int32_t warp_lower_bound(const int32_t *__restrict__ a, int32_t lo,
                                                    int32_t hi, int32_t key, int lane)
{
    while (lo < hi) {
        const int32_t step = (hi - lo + 31) / 32;
        const int32_t c = lo + lane * step;
        const bool less = c < hi && a[c] < key;
        const int k = __popc(__ballot_sync(0xffffffffu, less));
        if (k == 0) break;                        // a[lo] >= key
        const int32_t nhi = lo + k * step;
        lo = lo + (k - 1) * step + 1;
        hi = nhi < hi ? nhi : hi;
    }
    return lo;
}

// The dense rows of a chunk prepared in one pass: block x of grid row y
// owns a contiguous range of columns of heavy row y; it clears their flags,
// sets their values to the monoid's identity, then marks the row's mask
// entries that fall in its range (found by two warp-cooperative searches in
// the sorted mask row): 1 = allowed (plain mask), 2 = forbidden (complement).
// With one heavy row its flat index offsets {0, nnz(A(i,:))} are written too.
template <class SR>
__global__ void __launch_bounds__(256)
k_dense_prep(const int32_t *__restrict__ rows, int nrows_bin, int64_t ncols,
             uint8_t *__restrict__ flag_all, dense_val_t<SR> *__restrict__ val_all,
             const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
             bool has_mask, bool mask_comp, const int32_t *__restrict__ Ap,
             int64_t *__restrict__ hoff)
{
    __shared__ int32_t s_lo, s_hi;
    const int64_t per = ((ncols + gridDim.x - 1) / gridDim.x + 255) & ~(int64_t)255;
    const int64_t c0 = (int64_t)blockIdx.x * per;
    const int64_t c1 = c0 + per < ncols ? c0 + per : ncols;
    if (nrows_bin == 1 && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        const int32_t i = rows[0];
        hoff[0] = 0;
        hoff[1] = Ap[i + 1] - Ap[i];
    }
    constexpr bool packed = PackedDense<SR>::on;
    for (int64_t rb = blockIdx.y; rb < nrows_bin; rb += gridDim.y) {
        uint8_t *flag = flag_all + rb * ncols;
        dense_val_t<SR> *val = val_all + rb * ncols;
        for (int64_t j = c0 + threadIdx.x; j < c1; j += blockDim.x) {
            flag[j] = 0;
            if constexpr (packed) val[j] = 0;
            else val[j] = dense_init<SR>();
        }
        if (has_mask && c0 < c1) {
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            if (w < 2) {
                const int32_t i = rows[rb];
                const int32_t key = (int32_t)(w == 0 ? c0 : (c1 < INT32_MAX ? c1 : INT32_MAX));
                const int32_t r = warp_lower_bound(Mj, Mp[i], Mp[i + 1], key, lane);
                if (lane == 0) { if (w == 0) s_lo = r; else s_hi = r; }
            }
            __syncthreads();
            const uint8_t st = mask_comp ? 2 : 1;
            for (int32_t pm = s_lo + threadIdx.x; pm < s_hi; pm += blockDim.x) {
                if constexpr (packed) val[Mj[pm]] = (unsigned long long)st << 32;
                else flag[Mj[pm]] = st;
            }
        }
        __syncthreads();
    }
}
__global__ void k_heavy_alen(const int32_t *__restrict__ rows, int nr,
                             const int32_t *__restrict__ Ap, int64_t *__restrict__ hlen)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x) {
        const int32_t i = rows[t];
        hlen[t] = Ap[i + 1] - Ap[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) hlen[nr] = 0;
}

__device__ __forceinline__ int64_t upper_bound64(const int64_t *a, int64_t lo, int64_t hi,
                                                 int64_t key)
{
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] <= key) lo = mid + 1; else hi = mid;
    }
    return lo;
}


// heavy rows' offsets into the flat entry index (up to 1024 rows, one block)
__global__ void __launch_bounds__(1024)
k_heavy_offsets(const int32_t *__restrict__ rows, int nr, const int32_t *__restrict__ Ap,
                int64_t *__restrict__ hoff)
{
    __shared__ int64_t s_w[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    int64_t x = 0;
    if (t < nr) { const int32_t i = rows[t]; x = Ap[i + 1] - Ap[i]; }
    const int64_t own = x;
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t v = s_w[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        s_w[lane] = v;
    }
    __syncthreads();
    const int64_t ex = (w > 0 ? s_w[w - 1] : 0) + x - own;
    if (t < nr) hoff[t] = ex;
    if (t == nr - 1) hoff[nr] = ex + own;
}

// value e of the flat product index: nnz(B(k,:)) for the heavy rows' entry e
// (A(i,k), rows in order), 0 past the chunk's entries
struct LbLoadBlen {
    const int32_t *rows;
    int nr;
    const int64_t *hoff;
    const int32_t *Ap, *Aj, *Bp;
    __device__ int64_t operator()(int64_t e) const
    {
        if (e >= hoff[nr]) return 0;
        const int rb = nr == 1 ? 0 : (int)(upper_bound64(hoff, 0, nr + 1, e) - 1);
        const int32_t k = Aj[Ap[rows[rb]] + (e - hoff[rb])];
        return Bp[k + 1] - Bp[k];
    }
};

// Every product of the chunk's heavy rows, flat over the product index: a
// warp takes 32 consecutive products (one binary search for the first one's
// A entry; lanes walk forward), so a hub column of B is spread over many
// warps instead of one.
template <class SR>
__global__ void __launch_bounds__(256)
k_dense_atomic_flat(const int32_t *__restrict__ rows, int nr,
                    const int64_t *__restrict__ hoff, const int64_t *__restrict__ wprefix,
                    const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
                    const void *__restrict__ Ax, bool a_iso,
                    const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
                    const void *__restrict__ Bx, bool b_iso,
                    bool has_mask, bool mask_comp, int64_t ncols,
                    uint8_t *__restrict__ flag_all, dense_val_t<SR> *__restrict__ val_all)
{
    using Z = typename SR::z_t;
    constexpr bool idem = SR::M::any || SR::add_op == OP_MIN || SR::add_op == OP_MAX ||
                          SR::add_op == OP_LOR || SR::add_op == OP_LAND;
    const int lane = threadIdx.x & 31;
    const int64_t ne = hoff[nr];
    const int64_t total = wprefix[ne];
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    // each warp takes spans of consecutive products (about four per warp,
    // 32 to 1024 long): the A entry of a span's first product is searched
    // once, and every later step of 32 starts from the previous step's last
    int64_t span = (total + 4 * nw - 1) / (4 * nw);
    span = (span + 31) & ~(int64_t)31;
    span = span < 32 ? 32 : (span > 1024 ? 1024 : span);
    const int64_t nspan = (total + span - 1) / span;
    for (int64_t si = wid; si < nspan; si += nw) {
        // spans are taken from the last one down: the first blocks to run
        // carry the largest k, so an idempotent monoid (a max-k ANY) skips
        // most later atomics; the result does not depend on the order
        const int64_t s0 = (nspan - 1 - si) * span;
        const int64_t s1 = s0 + span < total ? s0 + span : total;
        int64_t e0 = warp_last_le<int64_t, int64_t>(wprefix, ne, s0, lane);
        for (int64_t base = s0; base < s1; base += 32) {
            const int64_t t = base + lane;
            int64_t e = e0;
            if (t < s1) while (wprefix[e + 1] <= t) e++;
            e0 = __shfl_sync(0xffffffffu, e, 31);      // the next step's first entry
            if (t >= s1) continue;
            const int rb = nr == 1 ? 0 : (int)(upper_bound64(hoff, 0, nr + 1, e) - 1);
            const int32_t i = rows[rb];
            const int32_t pa = Ap[i] + (int32_t)(e - hoff[rb]);
            const int32_t k = Aj[pa];
            const int32_t pb = Bp[k] + (int32_t)(t - wprefix[e]);
            const int32_t j = Bj[pb];
            if constexpr (PackedDense<SR>::on) {
                // one word: state and k
                unsigned long long *word = val_all + (int64_t)rb * ncols + j;
                const unsigned long long wv = *word;
                const unsigned st = (unsigned)(wv >> 32);
                if (has_mask) {
                    if (!mask_comp && st == 0) continue;
                    if (mask_comp && st == 2) continue;
                }
                Z a = Z(), b = Z();
                const Z tv = SR::F::f(a, b, i, k, j);
                const unsigned long long nv = PK_SET | (unsigned long long)(uint32_t)tv;
                if (wv >= nv) continue;
                atomicMax(word, nv);
                // the compaction's mark (the word holds the value)
                if (st != 3) flag_all[(int64_t)rb * ncols + j] = 3;
                continue;
            }
            uint8_t *flag = flag_all + (int64_t)rb * ncols;
            Z *val = (Z *)val_all + (int64_t)rb * ncols;
            const uint8_t f = flag[j];
            if (has_mask) {
                if (!mask_comp && f == 0) continue;
                if (mask_comp && f == 2) continue;
            }
            Z a = Z(), b = Z();
            if (SR::needs_a) a = ld_val<Z>(Ax, pa, a_iso);
            if (SR::needs_b) b = ld_val<Z>(Bx, pb, b_iso);
            const Z tv = SR::F::f(a, b, i, k, j);
            if constexpr (idem) {
                if (f == 3) {
                    if (SR::any_const) continue;
                    const Z cur = val[j];
                    if (SR::M::any ? !(tv > cur) : (SR::M::update(cur, tv) == cur)) continue;
                }
            }
            AtomicUpd<SR::add_op, Z>::run(&val[j], tv);
            if (f != 3) flag[j] = 3;
        }
    }
}

// grid-wide ordered compaction of dense heavy rows, so a single long row
// uses the whole GPU
static constexpr int DG_THREADS = 256, DG_ITEMS = 16, DG_CHUNK = DG_THREADS * DG_ITEMS;
template <class SR> constexpr int dense_tile() { return DG_CHUNK; }

// The same compaction in one launch: tiles of dense_tile() columns of one heavy
// row (tile = row * cblocks + chunk, from a ticket), 16 columns per thread;
// a tile counts its entries, takes its offset in the row from its
// predecessors by decoupled look-back (a row's first tile starts at 0), and
// writes them in column order: the tile's columns are staged in shared
// memory in order, then written out (and their values gathered) by
// consecutive threads (a packed row's values from its words).  ws: ntiles +
// 2 zero words, left zero.
template <class SR>
__global__ void __launch_bounds__(DG_THREADS)
k_dense_compact(const int32_t *__restrict__ rows, int cblocks, int64_t ncols,
                const uint8_t *__restrict__ flag_all,
                const dense_val_t<SR> *__restrict__ val_all,
                const int64_t *__restrict__ slot_off, int32_t *__restrict__ Tj,
                typename SR::z_t *__restrict__ Tx, int32_t *__restrict__ row_cnt,
                int64_t ntiles, unsigned long long *__restrict__ ws, int *__restrict__ err)
{
    __shared__ int s_tile, s_last, s_agg;
    __shared__ long long s_ex;
    __shared__ int s_w[DG_THREADS / 32];
    constexpr bool packed = PackedDense<SR>::on;
    __shared__ int32_t s_j[DG_CHUNK];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    unsigned long long *status = ws + 2;
    if (tid == 0) s_tile = (int)atomicAdd(&ws[0], 1ull);
    __syncthreads();
    const int64_t tile = s_tile;
    const int64_t rb = tile / cblocks, cb = tile % cblocks;
    const int32_t i = rows[rb];
    const int64_t c0 = cb * DG_CHUNK + (int64_t)tid * DG_ITEMS;
    unsigned bits = 0;
    const uint8_t *flag = flag_all + rb * ncols;
    if (c0 + DG_ITEMS <= ncols && (((uintptr_t)(flag + c0)) & 15) == 0) {
        const uint4 v = *reinterpret_cast<const uint4 *>(flag + c0);
        const uint32_t word[4] = {v.x, v.y, v.z, v.w};
        #pragma unroll
        for (int q = 0; q < 16; q++)
            if (((word[q >> 2] >> ((q & 3) * 8)) & 0xff) == 3) bits |= 1u << q;
    } else {
        for (int q = 0; q < DG_ITEMS; q++)
            if (c0 + q < ncols && flag[c0 + q] == 3) bits |= 1u << q;
    }
    const int cnt = __popc(bits);
    int x = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
        int v = lane < DG_THREADS / 32 ? s_w[lane] : 0;
        const int ownv = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        const long long agg = __shfl_sync(0xffffffffu, v, 31);
        if (lane < DG_THREADS / 32) s_w[lane] = v - ownv;
        long long ex = 0;
        if (cb == 0) {
            if (lane == 0) atomicExch(&status[tile], LB_INC | ((unsigned long long)agg & LB_VAL));
        } else {
            if (lane == 0) atomicExch(&status[tile], LB_AGG | ((unsigned long long)agg & LB_VAL));
            ex = lb_lookback(status, tile, lane, err);
            if (lane == 0)
                atomicExch(&status[tile], LB_INC | ((unsigned long long)(ex + agg) & LB_VAL));
        }
        if (lane == 0) {
            s_ex = ex;
            s_agg = (int)agg;
            if (cb == cblocks - 1) row_cnt[i] = (int32_t)(ex + agg);
        }
    }
    __syncthreads();
    int loc = s_w[w] + (x - cnt);
    while (bits) {
        const int q = __ffs(bits) - 1;
        bits &= bits - 1;
        s_j[loc++] = (int32_t)(c0 + q);
    }
    __syncthreads();
    const int64_t base = slot_off[i] + s_ex;
    const dense_val_t<SR> *val = val_all + rb * ncols;
    for (int k = tid; k < s_agg; k += DG_THREADS) {
        const int32_t j = s_j[k];
        Tj[base + k] = j;
        if constexpr (packed)
            Tx[base + k] = (typename SR::z_t)(uint32_t)(val[j] & 0xffffffffull);
        else
            Tx[base + k] = val[j];
    }
    // the last tile to finish clears the workspace
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(&ws[1], 1ull) == (unsigned long long)(ntiles - 1);
    }
    __syncthreads();
    if (s_last) {
        for (int64_t t = tid; t < ntiles; t += DG_THREADS) status[t] = 0;
        if (tid == 0) { ws[0] = 0; ws[1] = 0; }
    }
}

// ---------------------------------------------------------------------------
// phase 4: pack each row's (sorted) slot into CSR
// ---------------------------------------------------------------------------

// Flat over C's entries: entry e of C lies in the row r with
// Cp64[r] <= e < Cp64[r+1] and comes from position e - Cp64[r] of that row's
// slot.  One binary search per warp finds the row of its first entry; lanes
// walk forward from there.  A long row (vxm's single row) is copied by the
// whole grid.
template <typename Z>
__global__ void __launch_bounds__(256)
k_pack(int64_t nrows, int span, const int64_t *__restrict__ slot_off,
       const int32_t *__restrict__ Tj, const Z *__restrict__ Tx,
       const int64_t *__restrict__ Cp64, int32_t *__restrict__ Cj, Z *__restrict__ Cx,
       int64_t cap)
{
    const int lane = threadIdx.x & 31;
    const int64_t nnz = Cp64[nrows];
    if (nnz > cap) return;                 // C's arrays are too small: packed later
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * span;
         s0 < nnz; s0 += nw * span) {
        int64_t r0 = warp_last_le<int64_t, int64_t>(Cp64, nrows, s0, lane);
        const int64_t s1 = s0 + span < nnz ? s0 + span : nnz;
        for (int64_t base = s0; base < s1; base += 32) {
            const int64_t e = base + lane;
            int64_t r = r0;
            if (e < s1) {
                while (Cp64[r + 1] <= e) r++;
                const int64_t src = slot_off[r] + (e - Cp64[r]);
                Cj[e] = Tj[src];
                Cx[e] = Tx[src];
            }
            r0 = __shfl_sync(0xffffffffu, r, 31);
        }
    }
}



// ---------------------------------------------------------------------------
// configuration, plan, execution
// ---------------------------------------------------------------------------

SaxpyConfig saxpy_default_config()
{
    SaxpyConfig c;
    c.nb = 3;
    c.bin[0] = {256, 1, 256};          // expand-sort-compress, warp per row
    c.bin[1] = {1024, 32, 2048};       // shared-memory hash, warp per row
    c.bin[2] = {4096, 256, 8192};      // shared-memory hash, block per row
    c.blocks_per_sm = 16;
    return c;
}

// raise a kernel's dynamic shared-memory limit to what the device allows
// beside the kernel's static shared memory
static void allow_dynamic_smem(const void *fn)
{
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) { cudaGetLastError(); return; }
    const int dyn = (int)runtime().smem_optin - (int)fa.sharedSizeBytes;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess)
        cudaGetLastError();
}

static size_t bin_smem(const BinSpec &b, size_t zsize)
{
    if (b.tpr == 1) return (size_t)ESC_WARPS * b.cap * (8 + zsize);
    const size_t gb = ((size_t)b.cap * (4 + zsize + 1) + 15) / 16 * 16;
    return b.tpr >= 256 ? gb : gb * (128 / b.tpr);
}

bool saxpy_config_valid(const SaxpyConfig &cfg, size_t zsize)
{
    if (cfg.nb < 0 || cfg.nb > MAX_SMEM_BINS) return false;
    int64_t prev = 0;
    for (int q = 0; q < cfg.nb; q++) {
        const BinSpec &b = cfg.bin[q];
        if (b.limit <= prev || (b.cap & (b.cap - 1)) != 0) return false;
        if (b.tpr == 1) {
            // expand-sort-compress: one slot per product of the row
            if ((int64_t)b.cap < b.limit || b.cap < 8 || b.cap > (1 << 16)) return false;
        } else {
            if ((int64_t)b.cap < 2 * b.limit) return false;
            if (!(b.tpr == 4 || b.tpr == 8 || b.tpr == 16 || b.tpr == 32 || b.tpr == 256))
                return false;
        }
        if (bin_smem(b, zsize) + 256 > runtime().smem_optin) return false;
        prev = b.limit;
    }
    return cfg.blocks_per_sm >= 1 && cfg.blocks_per_sm <= 64;
}

// bins[] (ints) of a plan: 0..15 rows per bin, 32..47 fill cursors, 48-49
// the A entries of heavy rows (u64), 50-51 the slot total (i64), 52-53 the
// output count (i64), 54 the row-offset scan's error word, 55 the heavy-row
// scans' error word, 56 the slot-offset scan's error word.  The first
// BINS_READ ints come back to the host.
static constexpr int BINS_WORDS = 64;
static constexpr int BINS_READ = 57;
static constexpr int BIN_HEAVY_ALEN = 48, BIN_TOTAL_CAP = 50, BIN_NNZ = 52,
                     BIN_ROW_ERR = 54, BIN_HEAVY_ERR = 55, BIN_SLOT_ERR = 56;

struct SaxpyPlan {
    SemiringCode sr;
    SaxpyConfig cfg;
    size_t zsize = 8;
    bool order_free = false;
    int64_t m = 0, ncols = 0;
    bool has_mask = false, mask_comp = false;
    int64_t total_cap = 0;      // slots the rows need
    int64_t slot_avail = 0;     // slots Tj / Tx hold
    int64_t nnz = 0;            // output entries, once read back
    int h_bins[MAX_SMEM_BINS + 2] = {0};
    int h_start[MAX_SMEM_BINS + 2] = {0};
    // device buffers
    int64_t *flops = nullptr, *slot_off = nullptr, *Cp64 = nullptr;
    // single-pass scan workspaces of the slot and row offsets (zeroed with
    // the bin counters, left zero by every scan)
    unsigned long long *lb_slot = nullptr, *lb_row = nullptr;
    int8_t *row_bin = nullptr;
    int32_t *bin_rows = nullptr, *row_cnt = nullptr, *Tj = nullptr;
    void *Tx = nullptr;
    int *bins = nullptr;
    int64_t heavy_chunk = 0;
    int64_t *flag = nullptr;                       // order-dependent rows: row marks
    uint8_t *flag8 = nullptr;                      // order-free rows: 0/1/2/3 states
    void *val = nullptr;
    int64_t heavy_alen = 0;                         // A entries in the heavy rows
    int64_t *hlen = nullptr, *hoff = nullptr;       // flat product index (per chunk)
    int64_t *wprefix = nullptr, *hw_ws = nullptr;
    // look-back workspaces of the product-index scan and the compaction
    unsigned long long *lb_w = nullptr, *lb_c = nullptr;
    // the allocations the buffers above are carved from: symbolic arrays,
    // slots (Tj, Tx; null when the slots are the stream's scratch buffer),
    // heavy-row accumulators
    void *block = nullptr, *tblock = nullptr, *hblock = nullptr;
};

void saxpy_plan_free(SaxpyPlan *P, cudaStream_t s)
{
    if (!P) return;
    dfree(P->block, s); dfree(P->tblock, s); dfree(P->hblock, s);
    delete P;
}

int64_t saxpy_plan_capacity(const SaxpyPlan *P) { return P->total_cap; }

// entries per warp work unit of the flat kernels: one 32-entry step for
// small inputs (many warps, no walking), up to 1024 for large ones (one
// binary search per span instead of per step)
static inline int flat_span(int64_t n)
{
    const int64_t target = (int64_t)runtime().num_sms * 64;     // warps to fill
    int64_t sp = (n / target + 31) / 32 * 32;
    return (int)(sp < 32 ? 32 : sp > 1024 ? 1024 : sp);
}

static inline int nblocks(int64_t n, int threads, int per_sm = 8)
{
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)runtime().num_sms * per_sm;
    if (b > cap) b = cap;
    return b < 1 ? 1 : (int)b;
}

// Symbolic phase, with no host round trip: flop counts, bins and slot
// capacities, the slot offsets (their total lands in bins[50]) and the
// bins' row lists.
template <class SR>
static int plan_symbolic(SaxpyPlan *P, const DevCSR *M, bool mask_comp, const DevCSR &A,
                         const DevCSR &B, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t m = A.nrows, ncols = B.ncols;
    P->zsize = sizeof(Z);
    P->order_free = SR::order_free;
    P->m = m; P->ncols = ncols;
    P->has_mask = M != nullptr; P->mask_comp = mask_comp;
    // the symbolic arrays in one allocation: the bin counters, the scans'
    // workspaces, the flop counts, the slot offsets and the row counts first
    // and adjacent, so that one memset clears them all
    Carve cv(s);
    auto layout = [&]() {
        P->bins = cv.take<int>(BINS_WORDS);
        P->lb_slot = cv.take<unsigned long long>(scan_lb_ws_elems(m + 1));
        P->lb_row = cv.take<unsigned long long>(scan_lb_ws_elems(m + 1));
        P->flops = cv.take<int64_t>(m + 1);
        P->slot_off = cv.take<int64_t>(m + 1);
        P->row_cnt = cv.take<int32_t>(m + 1);
        P->Cp64 = cv.take<int64_t>(m + 2);
        P->row_bin = cv.take<int8_t>(m + 1);
        P->bin_rows = cv.take<int32_t>(m + 1);
    };
    layout();
    if (!cv.alloc()) return OUT_OF_MEMORY;
    layout();
    P->block = cv.base;
    const bool mask_bounds = (M != nullptr) && !mask_comp;
    cudaMemsetAsync(P->bins, 0, (size_t)((char *)(P->row_cnt + m + 1) - (char *)P->bins), s);
    if (m > 0 && A.nnz > 0)
        k_flops_flat<<<nblocks(A.nnz, 256, 16), 256, 0, s>>>(A.p, A.j, B.p, m, A.nnz,
            flat_span(A.nnz),
            (unsigned long long *)P->flops);
    BinLimits lim;
    lim.nb = P->cfg.nb;
    for (int q = 0; q < P->cfg.nb; q++) lim.limit[q] = P->cfg.bin[q].limit;
    if (m > 0)
        k_bin_rows<<<nblocks(m, 256), 256, 0, s>>>(P->flops, M ? M->p : nullptr,
            M != nullptr, mask_bounds, ncols, m, lim, P->bins, P->row_bin, P->slot_off,
            A.p, (unsigned long long *)(P->bins + BIN_HEAVY_ALEN));
    scan_exclusive_lb(P->slot_off, P->slot_off, m + 1, P->lb_slot, s,
                      (int64_t *)(P->bins + BIN_TOTAL_CAP), nullptr, P->bins + BIN_SLOT_ERR);
    // the row lists: a bin's list starts after those of the bins before it
    // (the fill kernel adds up the counts itself)
    if (m > 0)
        k_fill_bins<<<nblocks(m, 256), 256, 0, s>>>(P->row_bin, m, P->bins + 32, P->bins,
                                                   P->cfg.nb + 2, P->bin_rows);
    return cuda_to_info(cudaGetLastError());
}

// the bin counts, heavy-row size, slot total and output count, to the host
static int plan_read(SaxpyPlan *P, cudaStream_t s)
{
    int hb[BINS_READ];
    cudaError_t e = readback(hb, P->bins, sizeof(hb), s);
    if (e != cudaSuccess) return cuda_to_info(e);
    if (hb[BIN_SLOT_ERR] || hb[BIN_ROW_ERR] || hb[BIN_HEAVY_ERR]) return PANIC;
    const int nb = P->cfg.nb;
    for (int b = 0; b < nb + 2; b++) P->h_bins[b] = hb[b];
    memcpy(&P->heavy_alen, hb + BIN_HEAVY_ALEN, 8);
    memcpy(&P->total_cap, hb + BIN_TOTAL_CAP, 8);
    memcpy(&P->nnz, hb + BIN_NNZ, 8);
    P->h_start[0] = 0;
    for (int b = 1; b < nb + 2; b++) P->h_start[b] = P->h_start[b - 1] + P->h_bins[b - 1];
    return SUCCESS;
}

// Tj / Tx in a block of `bytes` at `base`: as many slots as fit
static void plan_place_slots(SaxpyPlan *P, void *base, size_t bytes)
{
    const int64_t per = 4 + (int64_t)P->zsize;
    int64_t slots = ((int64_t)bytes - 512) / per;
    if (slots < 1) slots = 1;
    P->Tj = (int32_t *)base;
    P->Tx = (char *)base + (((size_t)slots * 4 + 255) & ~(size_t)255);
    P->slot_avail = slots - 1;
}

static size_t slot_bytes(const SaxpyPlan *P, int64_t slots)
{
    return (size_t)(slots + 1) * (4 + P->zsize) + 512;
}

// the heavy rows' accumulators (sizes from plan_read)
template <class SR>
static int plan_alloc_heavy(SaxpyPlan *P, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int nb = P->cfg.nb;
    const int64_t ncols = P->ncols;
    const int nheavy = P->h_bins[nb + 1];
    if (nheavy == 0 || P->hblock) return SUCCESS;
    Carve hv(s);
    std::function<void()> hlayout;
    if (SR::order_free) {
        int64_t chunk = nheavy;
        const int64_t per_row = ncols * (1 + (int64_t)sizeof(Z));
        const int64_t budget = (int64_t)4 << 30;
        if (chunk * per_row > budget) chunk = budget / per_row > 0 ? budget / per_row : 1;
        P->heavy_chunk = chunk;
        const int64_t cblocks = (ncols + dense_tile<SR>() - 1) / dense_tile<SR>();
        const int64_t ntiles = chunk * cblocks;
        hlayout = [&, chunk, ntiles]() {
            P->flag8 = hv.take<uint8_t>(chunk * ncols + 1);
            P->val = hv.take<dense_val_t<SR>>(chunk * ncols + 1);
            P->hlen = hv.take<int64_t>(chunk + 1);
            P->hoff = hv.take<int64_t>(chunk + 1);
            P->wprefix = hv.take<int64_t>(P->heavy_alen + 1);
            P->hw_ws = hv.take<int64_t>(scan_ws_elems(chunk + 1));
            P->lb_w = hv.take<unsigned long long>(lb_ws_elems(P->heavy_alen + 1));
            P->lb_c = hv.take<unsigned long long>(ntiles + 2);   // a word per tile
        };
    } else {
        const int nbk = nheavy < runtime().num_sms * 2 ? nheavy : runtime().num_sms * 2;
        P->heavy_chunk = nbk;
        hlayout = [&, nbk]() {
            P->flag = hv.take<int64_t>((int64_t)nbk * ncols + 1);
            P->val = hv.take<Z>((int64_t)nbk * ncols + 1);
        };
    }
    hlayout();
    if (!hv.alloc()) return OUT_OF_MEMORY;
    hlayout();
    P->hblock = hv.base;
    if (P->lb_w) {
        // the two look-back workspaces, adjacent, zero before their first use
        const int64_t ntiles =
            P->heavy_chunk * ((ncols + dense_tile<SR>() - 1) / dense_tile<SR>());
        cudaMemsetAsync(P->lb_w, 0,
                        (size_t)((char *)(P->lb_c + ntiles + 2) - (char *)P->lb_w), s);
    }
    return SUCCESS;
}

template <class SR>
static int plan_t(SaxpyPlan *P, const DevCSR *M, bool mask_comp, const DevCSR &A,
                  const DevCSR &B, cudaStream_t s)
{
    using Z = typename SR::z_t;
    int info = plan_symbolic<SR>(P, M, mask_comp, A, B, s);
    if (info == SUCCESS) info = plan_read(P, s);
    if (info != SUCCESS) return info;
    Carve tv(s);
    auto tlayout = [&]() {
        P->Tj = tv.take<int32_t>(P->total_cap + 1);
        P->Tx = tv.take<Z>(P->total_cap + 1);
    };
    tlayout();
    if (!tv.alloc()) return OUT_OF_MEMORY;
    tlayout();
    P->tblock = tv.base;
    P->slot_avail = P->total_cap;
    info = plan_alloc_heavy<SR>(P, s);
    if (info != SUCCESS) return info;
    return cuda_to_info(cudaGetLastError());
}

// blocks of a kernel that can be resident on the device at once (cached per
// kernel and shared-memory size)
static int resident_blocks(const void *fn, int threads, size_t smem)
{
    struct Entry { const void *fn; size_t smem; int blocks; };
    static std::mutex mu;
    static std::vector<Entry> cache;
    std::lock_guard<std::mutex> lk(mu);
    for (const Entry &e : cache)
        if (e.fn == fn && e.smem == smem) return e.blocks;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 1;
    }
    if (per_sm < 1) per_sm = 1;
    const int blocks = per_sm * runtime().num_sms;
    cache.push_back({fn, smem, blocks});
    return blocks;
}

// Launch shared-memory bin q.  rows_bound: the bin's row count when the host
// knows it (exact = true: an empty bin launches nothing), else an upper bound
// (the grid is then at most one resident wave, and the kernel reads the count
// and, through `need`, whether the slots fit).
template <class SR>
static void launch_bin(const SaxpyPlan *P, int q, const DevCSR &A, const DevCSR &B,
                       const DevCSR *M, int64_t rows_bound, bool exact, const int64_t *need,
                       cudaStream_t s)
{
    using Z = typename SR::z_t;
    const BinSpec &b = P->cfg.bin[q];
    if (rows_bound <= 0) return;
    const BinRows br{P->bin_rows, P->bins, q + 1, need, P->slot_avail};
    const size_t smem = bin_smem(b, sizeof(Z));
    int64_t cap_blocks = (int64_t)runtime().num_sms * P->cfg.blocks_per_sm;
    auto clamp = [&](int64_t want, const void *fn, int threads, size_t sm) {
        int64_t c = cap_blocks;
        if (!exact) {
            const int64_t wave = resident_blocks(fn, threads, sm);
            if (wave < c) c = wave;
        }
        if (want > c) want = c;
        return (int)(want < 1 ? 1 : want);
    };
    if (b.tpr == 1) {
        static bool attr = false;
        if (!attr) {
            allow_dynamic_smem((const void *)k_saxpy_esc<SR, uint32_t>);
            allow_dynamic_smem((const void *)k_saxpy_esc<SR, uint64_t>);
            attr = true;
        }
        int posb = 0;
        while ((1 << posb) < b.cap) posb++;
        const int64_t want = (rows_bound + ESC_WARPS - 1) / ESC_WARPS;
        // 32-bit keys when every (column << posb) and the padding fit
        if (((uint64_t)B.ncols << posb) < 0xffffffffull) {
            const size_t sm32 = (size_t)ESC_WARPS * b.cap * (4 + sizeof(Z));
            const int blocks = clamp(want, (const void *)k_saxpy_esc<SR, uint32_t>,
                                     ESC_WARPS * 32, sm32);
            k_saxpy_esc<SR, uint32_t><<<blocks, ESC_WARPS * 32, sm32, s>>>(br, b.cap,
                posb, A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso,
                M ? M->p : nullptr, M ? M->j : nullptr, M != nullptr, P->mask_comp,
                P->slot_off, P->Tj, (Z *)P->Tx, P->row_cnt);
        } else {
            const int blocks = clamp(want, (const void *)k_saxpy_esc<SR, uint64_t>,
                                     ESC_WARPS * 32, smem);
            k_saxpy_esc<SR, uint64_t><<<blocks, ESC_WARPS * 32, smem, s>>>(br, b.cap,
                posb, A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso,
                M ? M->p : nullptr, M ? M->j : nullptr, M != nullptr, P->mask_comp,
                P->slot_off, P->Tj, (Z *)P->Tx, P->row_cnt);
        }
    } else if (b.tpr >= 256) {
        static bool attr = false;
        if (!attr) {
            allow_dynamic_smem((const void *)k_saxpy_hash<SR, true>);
            attr = true;
        }
        const int blocks = clamp(rows_bound, (const void *)k_saxpy_hash<SR, true>, 256, smem);
        k_saxpy_hash<SR, true><<<blocks, 256, smem, s>>>(br, 8, b.cap,
            A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso,
            M ? M->p : nullptr, M ? M->j : nullptr, M != nullptr, P->mask_comp,
            P->slot_off, P->Tj, (Z *)P->Tx, P->row_cnt);
    } else {
        static bool attr = false;
        if (!attr) {
            allow_dynamic_smem((const void *)k_saxpy_hash<SR, false>);
            attr = true;
        }
        const int lg = b.tpr == 4 ? 2 : b.tpr == 8 ? 3 : b.tpr == 16 ? 4 : 5;
        const int groups = 128 / b.tpr;
        const int blocks = clamp((rows_bound + groups - 1) / groups,
                                 (const void *)k_saxpy_hash<SR, false>, 128, smem);
        k_saxpy_hash<SR, false><<<blocks, 128, smem, s>>>(br, lg, b.cap,
            A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso,
            M ? M->p : nullptr, M ? M->j : nullptr, M != nullptr, P->mask_comp,
            P->slot_off, P->Tj, (Z *)P->Tx, P->row_cnt);
    }
}

// the shared-memory bins: with exact host counts (after plan_read), or with
// m as every bin's bound and the fit check on the device
template <class SR>
static void exec_light(const SaxpyPlan *P, const DevCSR *M, const DevCSR &A, const DevCSR &B,
                       bool exact, cudaStream_t s)
{
    const int64_t *need = exact ? nullptr : (const int64_t *)(P->bins + BIN_TOTAL_CAP);
    for (int q = 0; q < P->cfg.nb; q++)
        launch_bin<SR>(P, q, A, B, M, exact ? P->h_bins[q + 1] : P->m, exact, need, s);
}

// the heavy rows (counts from plan_read, accumulators from plan_alloc_heavy)
template <class SR>
static void exec_heavy(SaxpyPlan *P, const DevCSR *M, const DevCSR &A, const DevCSR &B,
                       cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t ncols = P->ncols;
    const int nb = P->cfg.nb;
    const int nheavy = P->h_bins[nb + 1];
    if (nheavy == 0) return;
    const int32_t *hrows = P->bin_rows + P->h_start[nb + 1];
    int64_t *flag = P->flag;
    uint8_t *flag8 = P->flag8;
    Z *val = (Z *)P->val;
    dense_val_t<SR> *dval = (dense_val_t<SR> *)P->val;
    if constexpr (SR::order_free) {
        const int64_t chunk = P->heavy_chunk;
        for (int64_t c0 = 0; c0 < nheavy; c0 += chunk) {
            const int nr = (int)((nheavy - c0 < chunk) ? nheavy - c0 : chunk);
            // cleared flags, identity values and mask marks (and, for one
            // row, its flat index offsets)
            dim3 g1(nblocks(ncols, 256, 4), nr > 65535 ? 65535 : nr);
            k_dense_prep<SR><<<g1, 256, 0, s>>>(hrows + c0, nr, ncols, flag8, dval,
                M ? M->p : nullptr, M ? M->j : nullptr, M != nullptr, P->mask_comp, A.p,
                P->hoff);
            // flat product index of the chunk (the rows' offsets into their
            // entries, then each entry's B-row length scanned), then every
            // product over the grid
            if (nr == 1) {
                // offsets written by the prep kernel
            } else if (nr <= 1024) {
                k_heavy_offsets<<<1, 1024, 0, s>>>(hrows + c0, nr, A.p, P->hoff);
            } else {
                k_heavy_alen<<<(nr + 255) / 256, 256, 0, s>>>(hrows + c0, nr, A.p, P->hlen);
                scan_exclusive_i64_ws(P->hlen, P->hoff, nr + 1, P->hw_ws, s);
            }
            lb_scan(LbLoadBlen{hrows + c0, nr, P->hoff, A.p, A.j, B.p}, P->wprefix,
                    P->heavy_alen + 1, P->lb_w, s, nullptr, nullptr, P->bins + BIN_HEAVY_ERR);
            k_dense_atomic_flat<SR><<<runtime().num_sms * 32, 256, 0, s>>>(hrows + c0, nr,
                P->hoff, P->wprefix, A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso,
                M != nullptr, P->mask_comp, ncols, flag8, dval);
            // ordered compaction into the rows' slots
            const int cblocks = (int)((ncols + dense_tile<SR>() - 1) / dense_tile<SR>());
            const int64_t ntiles = (int64_t)nr * cblocks;
            k_dense_compact<SR><<<(unsigned)ntiles, DG_THREADS, 0, s>>>(hrows + c0, cblocks,
                ncols, flag8, dval, P->slot_off, P->Tj, (Z *)P->Tx, P->row_cnt, ntiles,
                P->lb_c, P->bins + BIN_HEAVY_ERR);
        }
    } else {
        const int nbk = (int)P->heavy_chunk;
        cudaMemsetAsync(flag, 0, (size_t)nbk * ncols * 8, s);
        k_saxpy_dense_seq<SR><<<nbk, 256, 0, s>>>(hrows, nheavy, A.p, A.j, A.x, A.iso,
            B.p, B.j, B.x, B.iso, M ? M->p : nullptr, M ? M->j : nullptr,
            M != nullptr, P->mask_comp, ncols, flag, val, P->slot_off, P->Tj,
            (Z *)P->Tx, P->row_cnt);
    }
}

// exact row counts -> C's row offsets (int64 in Cp64, int32 in Cp) and the
// output count
static void exec_counts(SaxpyPlan *P, int32_t *Cp, int64_t *Cnnz64, cudaStream_t s)
{
    scan_exclusive_lb_counts(P->row_cnt, P->row_bin, P->m, P->Cp64, P->lb_row, s,
                             Cnnz64 ? Cnnz64 : (int64_t *)(P->bins + BIN_NNZ), Cp,
                             P->bins + BIN_ROW_ERR);
}

// the slots, packed into C's exact arrays
template <typename Z>
static void exec_pack(const SaxpyPlan *P, int32_t *Cj, Z *Cx, cudaStream_t s,
                      int64_t cap = -1)
{
    // cap < 0: the host knows the sizes (total_cap bounds the entries);
    // otherwise C holds cap entries and the kernel checks the count itself
    const int64_t grid_n = cap < 0 ? P->total_cap : cap;
    if (P->m > 0 && grid_n > 0)
        k_pack<Z><<<nblocks(grid_n, 256, 16), 256, 0, s>>>(P->m, flat_span(grid_n),
            P->slot_off, P->Tj, (const Z *)P->Tx, P->Cp64, Cj, Cx,
            cap < 0 ? (int64_t)INT64_MAX : cap);
}

template <class SR>
static int exec_t(SaxpyPlan *P, const DevCSR *M, const DevCSR &A, const DevCSR &B,
                  int32_t *Cp, int32_t *Cj, void *Cx, int64_t *Cnnz64, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int ps = prof_begin("saxpy3_numeric", s);
    exec_light<SR>(P, M, A, B, true, s);
    exec_heavy<SR>(P, M, A, B, s);
    prof_end(ps, s);
    exec_counts(P, Cp, Cnnz64, s);
    exec_pack<Z>(P, Cj, (Z *)Cx, s);
    return cuda_to_info(cudaGetLastError());
}

int saxpy_plan_create(SaxpyPlan **Pout, const DevCSR *M, bool mask_comp,
                      const DevCSR &A, const DevCSR &B, SemiringCode sr,
                      const SaxpyConfig &cfg, cudaStream_t s)
{
    if (A.ncols != B.nrows) return DIMENSION_MISMATCH;
    if (M && (M->nrows != A.nrows || M->ncols != B.ncols)) return DIMENSION_MISMATCH;
    SaxpyPlan *P = new SaxpyPlan();
    P->sr = sr;
    P->cfg = cfg;
    int info = NO_VALUE;
#define GRB_PLAN_CASE(ADD, MULT, TC, CT)                                        \
    if (sr.add == ADD && sr.mult == MULT && sr.type == TC) {                    \
        if (!saxpy_config_valid(cfg, sizeof(CT))) info = INVALID_VALUE;         \
        else info = plan_t<Semiring<ADD, MULT, CT>>(P, M, mask_comp, A, B, s);  \
    } else
    GRB_FOR_EACH_SEMIRING(GRB_PLAN_CASE) { info = NO_VALUE; }
#undef GRB_PLAN_CASE
    if (info != SUCCESS) { saxpy_plan_free(P, s); return info; }
    *Pout = P;
    return SUCCESS;
}

int saxpy_plan_exec(SaxpyPlan *P, const DevCSR *M, const DevCSR &A, const DevCSR &B,
                    int32_t *Cp, int32_t *Cj, void *Cx, int64_t *Cnnz64, cudaStream_t s)
{
    const SemiringCode sr = P->sr;
#define GRB_EXEC_CASE(ADD, MULT, TC, CT)                                        \
    if (sr.add == ADD && sr.mult == MULT && sr.type == TC)                      \
        return exec_t<Semiring<ADD, MULT, CT>>(P, M, A, B, Cp, Cj, Cx, Cnnz64, s);
    GRB_FOR_EACH_SEMIRING(GRB_EXEC_CASE)
#undef GRB_EXEC_CASE
    return NO_VALUE;
}

// Where the slots of a one-shot product live: the stream's scratch buffer
// when the library owns the stream, else a buffer for this call.
struct SlotSource {
    cudaStream_t s;
    bool shared;
    void *own = nullptr;
    size_t have = 0;
    explicit SlotSource(cudaStream_t st) : s(st), shared(stream_scratch_enabled(st))
    {
        if (shared) have = stream_scratch_size(st);
    }
    ~SlotSource() { dfree(own, s); }
    void *get(size_t want)
    {
        if (shared) return stream_scratch(s, want, &have);
        dfree(own, s);
        own = dalloc(want, s);
        have = own ? want : 0;
        return own;
    }
};

// A one-row product whose row is expected to be heavy (vxm with a large
// frontier), with an order-free monoid: straight to the dense accumulator,
// with no symbolic phase and no host round trip before it.  The row's A
// entries are its whole flat index; its slots hold every column.
template <class SR>
static int saxpy3_row_dense(DevCSR &C, const DevCSR *M, bool mask_comp, const DevCSR &A,
                            const DevCSR &B, SemiringCode sr, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t ncols = B.ncols;
    SaxpyPlan *P = new SaxpyPlan();
    struct PlanGuard { SaxpyPlan *P; cudaStream_t s; ~PlanGuard() { saxpy_plan_free(P, s); } }
        pg{P, s};
    P->sr = sr;
    P->cfg = saxpy_default_config();
    P->zsize = sizeof(Z);
    P->order_free = true;
    P->m = 1; P->ncols = ncols;
    P->has_mask = M != nullptr; P->mask_comp = mask_comp;
    const int nb = P->cfg.nb;
    P->h_bins[nb + 1] = 1;
    P->h_start[nb + 1] = 0;
    P->heavy_alen = A.nnz;
    P->heavy_chunk = 1;
    P->total_cap = ncols;
    const int64_t ntiles = (ncols + dense_tile<SR>() - 1) / dense_tile<SR>();
    // everything in one allocation; the counters, the look-back workspaces,
    // the slot offset, the row count and the row list (row 0) are zero
    Carve cv(s);
    auto layout = [&]() {
        P->bins = cv.take<int>(BINS_WORDS);
        P->lb_row = cv.take<unsigned long long>(scan_lb_ws_elems(2));
        P->slot_off = cv.take<int64_t>(2);
        P->row_cnt = cv.take<int32_t>(2);
        P->bin_rows = cv.take<int32_t>(2);
        P->lb_w = cv.take<unsigned long long>(lb_ws_elems(A.nnz + 1));
        P->lb_c = cv.take<unsigned long long>(ntiles + 2);
        P->Cp64 = cv.take<int64_t>(3);
        P->hoff = cv.take<int64_t>(2);
        P->hlen = cv.take<int64_t>(2);
        P->hw_ws = cv.take<int64_t>(scan_ws_elems(2));
        P->wprefix = cv.take<int64_t>(A.nnz + 1);
        P->flag8 = cv.take<uint8_t>(ncols + 1);
        P->val = cv.take<dense_val_t<SR>>(ncols + 1);
    };
    layout();
    if (!cv.alloc()) return OUT_OF_MEMORY;
    layout();
    P->block = cv.base;
    P->row_bin = nullptr;                 // the one row counts
    cudaMemsetAsync(P->bins, 0, (size_t)((char *)(P->lb_c + ntiles + 2) - (char *)P->bins), s);
    DevCSR T;
    T.nrows = 1; T.ncols = ncols; T.type = sr.type; T.iso = false;
    T.p = (int32_t *)dalloc(2 * 4, s);
    if (!T.p) return OUT_OF_MEMORY;
    SlotSource src(s);
    void *slots = src.get(src.have >= slot_bytes(P, ncols) ? src.have : slot_bytes(P, ncols));
    if (!slots) { dev_free(T, s); return OUT_OF_MEMORY; }
    plan_place_slots(P, slots, src.have);
    const int ps = prof_begin("saxpy3_numeric", s);
    exec_heavy<SR>(P, M, A, B, s);
    prof_end(ps, s);
    exec_counts(P, T.p, nullptr, s);
    int hb[BINS_READ];
    cudaError_t e = readback(hb, P->bins, sizeof(hb), s);
    if (e != cudaSuccess) { dev_free(T, s); return cuda_to_info(e); }
    if (hb[BIN_ROW_ERR] || hb[BIN_HEAVY_ERR]) { dev_free(T, s); return PANIC; }
    int64_t nnz = 0;
    memcpy(&nnz, hb + BIN_NNZ, 8);
    T.nnz = nnz;
    T.j = (int32_t *)dalloc((size_t)(nnz + 1) * 4, s);
    T.x = dalloc((size_t)(nnz + 1) * sizeof(Z), s);
    if (!T.j || !T.x) { dev_free(T, s); return OUT_OF_MEMORY; }
    exec_pack<Z>(P, T.j, (Z *)T.x, s);
    const int info = cuda_to_info(cudaGetLastError());
    if (info != SUCCESS) { dev_free(T, s); return info; }
    C = T;
    return SUCCESS;
}

// One-shot C<M> = A*B with one host round trip in the common case.  The
// symbolic phase, the shared-memory bins, the row offsets and the pack are
// queued together: the bins write their slots into the stream's scratch
// buffer and read their row counts and the slot total on the device, and the
// pack fills C's arrays, allocated beforehand from B's mean row length, if
// the product fits them.  One read brings back the counts, the slot total
// and the output size; only if the slots did not fit (the buffer then grows
// and the bins run again), heavy rows need their accumulators sized, or C
// needs larger arrays does more work follow the read.
// The one-launch path (k_saxpy_small) for products of SMALL_MIN_ROWS to
// SMALL_MAX_ROWS rows whose rows are expected to fit the expand-sort-compress
// bin (A's entries times B's mean row length, per row, at most half the
// bin), with fewer than 2^24 columns (32-bit sort keys).  The slots take
// SMALL_CAP entries a row from the stream's buffer; C's arrays are sized
// from B's mean row length as in the general path.  NO_VALUE when the
// product is not taken, or when the launch found a row past the bin or too
// little room in C (the caller then runs the general path).
static constexpr int64_t SMALL_MIN_ROWS = 256, SMALL_MAX_ROWS = 32768;


template <class SR>
static int saxpy3_small(DevCSR &C, const DevCSR *M, bool mask_comp, const DevCSR &A,
                        const DevCSR &B, SemiringCode sr, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t m = A.nrows;
    if (m < SMALL_MIN_ROWS || m > SMALL_MAX_ROWS || A.nnz <= 0 ||
        B.ncols >= ((int64_t)1 << 24))
        return NO_VALUE;
    const double mean_b = B.nrows > 0 ? (double)B.nnz / (double)B.nrows : 0.0;
    const double flops_est = (double)A.nnz * (mean_b > 1.0 ? mean_b : 1.0);
    if (flops_est > 0.5 * SMALL_CAP * (double)m) return NO_VALUE;
    const size_t smem = (size_t)ESC_WARPS * SMALL_CAP * (4 + sizeof(Z));
    const int resident = resident_blocks((const void *)k_saxpy_small<SR>, ESC_WARPS * 32, smem);
    const int64_t chunk = (m + resident - 1) / resident;
    if (chunk > SMALL_CHUNK) return NO_VALUE;
    const int G = (int)((m + chunk - 1) / chunk);

    // one block: tot[8] and the blocks' look-back words part[G], then
    // SMALL_CAP slots per row (values, then columns)
    const size_t hdr = ((size_t)(8 + (size_t)G) * 8 + 255) & ~(size_t)255;
    const size_t xbytes = ((size_t)m * SMALL_CAP * sizeof(Z) + 255) & ~(size_t)255;
    SlotSource src(s);
    char *base = (char *)src.get(hdr + xbytes + (size_t)m * SMALL_CAP * 4);
    if (!base) return NO_VALUE;
    long long *tot = (long long *)base;
    long long *part = tot + 8;
    Z *Tx = (Z *)(base + hdr);
    int32_t *Tj = (int32_t *)(base + hdr + xbytes);

    double cg = 1.15 * flops_est + 64.0;
    const double cfull = (double)m * (double)B.ncols;
    if (cg > cfull + 64.0) cg = cfull + 64.0;
    const int64_t ccap = (int64_t)cg;
    DevCSR T;
    T.nrows = m; T.ncols = B.ncols; T.type = sr.type; T.iso = false;
    T.p = (int32_t *)dalloc((size_t)(m + 1) * 4, s);
    T.j = (int32_t *)dalloc((size_t)(ccap + 1) * 4, s);
    T.x = dalloc((size_t)(ccap + 1) * sizeof(Z), s);
    if (!T.p || !T.j || !T.x) { dev_free(T, s); return NO_VALUE; }
    cudaMemsetAsync(tot, 0, (8 + (size_t)G) * sizeof(long long), s);
    const int ps = prof_begin("saxpy3_numeric", s);
    k_saxpy_small<SR><<<G, ESC_WARPS * 32, smem, s>>>((int32_t)m, (int32_t)chunk,
        A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso,
        M ? M->p : nullptr, M ? M->j : nullptr, M != nullptr, mask_comp,
        part, Tj, Tx, T.p, T.j, (Z *)T.x, ccap, tot);
    prof_end(ps, s);
    long long h[3] = {0, 0, 0};
    const cudaError_t e = readback(h, tot, sizeof(h), s);
    if (e != cudaSuccess) { dev_free(T, s); return cuda_to_info(e); }
    if (h[2] != 0 || h[1] != SMALL_DONE) { dev_free(T, s); return NO_VALUE; }
    T.nnz = h[0];
    C = T;
    return SUCCESS;
}

template <class SR>
static int saxpy3_t(DevCSR &C, const DevCSR *M, bool mask_comp, const DevCSR &A,
                    const DevCSR &B, SemiringCode sr, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t m = A.nrows;
    const double mean_b = B.nrows > 0 ? (double)B.nnz / (double)B.nrows : 0.0;
    if constexpr (SR::order_free) {
        // a one-row product expected far past the shared-memory bins, whose
        // dense row fits comfortably: the dense path directly
        const SaxpyConfig dc = saxpy_default_config();
        const double est = (double)A.nnz * mean_b;
        if (m == 1 && A.nnz > 0 && est >= 2.0 * (double)dc.bin[dc.nb - 1].limit &&
            (double)B.ncols * (1.0 + sizeof(Z)) <= (double)((int64_t)4 << 30))
            return saxpy3_row_dense<SR>(C, M, mask_comp, A, B, sr, s);
    }
    {
        const int r = saxpy3_small<SR>(C, M, mask_comp, A, B, sr, s);
        if (r != NO_VALUE) return r;
    }
    SaxpyPlan *P = new SaxpyPlan();
    P->sr = sr;
    P->cfg = saxpy_default_config();
    struct PlanGuard { SaxpyPlan *P; cudaStream_t s; ~PlanGuard() { saxpy_plan_free(P, s); } }
        pg{P, s};
    int info = plan_symbolic<SR>(P, M, mask_comp, A, B, s);
    if (info != SUCCESS) return info;
    DevCSR T;
    T.nrows = m; T.ncols = B.ncols; T.type = sr.type; T.iso = false;
    T.p = (int32_t *)dalloc((size_t)(m + 1) * 4, s);
    if (!T.p) return OUT_OF_MEMORY;
    // the slots: the stream's buffer as it is, or a first one sized from the
    // mean row length of B (grown below if the rows need more)
    SlotSource src(s);
    size_t want = src.have;
    if (want == 0) {
        double guess = 2.0 * (double)A.nnz * (mean_b > 1.0 ? mean_b : 1.0) + (double)m + 1024;
        const double full = (double)m * (double)B.ncols;
        if (guess > full + 1024) guess = full + 1024;
        if (guess > (double)(64 << 20)) guess = (double)(64 << 20);
        want = slot_bytes(P, (int64_t)guess);
    }
    void *slots = src.get(want);
    if (!slots) { dev_free(T, s); return OUT_OF_MEMORY; }
    plan_place_slots(P, slots, src.have);
    // C's arrays before the read, sized from B's mean row length: when the
    // product fits (as a product of evenly filled rows does), the pack runs
    // before the read and nothing follows it
    double cg = 1.15 * (double)A.nnz * (mean_b > 1.0 ? mean_b : 1.0) + 64.0;
    const double cfull = (double)m * (double)B.ncols;
    if (cg > cfull + 64.0) cg = cfull + 64.0;
    if (cg > (double)(INT32_MAX - 1)) cg = (double)(INT32_MAX - 1);
    int64_t cap = (int64_t)cg;
    T.j = (int32_t *)dalloc((size_t)(cap + 1) * 4, s);
    T.x = dalloc((size_t)(cap + 1) * sizeof(Z), s);
    if (!T.j || !T.x) {
        dfree(T.j, s); dfree(T.x, s);
        T.j = nullptr; T.x = nullptr;
        cap = -1;
    }
    const int ps = prof_begin("saxpy3_numeric", s);
    exec_light<SR>(P, M, A, B, false, s);
    prof_end(ps, s);
    exec_counts(P, T.p, nullptr, s);
    if (cap >= 0) exec_pack<Z>(P, T.j, (Z *)T.x, s, cap);
    info = plan_read(P, s);
    if (info != SUCCESS) { dev_free(T, s); return info; }
    bool again = false;
    if (P->total_cap > P->slot_avail) {
        // the bins did nothing: more slots, then the bins with exact counts
        slots = src.get(slot_bytes(P, P->total_cap + P->total_cap / 4));
        if (!slots) { dev_free(T, s); return OUT_OF_MEMORY; }
        plan_place_slots(P, slots, src.have);
        exec_light<SR>(P, M, A, B, true, s);
        again = true;
    }
    if (P->h_bins[P->cfg.nb + 1] > 0) {
        info = plan_alloc_heavy<SR>(P, s);
        if (info != SUCCESS) { dev_free(T, s); return info; }
        exec_heavy<SR>(P, M, A, B, s);
        again = true;
    }
    if (again) {
        exec_counts(P, T.p, nullptr, s);
        info = plan_read(P, s);
        if (info != SUCCESS) { dev_free(T, s); return info; }
    }
    const int64_t nnz = P->nnz;
    if (nnz >= INT32_MAX) { dev_free(T, s); return OUT_OF_MEMORY; }
    T.nnz = nnz;
    if (again || nnz > cap) {
        // the early pack saw incomplete rows or did not fit: pack now
        if (nnz > cap) {
            dfree(T.j, s); dfree(T.x, s);
            T.j = (int32_t *)dalloc((size_t)(nnz + 1) * 4, s);
            T.x = dalloc((size_t)(nnz + 1) * sizeof(Z), s);
            if (!T.j || !T.x) { dev_free(T, s); return OUT_OF_MEMORY; }
        }
        exec_pack<Z>(P, T.j, (Z *)T.x, s);
    } else if (cap > 2 * nnz + (1 << 20)) {
        // far more room than entries: exact arrays
        int32_t *j2 = (int32_t *)dalloc((size_t)(nnz + 1) * 4, s);
        void *x2 = dalloc((size_t)(nnz + 1) * sizeof(Z), s);
        if (j2 && x2) {
            cudaMemcpyAsync(j2, T.j, (size_t)nnz * 4, cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(x2, T.x, (size_t)nnz * sizeof(Z), cudaMemcpyDeviceToDevice, s);
            dfree(T.j, s); dfree(T.x, s);
            T.j = j2; T.x = x2;
        } else {
            dfree(j2, s); dfree(x2, s);
        }
    }
    info = cuda_to_info(cudaGetLastError());
    if (info != SUCCESS) { dev_free(T, s); return info; }
    C = T;
    return SUCCESS;
}

// one-shot C<M> = A*B
int saxpy3(DevCSR &C, const DevCSR *M, bool mask_comp, bool mask_struct,
           const DevCSR &A, const DevCSR &B, SemiringCode sr, cudaStream_t s)
{
    if (A.ncols != B.nrows) return DIMENSION_MISMATCH;
    if (M && (M->nrows != A.nrows || M->ncols != B.ncols)) return DIMENSION_MISMATCH;
    if (!semiring_supported(sr)) return NO_VALUE;
    DevCSR Ms;
    bool own_mask = false;
    if (M && !mask_struct && M->x) {
        // a valued mask is reduced to its true entries first
        int info = dev_mask_to_struct(Ms, *M, s);
        if (info != SUCCESS) return info;
        M = &Ms;
        own_mask = true;
    } else if (M && M->nzombies > 0) {
        return NO_VALUE;
    }
    struct Guard { DevCSR *m; bool own; cudaStream_t s;
        ~Guard() { if (own) dev_free(*m, s); } } guard{&Ms, own_mask, s};
    int info = NO_VALUE;
#define GRB_ONESHOT_CASE(ADD, MULT, TC, CT)                                     \
    if (sr.add == ADD && sr.mult == MULT && sr.type == TC)                      \
        info = saxpy3_t<Semiring<ADD, MULT, CT>>(C, M, mask_comp, A, B, sr, s); \
    else
    GRB_FOR_EACH_SEMIRING(GRB_ONESHOT_CASE) { info = NO_VALUE; }
#undef GRB_ONESHOT_CASE
    if (info != SUCCESS) return info;
    return cuda_to_info(cudaStreamSynchronize(s));
}

}  // namespace grb
