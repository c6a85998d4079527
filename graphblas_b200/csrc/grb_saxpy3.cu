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
//        tiny/small/medium rows: a group of TPR threads owns one row and a
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
//      spread all products over the grid with atomic updates.
//   4. each row's entries are sorted by column in shared memory (bitonic) and
//      written to its slot; a compaction kernel packs the slots into CSR.
//
// Masks: M (or !M) is scattered into the row's table first (the reference's
// "scatter M" step, GB_AxB_saxpy3_symbolic.c), with a state per slot:
// allowed-unset, set, or forbidden.

#include <cstdio>
#include <cstring>
#include "grb_runtime.h"
#include "grb_semirings.h"

namespace grb {

// slot states
static constexpr uint8_t S_EMPTY = 0, S_ALLOWED = 1, S_SET = 2, S_FORBID = 3;

// ---------------------------------------------------------------------------
// phase 1: flops and capacity per row
// ---------------------------------------------------------------------------

__global__ void k_flops(const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
                        const int32_t *__restrict__ Bp,
                        const int32_t *__restrict__ Mp, bool mask_bounds,
                        int64_t nrows, int64_t ncols,
                        int64_t *__restrict__ flops, int64_t *__restrict__ cap)
{
    // one warp per row
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int lane = threadIdx.x & 31;
    for (int64_t r = warp; r < nrows; r += nw) {
        int32_t lo = Ap[r], hi = Ap[r + 1];
        int64_t f = 0;
        for (int32_t p = lo + lane; p < hi; p += 32) {
            int32_t k = Aj[p];
            f += Bp[k + 1] - Bp[k];
        }
        for (int o = 16; o > 0; o >>= 1) f += __shfl_down_sync(0xffffffffu, f, o);
        if (lane == 0) {
            int64_t c = f < ncols ? f : ncols;
            if (mask_bounds) {
                int64_t mc = Mp[r + 1] - Mp[r];
                if (mc < c) c = mc;
            }
            if (f == 0) c = 0;
            flops[r] = f;
            cap[r] = c;
        }
    }
}

// bin of a row: 0 empty, 1..NB_SMEM smem hash bins, NB_SMEM+1 heavy
static constexpr int NB_SMEM = 4;
// max flops (+ mask entries) handled by each shared-memory bin
__constant__ int64_t c_bin_limit[NB_SMEM] = {64, 256, 1024, 4096};

__global__ void k_bin_rows(const int64_t *__restrict__ flops,
                           const int32_t *__restrict__ Mp, bool has_mask,
                           int64_t nrows, int *__restrict__ bin_count,
                           int32_t *__restrict__ bin_rows_scratch,
                           int8_t *__restrict__ row_bin)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = t; r < nrows; r += stride) {
        int64_t f = flops[r];
        int b;
        if (f == 0) b = 0;
        else {
            int64_t need = f + (has_mask ? (int64_t)(Mp[r + 1] - Mp[r]) : 0);
            b = NB_SMEM + 1;
            for (int q = 0; q < NB_SMEM; q++)
                if (need <= c_bin_limit[q]) { b = q + 1; break; }
        }
        row_bin[r] = (int8_t)b;
        if (b > 0) atomicAdd(&bin_count[b], 1);
    }
}

// scatter rows into per-bin lists (order within a bin does not matter)
__global__ void k_fill_bins(const int8_t *__restrict__ row_bin, int64_t nrows,
                            int *__restrict__ bin_fill,
                            const int *__restrict__ bin_start,
                            int32_t *__restrict__ bin_rows)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = t; r < nrows; r += stride) {
        int b = row_bin[r];
        if (b > 0) {
            int pos = atomicAdd(&bin_fill[b], 1);
            bin_rows[bin_start[b] + pos] = (int32_t)r;
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

template <class SR, int TPR, int CAP>
struct HashLayout {
    using Z = typename SR::z_t;
    static constexpr int GROUPS = (TPR >= 256) ? 1 : (128 / TPR);   // per block
    static constexpr int THREADS = GROUPS * TPR;
    // per group: keys[CAP] int32, vals[CAP] Z, state[CAP] u8
    static constexpr size_t GROUP_BYTES =
        ((CAP * 4 + CAP * sizeof(Z) + CAP + 15) / 16) * 16;
    static constexpr size_t BYTES = GROUP_BYTES * GROUPS;
};

template <class SR, int TPR, int CAP>
__global__ void __launch_bounds__(HashLayout<SR, TPR, CAP>::THREADS)
k_saxpy_hash(const int32_t *__restrict__ rows, int nrows_bin,
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
    using L = HashLayout<SR, TPR, CAP>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int g = threadIdx.x / TPR;
    const int t = threadIdx.x % TPR;
    unsigned char *base = smem + (size_t)g * L::GROUP_BYTES;
    int32_t *keys = (int32_t *)base;
    Z *vals = (Z *)(base + CAP * 4);
    uint8_t *state = (uint8_t *)(base + CAP * 4 + CAP * sizeof(Z));
    const uint32_t hmask = CAP - 1;

    for (int64_t rb = (int64_t)blockIdx.x * L::GROUPS + g; rb < nrows_bin;
         rb += (int64_t)gridDim.x * L::GROUPS) {
        const int32_t i = rows[rb];
        for (int s = t; s < CAP; s += TPR) { keys[s] = -1; state[s] = S_EMPTY; }
        group_sync<TPR>();
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
            group_sync<TPR>();
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
            group_sync<TPR>();
        }
        // gather the set slots into the row's output slot, then sort them
        // by column in the (now free) table memory with a bitonic network
        const int64_t off = slot_off[i];
        __shared__ int s_cnt[L::GROUPS];
        if (t == 0) s_cnt[g] = 0;
        group_sync<TPR>();
        for (int s = t; s < CAP; s += TPR) {
            if (state[s] == S_SET) {
                int q = atomicAdd(&s_cnt[g], 1);
                Tj[off + q] = keys[s];
                Tx[off + q] = vals[s];
            }
        }
        group_sync<TPR>();
        const int cnt = s_cnt[g];
        int n2 = 1;
        while (n2 < cnt) n2 <<= 1;
        for (int q = t; q < n2; q += TPR) {
            if (q < cnt) { keys[q] = Tj[off + q]; vals[q] = Tx[off + q]; }
            else keys[q] = INT32_MAX;
        }
        group_sync<TPR>();
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
                group_sync<TPR>();
            }
        }
        for (int q = t; q < cnt; q += TPR) { Tj[off + q] = keys[q]; Tx[off + q] = vals[q]; }
        if (t == 0) row_cnt[i] = cnt;
        group_sync<TPR>();
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

template <class SR>
__global__ void k_dense_init(const int32_t *__restrict__ rows, int nrows_bin,
                             int64_t ncols, int64_t *__restrict__ flag_all,
                             typename SR::z_t *__restrict__ val_all)
{
    // one block-row of workspace per heavy row (rows are few)
    for (int64_t rb = blockIdx.y; rb < nrows_bin; rb += gridDim.y) {
        int64_t *flag = flag_all + rb * ncols;
        typename SR::z_t *val = val_all + rb * ncols;
        for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ncols;
             j += (int64_t)gridDim.x * blockDim.x) {
            flag[j] = 0;
            val[j] = dense_init<SR>();
        }
    }
}

// mark mask columns: 1 allowed / 2 forbidden
__global__ void k_dense_mask(const int32_t *__restrict__ rows, int nrows_bin,
                             const int32_t *__restrict__ Mp,
                             const int32_t *__restrict__ Mj, bool mask_comp,
                             int64_t ncols, int64_t *__restrict__ flag_all)
{
    for (int64_t rb = blockIdx.y; rb < nrows_bin; rb += gridDim.y) {
        const int32_t i = rows[rb];
        int64_t *flag = flag_all + rb * ncols;
        for (int32_t pm = Mp[i] + blockIdx.x * blockDim.x + threadIdx.x; pm < Mp[i + 1];
             pm += gridDim.x * blockDim.x)
            flag[Mj[pm]] = mask_comp ? 2 : 1;
    }
}

// every product (i,k,j) of the heavy rows, spread over the grid: a warp takes
// one A entry (i,k) at a time and its lanes split B(k,:)
template <class SR>
__global__ void k_dense_atomic(const int32_t *__restrict__ rows, int nrows_bin,
                               const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
                               const void *__restrict__ Ax, bool a_iso,
                               const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
                               const void *__restrict__ Bx, bool b_iso,
                               bool has_mask, bool mask_comp, int64_t ncols,
                               int64_t *__restrict__ flag_all,
                               typename SR::z_t *__restrict__ val_all)
{
    using Z = typename SR::z_t;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t rb = blockIdx.y; rb < nrows_bin; rb += gridDim.y) {
        const int32_t i = rows[rb];
        int64_t *flag = flag_all + rb * ncols;
        Z *val = val_all + rb * ncols;
        const int32_t pa0 = Ap[i], pa1 = Ap[i + 1];
        for (int64_t pa = pa0 + warp; pa < pa1; pa += nw) {
            const int32_t k = Aj[pa];
            Z a = Z();
            if (SR::needs_a) a = ld_val<Z>(Ax, pa, a_iso);
            for (int32_t pb = Bp[k] + lane; pb < Bp[k + 1]; pb += 32) {
                const int32_t j = Bj[pb];
                if (has_mask) {
                    const int64_t f = flag[j];
                    if (!mask_comp && f == 0) continue;
                    if (mask_comp && f == 2) continue;
                }
                Z b = Z();
                if (SR::needs_b) b = ld_val<Z>(Bx, pb, b_iso);
                const Z tv = SR::F::f(a, b, i, k, j);
                AtomicUpd<SR::add_op, Z>::run(&val[j], tv);
                flag[j] = 3;
            }
        }
    }
}

// ordered compaction of the dense rows (one block per heavy row)
template <class SR>
__global__ void __launch_bounds__(256)
k_dense_gather(const int32_t *__restrict__ rows, int nrows_bin, int64_t ncols,
               const int64_t *__restrict__ flag_all,
               const typename SR::z_t *__restrict__ val_all,
               const int64_t *__restrict__ slot_off, int32_t *__restrict__ Tj,
               typename SR::z_t *__restrict__ Tx, int32_t *__restrict__ row_cnt)
{
    __shared__ int s_warp[8];
    __shared__ int s_base;
    for (int64_t rb = blockIdx.x; rb < nrows_bin; rb += gridDim.x) {
        const int32_t i = rows[rb];
        const int64_t *flag = flag_all + rb * ncols;
        const typename SR::z_t *val = val_all + rb * ncols;
        const int64_t off = slot_off[i];
        int total = 0;
        for (int64_t c0 = 0; c0 < ncols; c0 += blockDim.x) {
            const int64_t j = c0 + threadIdx.x;
            const bool on = (j < ncols) && (flag[j] == 3);
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
        if (threadIdx.x == 0) row_cnt[i] = total;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// phase 4: sort each row's slot by column and pack the slots into CSR
// ---------------------------------------------------------------------------

// copy each row's (sorted) slot to its place in C (one warp per row)
template <typename Z>
__global__ void __launch_bounds__(256)
k_pack(int64_t nrows, const int64_t *__restrict__ slot_off,
       const int32_t *__restrict__ Tj, const Z *__restrict__ Tx,
       const int32_t *__restrict__ row_cnt, const int64_t *__restrict__ Cp64,
       int32_t *__restrict__ Cj, Z *__restrict__ Cx)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < nrows; r += nw) {
        const int cnt = row_cnt[r];
        const int64_t src = slot_off[r], dst = Cp64[r];
        for (int q = lane; q < cnt; q += 32) { Cj[dst + q] = Tj[src + q]; Cx[dst + q] = Tx[src + q]; }
    }
}

__global__ void k_cnt_to_i64(const int32_t *__restrict__ cnt, const int8_t *__restrict__ row_bin,
                             int64_t n, int64_t *__restrict__ out)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < n; t += stride) out[t] = row_bin[t] ? (int64_t)cnt[t] : 0;
}

__global__ void k_i64_to_i32_p(const int64_t *__restrict__ in, int32_t *__restrict__ out, int64_t n)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < n; t += stride) out[t] = (int32_t)in[t];
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------

static inline int nblocks(int64_t n, int threads, int per_sm = 8)
{
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)runtime().num_sms * per_sm;
    if (b > cap) b = cap;
    return b < 1 ? 1 : (int)b;
}

template <class SR, int TPR, int CAP>
static void launch_hash_bin(const int32_t *rows, int cnt, const DevCSR &A,
                            const DevCSR &B, const DevCSR *M, bool mask_comp,
                            const int64_t *slot_off, int32_t *Tj,
                            typename SR::z_t *Tx, int32_t *row_cnt, cudaStream_t s)
{
    using L = HashLayout<SR, TPR, CAP>;
    if (cnt == 0) return;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_saxpy_hash<SR, TPR, CAP>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
        attr_set = true;
    }
    int64_t groups_needed = cnt;
    int blocks = (int)((groups_needed + L::GROUPS - 1) / L::GROUPS);
    int cap = runtime().num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_saxpy_hash<SR, TPR, CAP><<<blocks, L::THREADS, L::BYTES, s>>>(
        rows, cnt, A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso,
        M ? M->p : nullptr, M ? M->j : nullptr, M != nullptr, mask_comp,
        slot_off, Tj, Tx, row_cnt);
}

template <class SR>
static int saxpy3_t(DevCSR &C, const DevCSR *M, bool mask_comp,
                    const DevCSR &A, const DevCSR &B, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t m = A.nrows, ncols = B.ncols;
    Scratch ws(s);
    int64_t *flops = ws.get<int64_t>(m + 1);
    int64_t *capv = ws.get<int64_t>(m + 1);
    int8_t *row_bin = ws.get<int8_t>(m + 1);
    int *bins = ws.get<int>(64);
    int32_t *bin_rows = ws.get<int32_t>(m + 1);
    int32_t *row_cnt = ws.get<int32_t>(m + 1);
    if (ws.failed) return OUT_OF_MEMORY;
    const bool mask_bounds = (M != nullptr) && !mask_comp;
    if (m > 0)
        k_flops<<<nblocks(m * 32, 256), 256, 0, s>>>(A.p, A.j, B.p,
            M ? M->p : nullptr, mask_bounds, m, ncols, flops, capv);
    cudaMemsetAsync(bins, 0, 64 * sizeof(int), s);
    if (m > 0)
        k_bin_rows<<<nblocks(m, 256), 256, 0, s>>>(flops, M ? M->p : nullptr,
            M != nullptr, m, bins, nullptr, row_bin);
    // capacities -> slot offsets
    cudaMemsetAsync(capv + m, 0, 8, s);
    int info = scan_exclusive_i64(capv, capv, m + 1, s);
    if (info != SUCCESS) return info;
    int h_bins[NB_SMEM + 2] = {0};
    int64_t total_cap = 0;
    cudaMemcpyAsync(h_bins, bins, sizeof(h_bins), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&total_cap, capv + m, 8, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_to_info(e);
    // per-bin row lists
    int h_start[NB_SMEM + 2] = {0};
    for (int b = 1; b < NB_SMEM + 2; b++) h_start[b] = h_start[b - 1] + h_bins[b - 1];
    int *d_start = bins + 16, *d_fill = bins + 32;
    cudaMemcpyAsync(d_start, h_start, sizeof(h_start), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d_fill, 0, 16 * sizeof(int), s);
    if (m > 0)
        k_fill_bins<<<nblocks(m, 256), 256, 0, s>>>(row_bin, m, d_fill, d_start, bin_rows);
    int32_t *Tj = ws.get<int32_t>(total_cap + 1);
    Z *Tx = ws.get<Z>(total_cap + 1);
    if (ws.failed) return OUT_OF_MEMORY;
    cudaMemsetAsync(row_cnt, 0, (size_t)(m + 1) * 4, s);
    const int ps = prof_begin("saxpy3_numeric", s);
    launch_hash_bin<SR, 8, 128>(bin_rows + h_start[1], h_bins[1], A, B, M, mask_comp, capv, Tj, Tx, row_cnt, s);
    launch_hash_bin<SR, 32, 512>(bin_rows + h_start[2], h_bins[2], A, B, M, mask_comp, capv, Tj, Tx, row_cnt, s);
    launch_hash_bin<SR, 32, 2048>(bin_rows + h_start[3], h_bins[3], A, B, M, mask_comp, capv, Tj, Tx, row_cnt, s);
    launch_hash_bin<SR, 256, 8192>(bin_rows + h_start[4], h_bins[4], A, B, M, mask_comp, capv, Tj, Tx, row_cnt, s);
    const int heavy = NB_SMEM + 1;
    const int nheavy = h_bins[heavy];
    if (nheavy > 0) {
        const int32_t *hrows = bin_rows + h_start[heavy];
        if constexpr (SR::order_free) {
            // all heavy rows at once, one workspace row each (chunks bound memory)
            int64_t chunk = nheavy;
            int64_t per_row = ncols * (8 + (int64_t)sizeof(Z));
            int64_t budget = (int64_t)4 << 30;
            if (chunk * per_row > budget) chunk = budget / per_row > 0 ? budget / per_row : 1;
            int64_t *flag = ws.get<int64_t>(chunk * ncols);
            Z *val = ws.get<Z>(chunk * ncols);
            if (ws.failed) return OUT_OF_MEMORY;
            for (int64_t c0 = 0; c0 < nheavy; c0 += chunk) {
                int nr = (int)((nheavy - c0 < chunk) ? nheavy - c0 : chunk);
                dim3 g1(nblocks(ncols, 256, 4), nr > 65535 ? 65535 : nr);
                k_dense_init<SR><<<g1, 256, 0, s>>>(hrows + c0, nr, ncols, flag, val);
                if (M) {
                    dim3 g2(8, nr > 65535 ? 65535 : nr);
                    k_dense_mask<<<g2, 256, 0, s>>>(hrows + c0, nr, M->p, M->j, mask_comp, ncols, flag);
                }
                dim3 g3((unsigned)runtime().num_sms * 8 / (nr < 8 ? nr : 8) + 1, nr > 65535 ? 65535 : nr);
                k_dense_atomic<SR><<<g3, 256, 0, s>>>(hrows + c0, nr, A.p, A.j, A.x, A.iso,
                    B.p, B.j, B.x, B.iso, M != nullptr, mask_comp, ncols, flag, val);
                k_dense_gather<SR><<<nr < 1024 ? nr : 1024, 256, 0, s>>>(hrows + c0, nr, ncols,
                    flag, val, capv, Tj, Tx, row_cnt);
            }
        } else {
            int nb = nheavy < runtime().num_sms * 2 ? nheavy : runtime().num_sms * 2;
            int64_t *flag = ws.get<int64_t>((int64_t)nb * ncols);
            Z *val = ws.get<Z>((int64_t)nb * ncols);
            if (ws.failed) return OUT_OF_MEMORY;
            cudaMemsetAsync(flag, 0, (size_t)nb * ncols * 8, s);
            k_saxpy_dense_seq<SR><<<nb, 256, 0, s>>>(hrows, nheavy, A.p, A.j, A.x, A.iso,
                B.p, B.j, B.x, B.iso, M ? M->p : nullptr, M ? M->j : nullptr,
                M != nullptr, mask_comp, ncols, flag, val, capv, Tj, Tx, row_cnt);
        }
    }
    prof_end(ps, s);
    // exact row counts -> C row pointers
    int64_t *Cp64 = ws.get<int64_t>(m + 1);
    if (ws.failed) return OUT_OF_MEMORY;
    if (m > 0) k_cnt_to_i64<<<nblocks(m, 256), 256, 0, s>>>(row_cnt, row_bin, m, Cp64);
    cudaMemsetAsync(Cp64 + m, 0, 8, s);
    info = scan_exclusive_i64(Cp64, Cp64, m + 1, s);
    if (info != SUCCESS) return info;
    int64_t nnz = 0;
    cudaMemcpyAsync(&nnz, Cp64 + m, 8, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_to_info(e);
    if (nnz >= INT32_MAX) return OUT_OF_MEMORY;
    C.nrows = m; C.ncols = ncols; C.nnz = nnz; C.iso = false; C.nzombies = 0;
    C.p = (int32_t *)dalloc((size_t)(m + 1) * 4, s);
    C.j = (int32_t *)dalloc((size_t)(nnz ? nnz : 1) * 4, s);
    C.x = dalloc((size_t)(nnz ? nnz : 1) * sizeof(Z), s);
    if (!C.p || !C.j || !C.x) { dev_free(C, s); return OUT_OF_MEMORY; }
    k_i64_to_i32_p<<<nblocks(m + 1, 256), 256, 0, s>>>(Cp64, C.p, m + 1);
    if (m > 0 && nnz > 0)
        k_pack<Z><<<nblocks(m * 32, 256), 256, 0, s>>>(m, capv, Tj, Tx, row_cnt,
            Cp64, C.j, (Z *)C.x);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { dev_free(C, s); return cuda_to_info(e); }
    return SUCCESS;
}

int saxpy3(DevCSR &C, const DevCSR *M, bool mask_comp, bool mask_struct,
           const DevCSR &A, const DevCSR &B, SemiringCode sr, cudaStream_t s)
{
    if (A.ncols != B.nrows) return DIMENSION_MISMATCH;
    if (M && (M->nrows != A.nrows || M->ncols != B.ncols)) return DIMENSION_MISMATCH;
    DevCSR Ms;
    bool own_mask = false;
    if (M && !mask_struct && M->x) {
        // a valued mask is reduced to its true entries first
        int info = dev_mask_to_struct(Ms, *M, s);
        if (info != SUCCESS) return info;
        M = &Ms;
        own_mask = true;
    }
    struct Guard { DevCSR *m; bool own; cudaStream_t s;
        ~Guard() { if (own) dev_free(*m, s); } } guard{&Ms, own_mask, s};
#define GRB_SAXPY_CASE(ADD, MULT, TC, CT)                                      \
    if (sr.add == ADD && sr.mult == MULT && sr.type == TC) {                   \
        int info = saxpy3_t<Semiring<ADD, MULT, CT>>(C, M, mask_comp, A, B, s); \
        if (info == SUCCESS) C.type = TC;                                      \
        return info;                                                           \
    }
    GRB_FOR_EACH_SEMIRING(GRB_SAXPY_CASE)
#undef GRB_SAXPY_CASE
    return NO_VALUE;
}

}  // namespace grb
