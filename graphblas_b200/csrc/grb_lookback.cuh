// grb_lookback.cuh: single-pass exclusive scan with decoupled look-back,
// shared by the kernels that need a scan in one launch.  A `Load` functor
// supplies value i (0 <= i < n), so a scan can read its values from any
// layout (int64 counts, int32 counts under a row filter, B-row lengths
// gathered through A's column indices...).
//
// Tiles of LB_TILE values take their index from a ticket, so a tile's
// predecessors are always running or done.  A tile scans its values, posts
// its sum (flag 1) - or, for tile 0, its inclusive prefix (flag 2) - in a
// 64-bit word (flag << 62 | value); warp 0 then reads 32 predecessors' words
// at a time until it meets an inclusive prefix, and the tile posts its own.
// Waits are bounded: a tile that polls past the limit sets *err and stops
// looking back (the caller fails the call).  The last tile to finish (a
// completion counter) clears the words and both counters, so the workspace
// (lb_ws_elems(n) words, zero before its first use) is ready for the next
// scan without a memset.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace grb {

static constexpr int LB_THREADS = 256;
static constexpr int LB_ROWS = 8;
static constexpr int LB_TILE = LB_THREADS * LB_ROWS;
static constexpr unsigned long long LB_AGG = 1ull << 62, LB_INC = 2ull << 62;
static constexpr unsigned long long LB_VAL = (1ull << 62) - 1;
static constexpr int LB_SPIN_LIMIT = 1 << 22;
static constexpr int LB_TIGHT_SPINS = 64;   // polls before backing off

inline size_t lb_ws_elems(int64_t n) { return (size_t)((n + LB_TILE - 1) / LB_TILE) + 2; }

// Warp 0 finds the sum of every value before the tile: it reads the words of
// 32 predecessors at once, and once the nearest inclusive prefix in the
// window and every word above it are posted, adds them; otherwise it moves
// the window 32 tiles down.  Returns the exclusive prefix (lane 0's value).
// The words may be interleaved: tile t's word is status[t * stride + v].
static __device__ __forceinline__ long long lb_lookback(unsigned long long *status,
                                                       int64_t tile, int lane, int *err,
                                                       int stride = 1, int v = 0)
{
    long long ex = 0;
    int64_t hi = tile - 1;
    int spins = 0;
    while (true) {
        const int64_t idx = hi - (31 - lane);
        unsigned long long w = LB_INC;
        if (idx >= 0)
            w = *reinterpret_cast<volatile unsigned long long *>(&status[idx * stride + v]);
        const unsigned long long f = w & ~LB_VAL;
        const unsigned inc = __ballot_sync(0xffffffffu, f == LB_INC);
        const unsigned pending = __ballot_sync(0xffffffffu, f == 0);
        const int top = inc ? 31 - __clz(inc) : 0;
        const unsigned need = 0xffffffffu << top;
        if (pending & need) {
            if (++spins > LB_SPIN_LIMIT) {
                if (err && lane == 0) atomicExch(err, 1);
                return ex;
            }
            if (spins > LB_TIGHT_SPINS) __nanosleep(64);
            continue;
        }
        long long v = lane >= top ? (long long)(w & LB_VAL) : 0;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        ex += v;
        if (inc) return ex;
        hi -= 32;
    }
}

template <class Load>
__global__ void __launch_bounds__(LB_THREADS)
k_scan_lookback(Load load, int64_t *out, int64_t n, unsigned long long *__restrict__ ws,
                int64_t *__restrict__ total, int32_t *__restrict__ out32,
                int *__restrict__ err)
{
    __shared__ int s_tile, s_last;
    __shared__ long long s_ex;
    __shared__ int64_t warp_sums[LB_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long *status = ws + 2;
    if (tid == 0) s_tile = (int)atomicAdd(&ws[0], 1ull);
    __syncthreads();
    const int64_t tile = s_tile;
    const int64_t ntiles = (n + LB_TILE - 1) / LB_TILE;
    // a warp owns 256 consecutive values as 8 rows of 32 (coalesced)
    const int64_t base = tile * LB_TILE + (int64_t)warp * (32 * LB_ROWS) + lane;
    int64_t v[LB_ROWS];
    #pragma unroll
    for (int r = 0; r < LB_ROWS; r++) {
        const int64_t idx = base + r * 32;
        v[r] = idx < n ? load(idx) : 0;
    }
    int64_t run = 0;
    #pragma unroll
    for (int r = 0; r < LB_ROWS; r++) {
        int64_t x = v[r];
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        v[r] = run + x - v[r];
        run += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) warp_sums[warp] = run;
    __syncthreads();
    if (warp == 0) {
        // exclusive prefix of the eight warp sums, and the tile's sum
        int64_t x = lane < LB_THREADS / 32 ? warp_sums[lane] : 0;
        const int64_t own = x;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const int64_t agg = __shfl_sync(0xffffffffu, x, 31);
        if (lane < LB_THREADS / 32) warp_sums[lane] = x - own;
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
            if (total && tile == ntiles - 1) *total = ex + agg;
        }
    }
    __syncthreads();
    const int64_t wbase = s_ex + warp_sums[warp];
    #pragma unroll
    for (int r = 0; r < LB_ROWS; r++) {
        const int64_t idx = base + r * 32;
        if (idx < n) {
            const int64_t o = wbase + v[r];
            out[idx] = o;
            if (out32) out32[idx] = (int32_t)o;
        }
    }
    // the last tile to finish its look-back clears the workspace
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(&ws[1], 1ull) == (unsigned long long)(ntiles - 1);
    }
    __syncthreads();
    if (s_last) {
        for (int64_t t = tid; t < ntiles; t += LB_THREADS) status[t] = 0;
        if (tid == 0) { ws[0] = 0; ws[1] = 0; }
    }
}

// one launch: out[i] = value 0 + ... + value i-1 for i < n; *total (may be
// null) = the sum of all n; out32 (may be null) the same narrowed to int32
template <class Load>
inline void lb_scan(Load load, int64_t *out, int64_t n, unsigned long long *ws, cudaStream_t s,
                    int64_t *total, int32_t *out32, int *err)
{
    if (n <= 0) return;
    const int64_t ntiles = (n + LB_TILE - 1) / LB_TILE;
    k_scan_lookback<Load><<<(unsigned)ntiles, LB_THREADS, 0, s>>>(load, out, n, ws, total,
                                                                 out32, err);
}

}  // namespace grb
