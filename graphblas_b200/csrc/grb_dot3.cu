// grb_dot3.cu: masked dot-product SpGEMM, C<M> = A*B' (C(i,j) = A(i,:).B(j,:)
// for every (i,j) in the pattern of M), the B200 replacement of the
// reference's GB_AxB_dot3 (Source/mxm/GB_AxB_dot3.c:37) and of its draft GPU
// kernels (CUDA/template/GB_cuda_jit_AxB_dot3_phase{1,2,3_vsvs,3_mp}.cuh).
//
// Two launches, no host round trip between them:
//
//  1. classify (one warp per 32 consecutive mask entries, flat over M): each
//     lane takes one entry (i,j), trims A(i,:) and B(j,:) to their overlap
//     [max(first), min(last)] with binary searches (the reference trims when
//     one list is much longer, GB_AxB_dot_cij.c:538-617), turns an empty
//     overlap into a zombie at once and merges a short overlap itself (the
//     reference's VSVS bucket, phase3_vsvs.cuh:133).  Long overlaps go to a
//     global work queue (warp-aggregated append).
//  2. intersect (persistent warps pull queue entries in batches): one warp
//     per entry.  Balanced lists are merged with a register merge-path: each
//     step loads 32 elements of each list (coalesced), every lane locates its
//     B element in the A window by a 5-step shuffle binary search, and the
//     window that ends first advances.  Lopsided lists (the long one about
//     log2(n) times longer or more) are intersected by taking 32 elements of
//     the short list at a time and binary-searching each in the long one, the
//     search window advancing chunk by chunk.  The queue spreads R-MAT's
//     heavy entries over every warp of the GPU.
//
// Counting semirings (PLUS_PAIR on integers: triangle and support counts)
// on masks of 65536+ entries take a third route for most queued entries:
// entries sharing their longer list (row i of A, or row j of B) form a
// group, the shared row is loaded once into a shared-memory bitmap (key rows
// over 256 entries, one block per SM) or a per-warp hash table (shorter key
// rows), and every entry's other list is probed against it; the count of
// hits is C(i,j).  Entries of small groups, and rows too wide for the
// bitmap, stay on the merge path above.
//
// Matches come out of __ballot_sync in ascending k, so order-dependent
// monoids (floating PLUS/TIMES, ANY) fold them in exactly the reference's
// sequential order, first match assigned and later ones added
// (GB_AxB_dot_cij.c:516-652); order-free monoids keep per-lane partials and
// finish with a warp reduction.  ANY is terminal: the first match ends the
// dot product.  Empty results are zombies, Cj[p] = flip(j) (GB_zombie.h:37),
// counted in C.nzombies; C keeps M's row pointers, as the reference's dot3
// does (GB_AxB_dot3.c:172-197).

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include "../../include/grb_b200.h"
#include "grb_runtime.h"
#include "grb_semirings.h"
#include "grb_lookback.cuh"

namespace grb {

static constexpr int D3_SMALL = 64;        // per-lane merge threshold (nA+nB)
static constexpr int D3_BATCH = 8;         // queue entries taken per grab

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

// counting semirings: PLUS_PAIR on integers (C(i,j) = |A(i,:) and B(j,:)|)
template <class SR> struct IsCount {
    static constexpr bool value = SR::add_op == OP_PLUS && SR::mult_op == OP_PAIR &&
        std::is_integral<typename SR::z_t>::value &&
        !std::is_same<typename SR::z_t, bool>::value;
};

// queued entry: mask position, row, column, trimmed ranges (absolute)
struct __align__(32) D3Work { int32_t pm, i, j, a0, a1, b0, b1, pad; };

// ---------------------------------------------------------------------------
// launch 1: classify
// ---------------------------------------------------------------------------

template <class SR>
__global__ void __launch_bounds__(256)
k_dot3_classify(const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
                const void *__restrict__ Mx, int mtype, bool mask_struct,
                int64_t mnz, int64_t nrows,
                const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
                const void *__restrict__ Ax, bool a_iso,
                const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
                const void *__restrict__ Bx, bool b_iso,
                int32_t *__restrict__ Cj, typename SR::z_t *__restrict__ Cx,
                D3Work *__restrict__ queue, int *__restrict__ qlen,
                unsigned long long *__restrict__ nzombies,
                unsigned long long *__restrict__ out_sum)
{
    using Z = typename SR::z_t;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long zcount = 0, lsum = 0;
    for (int64_t base = warp * 32; base < mnz; base += nwarps * 32) {
        const int64_t pm = base + lane;
        const bool valid = pm < mnz;
        // row of the chunk's first entry (the last r with Mp[r] <= base,
        // searched by the whole warp), then each lane walks forward
        const int32_t r0 = warp_last_le<int32_t, int32_t>(Mp, (int32_t)nrows, (int32_t)base,
                                                          lane);
        int32_t i = r0;
        if (valid) while (Mp[i + 1] <= pm) i++;
        int32_t j = 0, a0 = 0, a1 = 0, b0 = 0, b1 = 0;
        bool coop = false, exists = false;
        Z cij = Z();
        if (valid) {
            j = Mj[pm];
            const bool mval = mask_struct || Mx == nullptr || mask_value_true(Mx, mtype, pm);
            const int32_t pa0 = Ap[i], pa1 = Ap[i + 1];
            const int32_t pb0 = Bp[j], pb1 = Bp[j + 1];
            if (mval && pa1 > pa0 && pb1 > pb0) {
                const int32_t blo = Bj[pb0], bhi = Bj[pb1 - 1];
                a0 = lower_bound(Aj, pa0, pa1, blo);
                a1 = upper_bound(Aj, a0, pa1, bhi);
                if (a1 > a0) {
                    const int32_t alo = Aj[a0], ahi = Aj[a1 - 1];
                    b0 = lower_bound(Bj, pb0, pb1, alo);
                    b1 = upper_bound(Bj, b0, pb1, ahi);
                    if (b1 > b0) {
                        if ((a1 - a0) + (b1 - b0) <= D3_SMALL) {
                            int32_t a = a0, b = b0;
                            while (a < a1 && b < b1) {
                                const int32_t ka = Aj[a], kb = Bj[b];
                                if (ka < kb) a++;
                                else if (kb < ka) b++;
                                else {
                                    Z av = Z(), bv = Z();
                                    if (SR::needs_a) av = ld_val<Z>(Ax, a, a_iso);
                                    if (SR::needs_b) bv = ld_val<Z>(Bx, b, b_iso);
                                    const Z t = SR::F::f(av, bv, i, ka, j);
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
            if (!coop) {
                if (exists) {
                    Cj[pm] = j; Cx[pm] = cij;
                    if constexpr (IsCount<SR>::value) lsum += (unsigned long long)cij;
                } else {
                    Cj[pm] = flip(j); zcount++;
                }
            }
        }
        // warp-aggregated append of the long entries
        const unsigned q = __ballot_sync(0xffffffffu, coop);
        if (q) {
            int qbase = 0;
            if (lane == 0) qbase = atomicAdd(qlen, __popc(q));
            qbase = __shfl_sync(0xffffffffu, qbase, 0);
            if (coop) {
                const int slot = qbase + __popc(q & ((1u << lane) - 1));
                queue[slot] = D3Work{(int32_t)pm, i, j, a0, a1, b0, b1, 0};
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        zcount += __shfl_down_sync(0xffffffffu, zcount, o);
        lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    }
    if (lane == 0 && zcount) atomicAdd(nzombies, zcount);
    if (lane == 0 && lsum && out_sum) atomicAdd(out_sum, lsum);
}

// ---------------------------------------------------------------------------
// launch 2: warp-cooperative intersections of the queued entries
// ---------------------------------------------------------------------------

// fold the matches flagged in `mm` (lane order = ascending k) into the result
template <class SR>
__device__ __forceinline__ void fold_matches(unsigned mm, bool match,
                                             typename SR::z_t t,
                                             Part<typename SR::z_t> &part,
                                             typename SR::z_t &acc, bool &acc_has)
{
    using Z = typename SR::z_t;
    if (SR::order_free && !SR::M::any) {
        if (match) part = combine<SR>(part, Part<Z>{t, true});
    } else {
        while (mm) {
            const int b = __ffs(mm) - 1;
            mm &= mm - 1;
            const Z tv = shfl<Z>(t, b);
            if (!acc_has) { acc = tv; acc_has = true; }
            else acc = SR::M::add(acc, tv);
            if (SR::M::any) break;
        }
    }
}

template <class SR>
__global__ void __launch_bounds__(256)
k_dot3_intersect(const D3Work *__restrict__ queue, const int32_t *__restrict__ sel,
                 const int *__restrict__ qlen_p, int *__restrict__ qnext,
                 const int32_t *__restrict__ Aj, const void *__restrict__ Ax, bool a_iso,
                 const int32_t *__restrict__ Bj, const void *__restrict__ Bx, bool b_iso,
                 int32_t *__restrict__ Cj, typename SR::z_t *__restrict__ Cx,
                 unsigned long long *__restrict__ nzombies,
                 unsigned long long *__restrict__ out_sum)
{
    using Z = typename SR::z_t;
    const int lane = threadIdx.x & 31;
    const int qlen = *qlen_p;
    unsigned long long zcount = 0, lsum = 0;
    while (true) {
        int w0 = 0;
        if (lane == 0) w0 = atomicAdd(qnext, D3_BATCH);
        w0 = __shfl_sync(0xffffffffu, w0, 0);
        if (w0 >= qlen) break;
        const int w1 = min(w0 + D3_BATCH, qlen);
        for (int w = w0; w < w1; w++) {
            const D3Work e = queue[sel ? sel[w] : w];
            const int32_t nA = e.a1 - e.a0, nB = e.b1 - e.b0;
            const int32_t nS = nA < nB ? nA : nB, nL = nA < nB ? nB : nA;
            Part<Z> part{Z(), false};
            Z acc = Z();
            bool acc_has = false;
            // lopsided: search the short list's elements in the long list
            const int lg = 32 - __clz(nL);
            const bool probe = (int64_t)nS * (lg + 2) < (int64_t)(nA + nB);
            if (probe) {
                const bool shortA = nA <= nB;
                const int32_t *S = shortA ? Aj : Bj;
                const int32_t *Lg = shortA ? Bj : Aj;
                const int32_t s0 = shortA ? e.a0 : e.b0, s1 = shortA ? e.a1 : e.b1;
                int32_t lo = shortA ? e.b0 : e.a0;
                const int32_t hi = shortA ? e.b1 : e.a1;
                for (int32_t c0 = s0; c0 < s1; c0 += 32) {
                    const int32_t sp = c0 + lane;
                    const bool has = sp < s1;
                    const int32_t key = has ? S[sp] : INT32_MAX;
                    const int32_t pos = lower_bound(Lg, lo, hi, key);
                    const bool match = has && pos < hi && Lg[pos] == key;
                    Z t = Z();
                    if (match) {
                        const int32_t apos = shortA ? sp : pos;
                        const int32_t bpos = shortA ? pos : sp;
                        Z av = Z(), bv = Z();
                        if (SR::needs_a) av = ld_val<Z>(Ax, apos, a_iso);
                        if (SR::needs_b) bv = ld_val<Z>(Bx, bpos, b_iso);
                        t = SR::F::f(av, bv, e.i, key, e.j);
                    }
                    fold_matches<SR>(__ballot_sync(0xffffffffu, match), match, t,
                                     part, acc, acc_has);
                    if (SR::M::any && acc_has) break;
                    lo = __shfl_sync(0xffffffffu, pos, 31);
                    if (lo >= hi) break;
                }
            } else {
                // register merge-path over 32-element windows of both lists
                int32_t a = e.a0, b = e.b0;
                while (a < e.a1 && b < e.b1) {
                    const int32_t ka = (a + lane < e.a1) ? Aj[a + lane] : INT32_MAX;
                    const int32_t kb = (b + lane < e.b1) ? Bj[b + lane] : INT32_MAX;
                    const int32_t alast = min(e.a1 - a, 32) - 1;
                    const int32_t blast = min(e.b1 - b, 32) - 1;
                    const int32_t amx = __shfl_sync(0xffffffffu, ka, alast);
                    const int32_t bmx = __shfl_sync(0xffffffffu, kb, blast);
                    // locate kb in the A window (5-step shuffle binary search:
                    // lo ends at the first lane whose ka >= kb, or 31)
                    int lo = 0;
                    #pragma unroll
                    for (int step = 16; step > 0; step >>= 1) {
                        const int32_t v = __shfl_sync(0xffffffffu, ka, lo + step - 1);
                        if (v < kb) lo += step;
                    }
                    const int32_t vlo = __shfl_sync(0xffffffffu, ka, lo);
                    // this window decides every B element up to its last A element
                    const bool match = (lane <= blast) && kb <= amx && vlo == kb;
                    Z t = Z();
                    if (match) {
                        Z av = Z(), bv = Z();
                        if (SR::needs_a) av = ld_val<Z>(Ax, a + lo, a_iso);
                        if (SR::needs_b) bv = ld_val<Z>(Bx, b + lane, b_iso);
                        t = SR::F::f(av, bv, e.i, kb, e.j);
                    }
                    fold_matches<SR>(__ballot_sync(0xffffffffu, match), match, t,
                                     part, acc, acc_has);
                    if (SR::M::any && acc_has) break;
                    if (amx < bmx) {
                        // the A window is used up; B elements <= amx are decided
                        const unsigned done = __ballot_sync(0xffffffffu, lane <= blast && kb <= amx);
                        a += alast + 1;
                        b += __popc(done);
                    } else if (bmx < amx) {
                        // every B element is decided; A elements <= bmx are spent
                        const unsigned done = __ballot_sync(0xffffffffu, lane <= alast && ka <= bmx);
                        b += blast + 1;
                        a += __popc(done);
                    } else {
                        a += alast + 1;
                        b += blast + 1;
                    }
                }
            }
            if (SR::order_free && !SR::M::any) {
                for (int o = 16; o > 0; o >>= 1) {
                    Part<Z> other;
                    other.v = shfl_down<Z>(part.v, o);
                    other.has = shfl_down<bool>(part.has, o);
                    part = combine<SR>(part, other);
                }
                acc = part.v;
                acc_has = part.has;
            }
            if (lane == 0) {
                if (acc_has) {
                    Cj[e.pm] = e.j; Cx[e.pm] = acc;
                    if constexpr (IsCount<SR>::value) lsum += (unsigned long long)acc;
                } else {
                    Cj[e.pm] = flip(e.j); zcount++;
                }
            }
        }
    }
    if (lane == 0 && zcount) atomicAdd(nzombies, zcount);
    if (lane == 0 && lsum && out_sum) atomicAdd(out_sum, lsum);
}

// ---------------------------------------------------------------------------
// counting path: PLUS_PAIR on integers (triangle and support counts)
//
// C(i,j) is the number of columns A(i,:) and B(j,:) share.  Every live entry
// is intersected by probing the elements of one of its two lists in a
// shared-memory structure built from the other, its "key" row, and the
// entries sharing a key row form a group that builds the structure once:
//
//   classify  one lane per mask entry: the longer of A(i,:) and B(j,:) (by
//             row length) becomes the key - row i of A (key i) or row j of B
//             (key nrows + j) - and the other list is trimmed to the key
//             row's first and last columns by binary searches; an empty list
//             or an empty trimmed remainder is a zombie at once.  The entry
//             takes a rank in its group, counted apart for long lists
//             (CT_LONG elements or more) and short ones, and queue[pm] holds
//             the key, the rank and the trimmed range.
//   plan      one single-pass scan (decoupled look-back) over the keys: bucket
//             offsets of every group, and work items of about CT_WORK_*
//             probes for every non-empty group - key rows longer than
//             CT_BM_KEY for the block-bitmap kernel, the others for the
//             warp-hash kernel.
//   route     every grouped entry to its bucket, long lists at the front and
//             short ones at the back, so that an item ends on short lists;
//             entries whose key row spans more columns than the bitmap holds
//             go to the merge kernel above.
//   hash      one warp per item: the key row in the warp's table of 4-slot
//             buckets in shared memory.
//   bitmap    one 1024-thread block per SM: the key row as a shared-memory
//             bitmap over its column span.
//
// Inside an item the warps take the long lists (CT_LONG elements or more)
// one at a time, each probed by the whole warp, then the short lists 32 at a
// time, probed flat (their elements end to end, one per lane); a lane keeps
// four 16-byte or scalar loads in flight.  The hit count is C(i,j); its sum
// over the live entries and the zombie count come back with the
// call, so a following sum reduction of C needs no pass.
// ---------------------------------------------------------------------------

static constexpr int CT_BM_KEY = 512;        // longer key rows: block bitmap
static constexpr int CT_H_BUCKETS = 256;     // 4-slot buckets of a warp's hash table
static constexpr int CT_H_WARPS = 8;         // warps (tables) per hash block
static constexpr int CT_BM_THREADS = 1024;
static constexpr int CT_ITEM_BM = 2048;      // entries per bitmap item, at most
static constexpr int CT_ITEM_H = 1024;       // entries per hash item, at most
static constexpr int64_t CT_WORK_BM = 1 << 20;   // probes per bitmap item, about
static constexpr int64_t CT_WORK_H = 1 << 14;    // probes per hash item, about
static constexpr int CT_PER_LANE = 16;       // list elements per lane of a lane group
static constexpr int CT_LONG = 256;          // lists this long go to the front of a bucket
static constexpr int CT_TILE_T = 256;        // plan: threads per tile
static constexpr int CT_TILE_K = 8;          // plan: keys per thread
static constexpr int CT_TILE = CT_TILE_T * CT_TILE_K;
static constexpr int CT_MERGE = -2;          // queue key of an entry for the merge kernel
static constexpr int64_t CT_MIN_ENTRIES = 1024;

// per mask entry: group key (-1: done, CT_MERGE: merge kernel), rank among
// the group's long (rank >= 0) or short (rank < 0: -rank-1) lists, and the
// trimmed probed range [q0, q0 + len)
struct __align__(16) CtQ { int32_t key, rank, q0, len; };
// a grouped entry in its group's bucket
struct __align__(16) CtRec { int32_t q0, len, pm, j; };
// a work item: bucket entries [e0, e1) of key's group, the long lists first
// ([e0, el)); the key row's offsets and its first and last column
struct __align__(16) CtItem { int32_t key, e0, e1, rp0, rp1, klo, khi, el; };

// totals[] written by the plan kernel and read by the count kernels
enum { CT_N_BM = 0, CT_N_H = 1, CT_N_BUCKET = 2, CT_ERR = 3 };

template <class SR>
__global__ void __launch_bounds__(256)
k_ct_classify(const int32_t *__restrict__ Mp, const int32_t *__restrict__ Mj,
              const void *__restrict__ Mx, int mtype, bool mask_struct,
              int64_t mnz, int64_t nrows,
              const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
              const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
              uint32_t bm_bits, bool spans_fit,
              int32_t *__restrict__ Cj, CtQ *__restrict__ queue,
              int32_t *__restrict__ gcnt, unsigned long long *__restrict__ gwork,
              unsigned long long *__restrict__ nzombies)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long zcount = 0;
    for (int64_t base = warp * 32; base < mnz; base += nwarps * 32) {
        const int64_t pm = base + lane;
        const bool valid = pm < mnz;
        const int32_t r0 = warp_last_le<int32_t, int32_t>(Mp, (int32_t)nrows, (int32_t)base,
                                                          lane);
        int32_t i = r0;
        if (valid) while (Mp[i + 1] <= pm) i++;
        int32_t key = -1, q0 = 0, q1 = 0;
        if (valid) {
            const int32_t j = Mj[pm];
            const bool mval = mask_struct || Mx == nullptr || mask_value_true(Mx, mtype, pm);
            const int32_t pa0 = Ap[i], pa1 = Ap[i + 1];
            const int32_t pb0 = Bp[j], pb1 = Bp[j + 1];
            if (mval && pa1 > pa0 && pb1 > pb0) {
                const bool akey = pa1 - pa0 > pb1 - pb0;
                const int32_t *K = akey ? Aj : Bj;
                const int32_t *S = akey ? Bj : Aj;
                const int32_t k0 = akey ? pa0 : pb0, k1 = akey ? pa1 : pb1;
                q0 = akey ? pb0 : pa0;
                q1 = akey ? pb1 : pa1;
                const int32_t klo = K[k0], khi = K[k1 - 1];
                const int32_t first = S[q0], last = S[q1 - 1];
                if (first < klo) q0 = lower_bound(S, q0 + 1, q1, klo);
                if (last > khi && q0 < q1) q1 = upper_bound(S, q0, q1 - 1, khi);
                if (q1 > q0) {
                    key = akey ? i : (int32_t)nrows + j;
                    if (!spans_fit && k1 - k0 > CT_BM_KEY && (uint32_t)(khi - klo) >= bm_bits)
                        key = CT_MERGE;
                }
            }
            if (key == -1) {
                Cj[pm] = flip(j);
                zcount++;
            }
        }
        // rank among the group's long or short lists, and the group's probe
        // work (to size its items): one atomic each per distinct key and
        // kind of the warp
        int32_t rank = 0;
        const bool grouped = key >= 0;
        const int len = q1 - q0;
        const bool lng = len >= CT_LONG;
        const int slot = grouped ? 2 * key + (lng ? 0 : 1) : 0;
        const unsigned gm = __ballot_sync(0xffffffffu, grouped);
        if (grouped) {
            const unsigned same = __match_any_sync(gm, slot);
            const int leader = __ffs(same) - 1;
            const unsigned w = __reduce_add_sync(same, (unsigned)min(len, 1 << 20));
            int32_t b = 0;
            if (lane == leader) {
                b = atomicAdd(&gcnt[slot], __popc(same));
                atomicAdd(&gwork[key], (unsigned long long)w);
            }
            b = __shfl_sync(same, b, leader);
            rank = b + __popc(same & ((1u << lane) - 1));
            if (!lng) rank = -rank - 1;
        }
        if (valid) queue[pm] = CtQ{key, rank, q0, len};
    }
    for (int o = 16; o > 0; o >>= 1) zcount += __shfl_down_sync(0xffffffffu, zcount, o);
    if (lane == 0 && zcount) atomicAdd(nzombies, zcount);
}

// ---- plan: single-pass scan over the keys -------------------------------

// A tile publishes its three sums (item counts for the two kernels, bucket
// entries) as 64-bit words (flag << 62 | value): flag 1 = the tile's own
// sum, 2 = the sum of every tile up to and including it.  A tile waits for
// its predecessors' words with a bounded number of polls; if the bound is
// reached the error flag is set and the call fails.
static constexpr unsigned long long CT_FLAG_AGG = 1ull << 62, CT_FLAG_INC = 2ull << 62;
static constexpr unsigned long long CT_VAL = (1ull << 62) - 1;

// A group's entries c (long and short), its bucket share and its items:
// about CT_WORK_* probes each, at most CT_ITEM_* entries each, at least 16
// entries each.
__device__ __forceinline__ void ct_key_plan(const int32_t *__restrict__ gcnt,
                                            const unsigned long long *__restrict__ gwork,
                                            int64_t t, int64_t nkeys, int32_t nrows,
                                            const int32_t *__restrict__ Ap,
                                            const int32_t *__restrict__ Bp,
                                            int32_t &c, int32_t &nb, int32_t &nh)
{
    c = 0; nb = 0; nh = 0;
    if (t >= nkeys) return;
    c = gcnt[2 * t] + gcnt[2 * t + 1];
    if (c <= 0) return;
    const bool by_row = t < nrows;
    const int32_t r = by_row ? (int32_t)t : (int32_t)(t - nrows);
    const int32_t klen = by_row ? Ap[r + 1] - Ap[r] : Bp[r + 1] - Bp[r];
    const bool big = klen > CT_BM_KEY;
    const int64_t chunk = big ? CT_WORK_BM : CT_WORK_H;
    const int32_t emax = big ? CT_ITEM_BM : CT_ITEM_H;
    int64_t n = ((int64_t)gwork[t] + chunk - 1) / chunk;
    const int64_t nmin = (c + emax - 1) / emax, nmax = c / 16 > nmin ? c / 16 : nmin;
    n = n < nmin ? nmin : (n > nmax ? nmax : n);
    if (big) nb = (int32_t)n; else nh = (int32_t)n;
}

// inclusive scan of three ints across the block (256 threads)
__device__ __forceinline__ void ct_block_scan3(int &a, int &b, int &c, int &ta, int &tb,
                                               int &tc, int (*s_w)[CT_TILE_T / 32])
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int xa = __shfl_up_sync(0xffffffffu, a, o);
        const int xb = __shfl_up_sync(0xffffffffu, b, o);
        const int xc = __shfl_up_sync(0xffffffffu, c, o);
        if (lane >= o) { a += xa; b += xb; c += xc; }
    }
    if (lane == 31) { s_w[0][w] = a; s_w[1][w] = b; s_w[2][w] = c; }
    __syncthreads();
    int pa = 0, pb = 0, pc = 0;
    ta = 0; tb = 0; tc = 0;
    #pragma unroll
    for (int k = 0; k < CT_TILE_T / 32; k++) {
        if (k < w) { pa += s_w[0][k]; pb += s_w[1][k]; pc += s_w[2][k]; }
        ta += s_w[0][k]; tb += s_w[1][k]; tc += s_w[2][k];
    }
    a += pa; b += pb; c += pc;
}

__global__ void __launch_bounds__(CT_TILE_T)
k_ct_plan(const int32_t *__restrict__ gcnt, const unsigned long long *__restrict__ gwork,
          int64_t nkeys, int32_t nrows,
          const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
          const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
          unsigned long long *__restrict__ status, int *__restrict__ tile_ctr,
          int32_t *__restrict__ boff, CtItem *__restrict__ items_bm,
          CtItem *__restrict__ items_h, int32_t *__restrict__ totals)
{
    __shared__ int s_tile;
    __shared__ int s_w[3][CT_TILE_T / 32];
    __shared__ long long s_ex[3];
    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1);
    __syncthreads();
    const int64_t tile = s_tile;
    const int64_t ntiles = (nkeys + CT_TILE - 1) / CT_TILE;
    const int64_t t0 = tile * CT_TILE + (int64_t)tid * CT_TILE_K;
    int sb = 0, sh = 0, sc = 0;
    #pragma unroll
    for (int k = 0; k < CT_TILE_K; k++) {
        int32_t c, nb, nh;
        ct_key_plan(gcnt, gwork, t0 + k, nkeys, nrows, Ap, Bp, c, nb, nh);
        sb += nb; sh += nh; sc += c;
    }
    int ib = sb, ih = sh, ic = sc, tb, th, tc;
    ct_block_scan3(ib, ih, ic, tb, th, tc, s_w);
    if (tid < 32) {
        // warp 0: post the tile's three sums, then look back over 32
        // predecessors at a time for each of them
        const int lane = tid;
        unsigned long long *my = status + tile * 3;
        const unsigned long long agg[3] = {(unsigned long long)tb, (unsigned long long)th,
                                           (unsigned long long)tc};
        long long ex[3] = {0, 0, 0};
        if (tile == 0) {
            if (lane == 0)
                for (int v = 0; v < 3; v++) atomicExch(&my[v], CT_FLAG_INC | agg[v]);
        } else {
            if (lane == 0)
                for (int v = 0; v < 3; v++) atomicExch(&my[v], CT_FLAG_AGG | agg[v]);
            for (int v = 0; v < 3; v++)
                ex[v] = lb_lookback(status, tile, lane, (int *)&totals[CT_ERR], 3, v);
            if (lane == 0)
                for (int v = 0; v < 3; v++)
                    atomicExch(&my[v], CT_FLAG_INC |
                                       ((unsigned long long)(ex[v] + (long long)agg[v]) & CT_VAL));
        }
        if (lane == 0) {
            s_ex[0] = ex[0]; s_ex[1] = ex[1]; s_ex[2] = ex[2];
            if (tile == ntiles - 1) {
                totals[CT_N_BM] = (int32_t)(ex[0] + tb);
                totals[CT_N_H] = (int32_t)(ex[1] + th);
                totals[CT_N_BUCKET] = (int32_t)(ex[2] + tc);
            }
        }
    }
    __syncthreads();
    long long ob = s_ex[0] + ib - sb, oh = s_ex[1] + ih - sh, oc = s_ex[2] + ic - sc;
    #pragma unroll 1
    for (int k = 0; k < CT_TILE_K; k++) {
        const int64_t t = t0 + k;
        int32_t c, nb, nh;
        ct_key_plan(gcnt, gwork, t, nkeys, nrows, Ap, Bp, c, nb, nh);
        if (t < nkeys) boff[t] = (int32_t)oc;
        const int32_t n = nb + nh;
        if (n > 0) {
            const bool by_row = t < nrows;
            const int32_t r = by_row ? (int32_t)t : (int32_t)(t - nrows);
            const int32_t *P = by_row ? Ap : Bp;
            const int32_t *J = by_row ? Aj : Bj;
            const int32_t rp0 = P[r], rp1 = P[r + 1];
            const int32_t klo = J[rp0], khi = J[rp1 - 1];
            CtItem *out = nb ? items_bm + ob : items_h + oh;
            const int64_t lend = oc + gcnt[2 * t];          // end of the long lists
            for (int32_t q = 0; q < n; q++) {
                const int64_t e0 = oc + (int64_t)c * q / n, e1 = oc + (int64_t)c * (q + 1) / n;
                const int64_t el = lend < e0 ? e0 : (lend > e1 ? e1 : lend);
                out[q] = CtItem{(int32_t)t, (int32_t)e0, (int32_t)e1, rp0, rp1, klo, khi,
                                (int32_t)el};
            }
        }
        ob += nb; oh += nh; oc += c;
    }
}

// grouped entries to their buckets (long lists from the front, short ones
// from the back); entries for the merge kernel to its queue
__global__ void __launch_bounds__(256)
k_ct_route(const CtQ *__restrict__ queue, int64_t mnz, int32_t nrows,
           const int32_t *__restrict__ gcnt, const int32_t *__restrict__ boff,
           CtRec *__restrict__ bucket, const int32_t *__restrict__ Mp,
           const int32_t *__restrict__ Mj, const int32_t *__restrict__ Ap,
           const int32_t *__restrict__ Bp, D3Work *__restrict__ mq, int *__restrict__ mq_len)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < mnz; base += nwarps * 32) {
        const int64_t pm = base + lane;
        CtQ q{-1, 0, 0, 0};
        if (pm < mnz) q = queue[pm];
        if (q.key >= 0) {
            const int32_t b0 = boff[q.key];
            const int32_t pos = q.rank >= 0 ? b0 + q.rank
                : b0 + gcnt[2 * q.key] + gcnt[2 * q.key + 1] + q.rank;   // rank = -r-1
            bucket[pos] = CtRec{q.q0, q.len, (int32_t)pm, Mj[pm]};
        }
        const unsigned mm = __ballot_sync(0xffffffffu, q.key == CT_MERGE);
        if (mm) {
            const int32_t r0 = warp_last_le<int32_t, int32_t>(Mp, nrows, (int32_t)base, lane);
            int32_t mb = 0;
            if (lane == 0) mb = atomicAdd(mq_len, __popc(mm));
            mb = __shfl_sync(0xffffffffu, mb, 0);
            if (q.key == CT_MERGE) {
                int32_t i = r0;
                while (Mp[i + 1] <= pm) i++;
                const int32_t j = Mj[pm];
                mq[mb + __popc(mm & ((1u << lane) - 1))] =
                    D3Work{(int32_t)pm, i, j, Ap[i], Ap[i + 1], Bp[j], Bp[j + 1], 0};
            }
        }
    }
}

// ---- probing ------------------------------------------------------------

// The G lanes of a group (lane gl of G, a power of two) count the elements
// of S[q0, q1) for which hit() is 1.  A step covers 16 elements per lane:
// four 16-byte vectors (lane gl takes vectors gl, G + gl, 2G + gl, 3G + gl
// of the step, so each of the four loads is coalesced across the group),
// all loaded before any is probed so that their latencies overlap.  A vector
// that lies inside the range is one 16-byte load when `vec` (S 16-byte
// aligned); a vector at either end is read element by element, and its
// slots outside the range read `none`, a value hit() always misses.
template <class Hit>
__device__ __forceinline__ int ct_count(const int32_t *__restrict__ S, int32_t q0, int32_t q1,
                                        int G, int gl, bool vec, int32_t none, const Hit &hit)
{
    int cnt = 0;
    for (int32_t base = q0 & ~3; base < q1; base += 16 * G) {
        int4 v[4];
        #pragma unroll
        for (int u = 0; u < 4; u++) {
            const int32_t b = base + 4 * (u * G + gl);
            if (vec && b >= q0 && b + 4 <= q1) {
                v[u] = __ldg(reinterpret_cast<const int4 *>(S + b));
            } else {
                v[u].x = (b >= q0 && b < q1) ? S[b] : none;
                v[u].y = (b + 1 >= q0 && b + 1 < q1) ? S[b + 1] : none;
                v[u].z = (b + 2 >= q0 && b + 2 < q1) ? S[b + 2] : none;
                v[u].w = (b + 3 >= q0 && b + 3 < q1) ? S[b + 3] : none;
            }
        }
        #pragma unroll
        for (int u = 0; u < 4; u++)
            cnt += hit(v[u].x) + hit(v[u].y) + hit(v[u].z) + hit(v[u].w);
    }
    return cnt;
}

// write one counted entry: C(i,j) = c, or a zombie when c is 0
template <typename Z>
__device__ __forceinline__ void ct_write(int32_t pm, int32_t j, int c, int32_t *__restrict__ Cj,
                                         Z *__restrict__ Cx, unsigned long long &sum,
                                         unsigned long long &zc)
{
    if (c) { Cj[pm] = j; Cx[pm] = (Z)c; sum += (unsigned long long)c; }
    else { Cj[pm] = flip(j); zc++; }
}

// The bitmap kernel's batches of short lists: up to 32 bucket entries, one
// per lane (valid, trimmed list [q0, q0 + len), output position pm and
// column j), probed by lane groups (a bitmap probe is cheap enough that the
// flat batches' per-window bookkeeping would cost more than idle lanes).  Every entry gets a
// group of 2^lg lanes, about CT_PER_LANE elements of its list per lane (1 to
// 32 lanes).  The groups are packed into lane slots - larger groups first,
// lane order within a size - so that every group starts on a multiple of its
// size, and the warp runs the slots 32 at a time: in each round every lane
// finds its group (the last group start at or below it, from the starts the
// entries' lanes write into the warp's `owner` row) and the groups probe
// side by side.  `owner` holds 32 ints, all -1 between calls.
template <typename Z, class Hit>
__device__ __forceinline__ void ct_batch_packed(bool valid, int32_t q0, int32_t len, int32_t pm,
                                         int32_t j, const int32_t *__restrict__ S, bool vec,
                                         int32_t none, const Hit &hit, int32_t *__restrict__ Cj,
                                         Z *__restrict__ Cx, unsigned long long &sum,
                                         unsigned long long &zc, int *owner)
{
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1;
    int lg = -1;
    if (valid) {
        const int32_t w = len / CT_PER_LANE;
        lg = w >= 32 ? 5 : (w > 1 ? 31 - __clz(w) : 0);
    }
    int32_t start = 0, total = 0;
    #pragma unroll
    for (int c = 5; c >= 0; c--) {
        const unsigned m = __ballot_sync(0xffffffffu, lg == c);
        if (lg == c) start = total + (int32_t)(__popc(m & below) << c);
        total += (int32_t)(__popc(m) << c);
    }
    for (int32_t r0 = 0; r0 < total; r0 += 32) {
        if (lg >= 0 && start >= r0 && start < r0 + 32) owner[start - r0] = lane;
        __syncwarp();
        const int o = owner[lane];
        int v = o >= 0 ? ((lane << 5) | o) : -1;
        #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v = max(v, u);
        }
        __syncwarp();
        if (o >= 0) owner[lane] = -1;
        // every reset lands before any lane writes the next round's starts
        __syncwarp();
        const int src = v & 31, gs = v >> 5;
        const int elg = __shfl_sync(0xffffffffu, lg, src);
        const int32_t eq0 = __shfl_sync(0xffffffffu, q0, src);
        const int32_t elen = __shfl_sync(0xffffffffu, len, src);
        const int32_t epm = __shfl_sync(0xffffffffu, pm, src);
        const int32_t ej = __shfl_sync(0xffffffffu, j, src);
        // lanes past the last group probe an empty range, so every lane
        // takes part in the group sums (xor shuffles stay inside an aligned
        // group of G lanes)
        const bool act = r0 + lane < total;
        const int G = 1 << elg, gl = lane - gs;
        int c = act ? ct_count(S, eq0, eq0 + elen, G, gl, vec, none, hit) : 0;
        #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_xor_sync(0xffffffffu, c, d);
            if (d < G) c += u;
        }
        if (act && gl == 0) ct_write<Z>(epm, ej, c, Cj, Cx, sum, zc);
        __syncwarp();
    }
}

// One batch of up to 32 short lists, one entry per lane (valid, trimmed list
// [q0, q0 + len), output position pm and column j), probed flat: the
// entries' elements are laid end to end and the warp takes windows of 32
// consecutive elements, lane d the d-th of each, four windows per step (four
// loads in flight per lane).  In a window a lane's entry is the window's
// first entry (the last one starting at or before the window, a ballot) plus
// the entries starting between the window's start and the lane (a popcount
// of the OR of their start offsets), so every lane probes in every window
// but the batch's last.  Hits go to the entry's counter in `cnt` (32 ints,
// all zero between calls).
template <typename Z, class Hit>
__device__ __forceinline__ void ct_batch(bool valid, int32_t q0, int32_t len, int32_t pm,
                                         int32_t j, const int32_t *__restrict__ S,
                                         int32_t none, const Hit &hit,
                                         int32_t *__restrict__ Cj, Z *__restrict__ Cx,
                                         unsigned long long &sum, unsigned long long &zc,
                                         int *cnt)
{
    const int lane = threadIdx.x & 31;
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    const int n = __popc(vm);
    if (n == 0) return;
    // the valid entries move to lanes 0 .. n-1, in order
    const int src = lane < n ? (int)__fns(vm, 0, lane + 1) : 0;
    const int32_t eq0 = __shfl_sync(0xffffffffu, q0, src);
    int32_t elen = __shfl_sync(0xffffffffu, len, src);
    const int32_t epm = __shfl_sync(0xffffffffu, pm, src);
    const int32_t ej = __shfl_sync(0xffffffffu, j, src);
    if (lane >= n) elen = 0;
    int32_t inc = elen;
    #pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int32_t u = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += u;
    }
    const int32_t start = inc - elen;
    const int32_t total = __shfl_sync(0xffffffffu, inc, 31);
    const unsigned upto = lane == 31 ? 0xffffffffu : (2u << lane) - 1u;
    for (int32_t f0 = 0; f0 < total; f0 += 128) {
        int32_t x[4];
        int ent[4];
        #pragma unroll
        for (int u = 0; u < 4; u++) {
            const int32_t w0 = f0 + 32 * u;
            const unsigned le = __ballot_sync(0xffffffffu, lane < n && start <= w0);
            const int elo = 31 - __clz(le);
            const bool inside = lane < n && start > w0 && start < w0 + 32;
            const unsigned sm = __reduce_or_sync(0xffffffffu,
                                                 inside ? 1u << (start - w0) : 0u);
            const int e = elo + __popc(sm & upto);
            const int32_t se = __shfl_sync(0xffffffffu, start, e);
            const int32_t qe = __shfl_sync(0xffffffffu, eq0, e);
            const int32_t f = w0 + lane;
            x[u] = f < total ? S[qe + (f - se)] : none;
            ent[u] = e;
        }
        #pragma unroll
        for (int u = 0; u < 4; u++)
            if (hit(x[u])) atomicAdd(&cnt[ent[u]], 1);
    }
    __syncwarp();
    if (lane < n) {
        const int c = cnt[lane];
        cnt[lane] = 0;
        ct_write<Z>(epm, ej, c, Cj, Cx, sum, zc);
    }
    __syncwarp();
}

// one long list by the whole warp: C(i,j) for the bucket entry r
template <typename Z, class Hit>
__device__ __forceinline__ void ct_long_rec(const CtRec &r, const int32_t *__restrict__ S,
                                            bool vec, int32_t none, const Hit &hit,
                                            int32_t *__restrict__ Cj, Z *__restrict__ Cx,
                                            unsigned long long &sum, unsigned long long &zc)
{
    const int lane = threadIdx.x & 31;
    int c = ct_count(S, r.q0, r.q0 + r.len, 32, lane, vec, none, hit);
    c = (int)__reduce_add_sync(0xffffffffu, (unsigned)c);
    if (lane == 0) ct_write<Z>(r.pm, r.j, c, Cj, Cx, sum, zc);
}

// one long list by the whole warp: C(i,j) for the entry in bucket slot e
template <typename Z, class Hit>
__device__ __forceinline__ void ct_long(const CtRec *__restrict__ bucket, int32_t e,
                                        const int32_t *__restrict__ S, bool vec, int32_t none,
                                        const Hit &hit, int32_t *__restrict__ Cj,
                                        Z *__restrict__ Cx, unsigned long long &sum,
                                        unsigned long long &zc)
{
    ct_long_rec<Z>(bucket[e], S, vec, none, hit, Cj, Cx, sum, zc);
}

__device__ __forceinline__ void ct_load_entry(const CtItem &I, int32_t e,
                                              const CtRec *__restrict__ bucket, bool &valid,
                                              int32_t &q0, int32_t &len, int32_t &pm,
                                              int32_t &j)
{
    valid = e < I.e1;
    CtRec r{0, 0, 0, 0};
    if (valid) r = bucket[e];
    q0 = r.q0; len = r.len; pm = r.pm; j = r.j;
}

__device__ __forceinline__ uint32_t ct_hash(int32_t k, int bits)
{
    return ((uint32_t)k * 0x9E3779B1u) >> (32 - bits);
}

// One warp per item whose key row has at most CT_BM_KEY entries.  The key
// row goes into the warp's hash table of 4-slot buckets (a power of two of
// buckets, at least half as many as the row's entries; a bucket's slots fill
// in order, and a full bucket overflows into the next), so most probes read
// one 16-byte bucket: the element is in the row if a slot holds it, absent
// if the bucket still has an empty slot.
template <class SR>
__global__ void __launch_bounds__(CT_H_WARPS * 32)
k_ct_hash(const CtItem *__restrict__ items, const int32_t *__restrict__ totals,
          int *__restrict__ inext, int32_t nrows, const CtRec *__restrict__ bucket,
          const int32_t *__restrict__ Aj, const int32_t *__restrict__ Bj, bool vec,
          int32_t *__restrict__ Cj, typename SR::z_t *__restrict__ Cx,
          unsigned long long *__restrict__ out_sum, unsigned long long *__restrict__ nzombies)
{
    using Z = typename SR::z_t;
    __shared__ int4 s_tab[CT_H_WARPS][CT_H_BUCKETS];
    __shared__ int s_cnt[CT_H_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int4 *tab = s_tab[w];
    int32_t *slots = reinterpret_cast<int32_t *>(tab);
    for (int q = lane; q < CT_H_BUCKETS; q += 32) tab[q] = make_int4(-1, -1, -1, -1);
    s_cnt[w][lane] = 0;
    __syncwarp();
    const int nitems = totals[CT_N_H];
    unsigned long long sum = 0, zc = 0;
    while (true) {
        int it = 0;
        if (lane == 0) it = atomicAdd(inext, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        const CtItem I = items[it];
        const bool by_row = I.key < nrows;
        const int32_t *J = by_row ? Aj : Bj;
        const int32_t *S = by_row ? Bj : Aj;
        const int32_t klen = I.rp1 - I.rp0;
        int bits = 3;
        while ((1 << bits) * 2 < klen) bits++;
        const uint32_t bmask = (1u << bits) - 1;
        for (int32_t q = I.rp0 + lane; q < I.rp1; q += 32) {
            const int32_t k = J[q];
            uint32_t b = ct_hash(k, bits);
            for (int t = 0;; t++) {
                if (atomicCAS(&slots[b * 4 + (t & 3)], -1, k) == -1) break;
                if ((t & 3) == 3) b = (b + 1) & bmask;
            }
        }
        __syncwarp();
        auto hit = [&](int32_t x) -> int {
            uint32_t b = ct_hash(x, bits);
            while (true) {
                const int4 v = tab[b];
                if (v.x == x || v.y == x || v.z == x || v.w == x) return 1;
                if (v.w < 0) return 0;
                b = (b + 1) & bmask;
            }
        };
        // `none` is INT32_MIN: never a column, and not the empty-slot mark
        for (int32_t e = I.e0; e < I.el; e++)
            ct_long<Z>(bucket, e, S, vec, INT32_MIN, hit, Cj, Cx, sum, zc);
        for (int32_t e = I.el; e < I.e1; e += 32) {
            bool valid;
            int32_t q0, len, pm, j;
            ct_load_entry(I, e + lane, bucket, valid, q0, len, pm, j);
            ct_batch<Z>(valid, q0, len, pm, j, S, INT32_MIN, hit, Cj, Cx, sum, zc,
                        s_cnt[w]);
        }
        __syncwarp();
        for (int q = lane; q <= (int)bmask; q += 32) tab[q] = make_int4(-1, -1, -1, -1);
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        zc += __shfl_down_sync(0xffffffffu, zc, o);
    }
    if (lane == 0) {
        if (sum) atomicAdd(out_sum, sum);
        if (zc) atomicAdd(nzombies, zc);
    }
}

// One block per SM, persistent over the items whose key row is longer than
// CT_BM_KEY: the key row's columns (relative to its first) are set as bits
// of a shared-memory bitmap, the warps take the item's entries 32 at a time
// from a shared counter and count them, and the bits are cleared again.
// bm_words words hold the bits; the word after them stays zero and absorbs
// every probe outside the row's span.
template <class SR>
__global__ void __launch_bounds__(CT_BM_THREADS, 1)
k_ct_bitmap(const CtItem *__restrict__ items, const int32_t *__restrict__ totals,
            int *__restrict__ inext, int32_t nrows, const CtRec *__restrict__ bucket,
            const int32_t *__restrict__ Aj, const int32_t *__restrict__ Bj, bool vec,
            uint32_t bm_words, int32_t *__restrict__ Cj, typename SR::z_t *__restrict__ Cx,
            unsigned long long *__restrict__ out_sum, unsigned long long *__restrict__ nzombies)
{
    using Z = typename SR::z_t;
    extern __shared__ __align__(16) uint32_t bm[];
    // the item being processed and the one fetched ahead alternate between
    // two slots, so the fetch never writes the slot the block is reading
    __shared__ int s_item[2], s_next, s_long;
    __shared__ CtItem s_I[2];
    __shared__ int s_cnt[CT_BM_THREADS / 32][32];
    const int tid = threadIdx.x, lane = tid & 31;
    for (uint32_t q = tid; q <= bm_words; q += blockDim.x) bm[q] = 0;
    s_cnt[tid >> 5][lane] = -1;        // the lane groups' owner rows
    const uint32_t nbits = bm_words * 32u;        // the guard bit
    const int nitems = totals[CT_N_BM];
    unsigned long long sum = 0, zc = 0;
    int cur = 0;
    if (tid == 0) {
        s_item[0] = atomicAdd(inext, 1);
        if (s_item[0] < nitems) s_I[0] = items[s_item[0]];
    }
    // every block barrier below follows code in which a warp's lanes may
    // diverge (the lane groups, the strided set and clear loops): each warp
    // reconverges first, as a block barrier must be reached by whole warps
    while (true) {
        __syncwarp();
        __syncthreads();
        if (s_item[cur] >= nitems) break;
        const CtItem I = s_I[cur];
        __syncwarp();
        __syncthreads();
        if (tid == 0) { s_next = 0; s_long = 0; }
        const bool by_row = I.key < nrows;
        const int32_t *J = by_row ? Aj : Bj;
        const int32_t *S = by_row ? Bj : Aj;
        const int32_t klo = I.klo, khi = I.khi;
        {
            const int32_t nt = (int32_t)blockDim.x;
            int32_t q = I.rp0 + tid;
            for (; q + 3 * nt < I.rp1; q += 4 * nt) {
                const uint32_t k0 = (uint32_t)(J[q] - klo), k1 = (uint32_t)(J[q + nt] - klo);
                const uint32_t k2 = (uint32_t)(J[q + 2 * nt] - klo);
                const uint32_t k3 = (uint32_t)(J[q + 3 * nt] - klo);
                atomicOr(&bm[k0 >> 5], 1u << (k0 & 31));
                atomicOr(&bm[k1 >> 5], 1u << (k1 & 31));
                atomicOr(&bm[k2 >> 5], 1u << (k2 & 31));
                atomicOr(&bm[k3 >> 5], 1u << (k3 & 31));
            }
            for (; q < I.rp1; q += nt) {
                const uint32_t k = (uint32_t)(J[q] - klo);
                atomicOr(&bm[k >> 5], 1u << (k & 31));
            }
        }
        __syncwarp();
        __syncthreads();
        // the next item is fetched while this one runs
        if (tid == 0) {
            const int nx = atomicAdd(inext, 1);
            s_item[cur ^ 1] = nx;
            if (nx < nitems) s_I[cur ^ 1] = items[nx];
        }
        // probed ranges lie inside [klo, khi]; `none` maps to the guard bit
        auto hit = [&](int32_t x) -> int {
            const uint32_t k = (uint32_t)(x - klo);
            return (int)((bm[k >> 5] >> (k & 31)) & 1u);
        };
        const int32_t none = klo + (int32_t)nbits;
        // long lists one at a time, each by the whole warp, so that no warp
        // holds many of them (the next list's record is read while the
        // current list is probed); then the short ones 32 at a time
        {
            auto grab = [&]() -> int {
                int e = 0;
                if (lane == 0) e = atomicAdd(&s_long, 1);
                return __shfl_sync(0xffffffffu, e, 0) + I.e0;
            };
            int e = grab();
            CtRec r{0, 0, 0, 0};
            if (e < I.el) r = bucket[e];
            while (e < I.el) {
                const int en = grab();
                CtRec rn{0, 0, 0, 0};
                if (en < I.el) rn = bucket[en];
                ct_long_rec<Z>(r, S, vec, none, hit, Cj, Cx, sum, zc);
                e = en;
                r = rn;
            }
        }
        while (true) {
            int e = 0;
            if (lane == 0) e = atomicAdd(&s_next, 32);
            e = __shfl_sync(0xffffffffu, e, 0) + I.el;
            if (e >= I.e1) break;
            bool valid;
            int32_t q0, len, pm, j;
            ct_load_entry(I, e + lane, bucket, valid, q0, len, pm, j);
            ct_batch_packed<Z>(valid, q0, len, pm, j, S, vec, none, hit, Cj, Cx, sum, zc,
                               s_cnt[tid >> 5]);
        }
        __syncwarp();
        __syncthreads();
        // clear: zero the span's words with 16-byte stores (at most a few
        // per thread, and no global loads)
        {
            const uint32_t span_words = (uint32_t)(khi - klo) / 32u + 1u;
            uint4 *b4 = reinterpret_cast<uint4 *>(bm);
            const uint32_t n4 = (span_words + 3u) / 4u;
            for (uint32_t q = tid; q < n4; q += blockDim.x) b4[q] = make_uint4(0, 0, 0, 0);
        }
        cur ^= 1;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        zc += __shfl_down_sync(0xffffffffu, zc, o);
    }
    if (lane == 0) {
        if (sum) atomicAdd(out_sum, sum);
        if (zc) atomicAdd(nzombies, zc);
    }
}

// Words of the bitmap: enough for every column index when that fits beside
// the kernel's static shared memory (plus the zero guard word, the total a
// multiple of 4 words for the 16-byte clears), else the most that fits (key
// rows spanning more columns go to the merge kernel).  0 disables the
// bitmap (the counting path is then not taken).
template <class SR>
static uint32_t ct_bitmap_words(int64_t ncols)
{
    static int64_t avail = -1;
    if (avail < 0) {
        const void *fn = (const void *)k_ct_bitmap<SR>;
        cudaFuncAttributes fa;
        int64_t a = 0;
        if (cudaFuncGetAttributes(&fa, fn) == cudaSuccess) {
            a = (int64_t)runtime().smem_optin - (int64_t)fa.sharedSizeBytes - 1024;
            if (a < 0 ||
                cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)a) != cudaSuccess)
                a = 0;
        }
        cudaGetLastError();
        avail = a / 4;
    }
    // words for the bits, rounded so that bits + guard is a multiple of 4
    const int64_t need = ((ncols + 31) / 32 + 1 + 3) & ~(int64_t)3;
    const int64_t cap = avail & ~(int64_t)3;
    const int64_t w = need < cap ? need : cap;
    return w >= 1024 ? (uint32_t)(w - 1) : 0;
}

template <class SR>
static int dot3_count_launch(DevCSR &C, const DevCSR &M, bool mask_struct, const DevCSR &A,
                             const DevCSR &B, cudaStream_t s, int64_t *live_sum)
{
    using Z = typename SR::z_t;
    const int64_t mnz = M.nnz;
    const int64_t nkeys = M.nrows + B.nrows;
    const int64_t ntiles = (nkeys + CT_TILE - 1) / CT_TILE;
    const uint32_t bm_words = ct_bitmap_words<SR>(A.ncols);
    const bool spans_fit = bm_words > 0 && (int64_t)bm_words * 32 >= A.ncols;
    if (bm_words == 0) return NO_VALUE;
    const int nsm = runtime().num_sms;
    C.p = (int32_t *)dalloc((size_t)(M.nrows + 1) * 4, s);
    C.j = (int32_t *)dalloc((size_t)mnz * 4, s);
    C.x = dalloc((size_t)mnz * sizeof(Z), s);
    const int64_t nitems_max = std::min<int64_t>(nkeys, mnz) + mnz / 16 + 1;
    // counters, tile words, group work and group counts first and adjacent:
    // one memset
    int *counter = nullptr;
    int32_t *gcnt = nullptr, *boff = nullptr;
    unsigned long long *status = nullptr, *gwork = nullptr;
    CtQ *queue = nullptr;
    CtRec *bucket = nullptr;
    CtItem *items_bm = nullptr, *items_h = nullptr;
    D3Work *mq = nullptr;
    Carve cv(s);
    auto layout = [&]() {
        counter = cv.take<int>(32);
        status = cv.take<unsigned long long>((size_t)ntiles * 3);
        gwork = cv.take<unsigned long long>(nkeys);
        gcnt = cv.take<int32_t>(2 * nkeys);
        queue = cv.take<CtQ>(mnz);
        boff = cv.take<int32_t>(nkeys);
        bucket = cv.take<CtRec>(mnz);
        items_bm = cv.take<CtItem>(nitems_max);
        items_h = cv.take<CtItem>(nitems_max);
        mq = cv.take<D3Work>(spans_fit ? 1 : mnz);
    };
    layout();
    CallBlock blk(s);
    const bool got = blk.get(cv.off);
    cv.base = blk.base;
    cv.off = 0;
    layout();
    if (!C.p || !C.j || !C.x || !got) { dev_free(C, s); return OUT_OF_MEMORY; }
    cudaMemcpyAsync(C.p, M.p, (size_t)(M.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(counter, 0, (size_t)((const char *)(gcnt + 2 * nkeys) - (const char *)counter),
                    s);
    // counter layout: [0..3] totals, [4] tile ticket, [5] hash items, [6] bitmap
    // items, [7] merge items, [8] merge taken; zombies at byte 64, sum at 72
    int32_t *totals = counter;
    int *tile_ctr = counter + 4, *inext_h = counter + 5, *inext_bm = counter + 6;
    int *mq_len = counter + 7, *mq_next = counter + 8;
    unsigned long long *zc = (unsigned long long *)((char *)counter + 64);
    unsigned long long *sum = zc + 1;
    const bool vec = ((((uintptr_t)A.j) | ((uintptr_t)B.j)) & 15) == 0;
    int64_t blocks = ((mnz + 31) / 32 + 7) / 8;
    if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
    const int ps = prof_begin("dot3", s);
    k_ct_classify<SR><<<(unsigned)blocks, 256, 0, s>>>(
        M.p, M.j, mask_struct ? nullptr : M.x, M.type, mask_struct, mnz, M.nrows,
        A.p, A.j, B.p, B.j, bm_words * 32u, spans_fit, C.j, queue, gcnt, gwork, zc);
    k_ct_plan<<<(unsigned)ntiles, CT_TILE_T, 0, s>>>(
        gcnt, gwork, nkeys, (int32_t)M.nrows, A.p, A.j, B.p, B.j, status, tile_ctr, boff,
        items_bm, items_h, totals);
    k_ct_route<<<(unsigned)blocks, 256, 0, s>>>(queue, mnz, (int32_t)M.nrows, gcnt, boff,
                                                 bucket, M.p, M.j, A.p, B.p, mq, mq_len);
    k_ct_hash<SR><<<nsm * 5, CT_H_WARPS * 32, 0, s>>>(
        items_h, totals, inext_h, (int32_t)M.nrows, bucket, A.j, B.j, vec,
        C.j, (Z *)C.x, sum, zc);
    k_ct_bitmap<SR><<<nsm, CT_BM_THREADS, (size_t)(bm_words + 1) * 4, s>>>(
        items_bm, totals, inext_bm, (int32_t)M.nrows, bucket, A.j, B.j, vec,
        bm_words, C.j, (Z *)C.x, sum, zc);
    k_dot3_intersect<SR><<<nsm * 8, 256, 0, s>>>(
        mq, nullptr, mq_len, mq_next, A.j, A.x, A.iso, B.j, B.x, B.iso, C.j, (Z *)C.x, zc,
        sum);
    prof_end(ps, s);
    // the totals, the zombie count and the live sum in one read
    unsigned long long hv[10];
    cudaError_t e = readback(hv, counter, 80, s);
    if (e != cudaSuccess) { dev_free(C, s); return cuda_to_info(e); }
    if (((const int32_t *)hv)[CT_ERR]) { dev_free(C, s); return PANIC; }
    C.nzombies = (int64_t)hv[8];
    if (live_sum) *live_sum = (int64_t)hv[9];
    return SUCCESS;
}

template <class SR>
static int dot3_launch(DevCSR &C, const DevCSR &M, bool mask_struct,
                       const DevCSR &A, const DevCSR &B, cudaStream_t s, int64_t *live_sum)
{
    using Z = typename SR::z_t;
    const int64_t mnz = M.nnz;
    C.nrows = M.nrows; C.ncols = M.ncols; C.nnz = mnz; C.type = 0; C.iso = false;
    if constexpr (IsCount<SR>::value) {
        if (mnz >= CT_MIN_ENTRIES && M.nrows + B.nrows < INT32_MAX) {
            const int info = dot3_count_launch<SR>(C, M, mask_struct, A, B, s, live_sum);
            if (info != NO_VALUE) return info;
        }
    }
    C.p = (int32_t *)dalloc((size_t)(M.nrows + 1) * 4, s);
    C.j = (int32_t *)dalloc((size_t)(mnz ? mnz : 1) * 4, s);
    C.x = dalloc((size_t)(mnz ? mnz : 1) * sizeof(Z), s);
    // the work queue and its counters in one allocation
    int *counter = nullptr;
    D3Work *queue = nullptr;
    Carve cv(s);
    auto layout = [&]() {
        counter = cv.take<int>(16);
        queue = cv.take<D3Work>(mnz ? mnz : 1);
    };
    layout();
    CallBlock blk(s);
    const bool got = blk.get(cv.off);
    cv.base = blk.base;
    cv.off = 0;
    layout();
    if (!C.p || !C.j || !C.x || !got) {
        dev_free(C, s); return OUT_OF_MEMORY;
    }
    cudaMemcpyAsync(C.p, M.p, (size_t)(M.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(counter, 0, 16 * sizeof(int), s);
    int *qlen = counter, *qnext = counter + 1;
    unsigned long long *zc = (unsigned long long *)((char *)counter + 32);
    unsigned long long *sum = zc + 1;
    if (mnz > 0 && M.nrows > 0) {
        const int nsm = runtime().num_sms;
        int64_t warps_needed = (mnz + 31) / 32;
        int64_t blocks = (warps_needed + 7) / 8;
        if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
        const int ps = prof_begin("dot3", s);
        k_dot3_classify<SR><<<(unsigned)blocks, 256, 0, s>>>(
            M.p, M.j, mask_struct ? nullptr : M.x, M.type, mask_struct, mnz, M.nrows,
            A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso, C.j, (Z *)C.x,
            queue, qlen, zc, sum);
        k_dot3_intersect<SR><<<nsm * 8, 256, 0, s>>>(
            queue, nullptr, qlen, qnext, A.j, A.x, A.iso, B.j, B.x, B.iso, C.j,
            (Z *)C.x, zc, sum);
        prof_end(ps, s);
    }
    unsigned long long hv[2] = {0, 0};
    cudaError_t e = readback(hv, zc, 16, s);
    if (e != cudaSuccess) { dev_free(C, s); return cuda_to_info(e); }
    C.nzombies = (int64_t)hv[0];
    if (live_sum && IsCount<SR>::value) *live_sum = (int64_t)hv[1];
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
         const DevCSR &B, SemiringCode sr, cudaStream_t s, int64_t *live_sum)
{
    if (live_sum) *live_sum = 0;
    if (A.ncols != B.ncols || M.nrows != A.nrows || M.ncols != B.nrows)
        return DIMENSION_MISMATCH;
    if (M.nzombies > 0) return NO_VALUE;   // the mask must be free of zombies
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
        int info = dot3_launch<Semiring<ADD, MULT, CT>>(C, M, mask_struct, A, B, s, \
                                                        live_sum);                 \
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


// ---------------------------------------------------------------------------
// dot3 with no allocation at all
//
// Some callers cannot allocate device memory: a host application whose
// device memory is owned by another allocator (a framework's caching pool or
// a preallocated arena it must not bypass), or a latency-bound loop that may
// not call cudaMalloc/cudaFree because they can synchronise the device.  For
// them grb_b200_dot3_noalloc runs the same two kernels as dot3 above, with
// every input and output in caller-owned device memory and the work queue
// and counters in the fixed array below.  The array lives in the library's
// device image: every GPU that loads the library holds its 32 MiB until the
// process exits.  All calls share it and it keeps the last call's contents;
// the counters are cleared at the start of each call.  Calls that overlap on
// the same GPU (from concurrent streams or host threads) race on the array
// and must be serialised by the caller; each GPU has its own copy.
// ---------------------------------------------------------------------------

static constexpr size_t NOALLOC_BYTES = (size_t)32 << 20;
static constexpr size_t NOALLOC_HEAD = 256;        // counters, then the queue
static constexpr int64_t NOALLOC_MAX_ENTRIES =
    (int64_t)((NOALLOC_BYTES - NOALLOC_HEAD) / sizeof(D3Work));
// the limit the header publishes is the one enforced here
static_assert(NOALLOC_MAX_ENTRIES == GRB_B200_DOT3_NOALLOC_MAX_ENTRIES,
              "GRB_B200_DOT3_NOALLOC_MAX_ENTRIES must match the scratch array's capacity");

static __device__ __align__(256) unsigned char g_dot3_scratch[NOALLOC_BYTES];

// Device address of the array, looked up once per device with that device
// current (host code may not use the symbol's host-side name as a pointer).
static std::mutex g_scratch_mu;
static void *g_scratch_addr[128];

static int noalloc_scratch(void **addr)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 128) return PANIC;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_dot3_scratch);
        if (e != cudaSuccess || p == nullptr) { cudaGetLastError(); return PANIC; }
        g_scratch_addr[dev] = p;
    }
    *addr = g_scratch_addr[dev];
    return SUCCESS;
}

template <class SR>
static int dot3_noalloc_launch(int64_t nrows, int64_t mnz, const int32_t *Mp,
                               const int32_t *Mj, const int32_t *Ap, const int32_t *Aj,
                               const void *Ax, bool a_iso, const int32_t *Bp,
                               const int32_t *Bj, const void *Bx, bool b_iso,
                               int32_t *Cj, void *Cx, int64_t *nzombies,
                               cudaStream_t s)
{
    using Z = typename SR::z_t;
    if ((SR::needs_a && Ax == nullptr) || (SR::needs_b && Bx == nullptr)) return NULL_POINTER;
    void *scratch = nullptr;
    int info = noalloc_scratch(&scratch);
    if (info != SUCCESS) return info;
    int nsm = 0;
    info = device_sm_count(&nsm);
    if (info != SUCCESS) return info;
    int *qlen = (int *)scratch, *qnext = qlen + 1;
    unsigned long long *zc = (unsigned long long *)((char *)scratch + 32);
    D3Work *queue = (D3Work *)((char *)scratch + NOALLOC_HEAD);
    cudaError_t e = cudaMemsetAsync(scratch, 0, NOALLOC_HEAD, s);
    if (e != cudaSuccess) return cuda_to_info(e);
    if (mnz > 0 && nrows > 0) {
        int64_t blocks = ((mnz + 31) / 32 + 7) / 8;
        if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
        k_dot3_classify<SR><<<(unsigned)blocks, 256, 0, s>>>(
            Mp, Mj, nullptr, T_BOOL, true, mnz, nrows, Ap, Aj, Ax, a_iso,
            Bp, Bj, Bx, b_iso, Cj, (Z *)Cx, queue, qlen, zc, nullptr);
        k_dot3_intersect<SR><<<nsm * 8, 256, 0, s>>>(
            queue, nullptr, qlen, qnext, Aj, Ax, a_iso, Bj, Bx, b_iso, Cj, (Z *)Cx, zc,
            nullptr);
    }
    unsigned long long hz = 0;
    e = cudaMemcpyAsync(&hz, zc, sizeof(hz), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_to_info(e);
    if (nzombies) *nzombies = (int64_t)hz;
    return SUCCESS;
}

}  // namespace grb

extern "C" int grb_b200_dot3_noalloc(
    int64_t nrows, int64_t ncols, int64_t mnz,
    const int32_t *Mp, const int32_t *Mj,
    const int32_t *Ap, const int32_t *Aj, const void *Ax, bool A_iso,
    const int32_t *Bp, const int32_t *Bj, const void *Bx, bool B_iso,
    const grb_b200_semiring *semiring, int32_t *Cj, void *Cx, int64_t *nzombies,
    void *stream)
{
    using namespace grb;
    if (!Mp || !Mj || !Ap || !Aj || !Bp || !Bj || !Cj || !Cx || !semiring)
        return NULL_POINTER;
    if (nrows < 0 || ncols < 0 || mnz < 0) return INVALID_VALUE;
    if (mnz > NOALLOC_MAX_ENTRIES) {
        fprintf(stderr, "grb_b200_dot3_noalloc: %lld mask entries exceed the fixed "
                "scratch capacity of %lld entries\n", (long long)mnz,
                (long long)NOALLOC_MAX_ENTRIES);
        return INVALID_VALUE;
    }
    if (nrows >= INT32_MAX || ncols >= INT32_MAX) {
        fprintf(stderr, "grb_b200_dot3_noalloc: dimensions %lld x %lld do not fit the "
                "int32 indices of the device arrays\n", (long long)nrows, (long long)ncols);
        return INVALID_VALUE;
    }
    // no init_device() here: it changes the default memory pool's release
    // threshold, and this entry point leaves the caller's allocator alone
    cudaStream_t s = (cudaStream_t)stream;
    SemiringCode sr{semiring->add_opcode, semiring->mult_opcode, semiring->type};
#define GRB_NOALLOC_CASE(ADD, MULT, TC, CT)                                      \
    if (sr.add == ADD && sr.mult == MULT && sr.type == TC)                       \
        return dot3_noalloc_launch<Semiring<ADD, MULT, CT>>(nrows, mnz, Mp, Mj,  \
            Ap, Aj, Ax, A_iso, Bp, Bj, Bx, B_iso, Cj, Cx, nzombies, s);
    GRB_FOR_EACH_SEMIRING(GRB_NOALLOC_CASE)
#undef GRB_NOALLOC_CASE
    return NO_VALUE;
}
