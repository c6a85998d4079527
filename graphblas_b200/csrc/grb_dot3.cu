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
                int32_t *__restrict__ gcnt, uint32_t bm_bits)
{
    using Z = typename SR::z_t;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long zcount = 0;
    for (int64_t base = warp * 32; base < mnz; base += nwarps * 32) {
        const int64_t pm = base + lane;
        const bool valid = pm < mnz;
        // row of the chunk's first entry (the last r with Mp[r] <= base,
        // searched by the whole warp), then each lane walks forward
        const int32_t r0 = warp_last_le<int32_t, int32_t>(Mp, (int32_t)nrows, (int32_t)base,
                                                          lane);
        int32_t i = r0;
        if (valid) while (Mp[i + 1] <= pm) i++;
        int32_t j = 0, a0 = 0, a1 = 0, b0 = 0, b1 = 0, key = -1;
        bool coop = false, exists = false;
        Z cij = Z();
        if (valid) {
            j = Mj[pm];
            const bool mval = mask_struct || Mx == nullptr || mask_value_true(Mx, mtype, pm);
            const int32_t pa0 = Ap[i], pa1 = Ap[i + 1];
            const int32_t pb0 = Bp[j], pb1 = Bp[j + 1];
            if (mval && pa1 > pa0 && pb1 > pb0) {
                const int32_t blo = Bj[pb0], bhi = Bj[pb1 - 1];
                // A row that will be the bitmap / hash key whole (the longer
                // list, its column span fits the bitmap, and the entry is not
                // merged here) needs no trimmed range: its two searches in
                // the long row are skipped, and only the other list is
                // trimmed, to the key row's first and last columns.  A's row
                // is tested on the untrimmed lengths, B's after A's trim.
                const bool akey = bm_bits && (pa1 - pa0) > (pb1 - pb0) &&
                                  (pa1 - pa0) + (pb1 - pb0) > D3_SMALL &&
                                  (uint32_t)(Aj[pa1 - 1] - Aj[pa0]) < bm_bits;
                if (akey) {
                    a0 = pa0;
                    a1 = pa1;
                } else {
                    a0 = lower_bound(Aj, pa0, pa1, blo);
                    a1 = upper_bound(Aj, a0, pa1, bhi);
                }
                const bool bkey = !akey && bm_bits && (pb1 - pb0) >= (a1 - a0) &&
                                  (uint32_t)(bhi - blo) < bm_bits &&
                                  (a1 - a0) + (pb1 - pb0) > D3_SMALL;
                if (a1 > a0) {
                    const int32_t alo = Aj[a0], ahi = Aj[a1 - 1];
                    if (bkey) {
                        b0 = pb0;
                        b1 = pb1;
                    } else {
                        b0 = lower_bound(Bj, pb0, pb1, alo);
                        b1 = upper_bound(Bj, b0, pb1, ahi);
                    }
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
                        } else if (bkey) {
                            coop = true;
                            if ((a1 - a0) <= (1 << 20)) key = (int32_t)nrows + j;
                        } else if (akey) {
                            coop = true;
                            if ((b1 - b0) <= (1 << 20)) key = i;
                        } else {
                            coop = true;
                            if (bm_bits && min(a1 - a0, b1 - b0) <= (1 << 20)) {
                                // bitmap of the longer list's whole row, if
                                // its column span fits the bitmap (probed
                                // lists of at most 2^20 keep the bitmap
                                // kernel's per-round probe sums in int32)
                                if ((a1 - a0) > (b1 - b0)) {
                                    if ((uint32_t)(Aj[pa1 - 1] - Aj[pa0]) < bm_bits) key = i;
                                } else if ((uint32_t)(bhi - blo) < bm_bits) {
                                    key = (int32_t)nrows + j;
                                }
                            }
                        }
                    }
                }
            }
            if (!coop) {
                if (exists) { Cj[pm] = j; Cx[pm] = cij; }
                else { Cj[pm] = flip(j); zcount++; }
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
                queue[slot] = D3Work{(int32_t)pm, i, j, a0, a1, b0, b1, key};
            }
        }
        if (bm_bits) {
            // group sizes, one atomic per distinct key in the warp
            const bool grouped = coop && key >= 0;
            const unsigned gm = __ballot_sync(0xffffffffu, grouped);
            if (grouped) {
                const unsigned same = __match_any_sync(gm, key);
                if ((int)(__ffs(same) - 1) == lane) atomicAdd(&gcnt[key], __popc(same));
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) zcount += __shfl_down_sync(0xffffffffu, zcount, o);
    if (lane == 0 && zcount) atomicAdd(nzombies, zcount);
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
                 unsigned long long *__restrict__ nzombies)
{
    using Z = typename SR::z_t;
    const int lane = threadIdx.x & 31;
    const int qlen = *qlen_p;
    unsigned long long zcount = 0;
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
                if (acc_has) { Cj[e.pm] = e.j; Cx[e.pm] = acc; }
                else { Cj[e.pm] = flip(e.j); zcount++; }
            }
        }
    }
    if (lane == 0 && zcount) atomicAdd(nzombies, zcount);
}

// ---------------------------------------------------------------------------
// bitmap path for counting semirings (PLUS_PAIR on integers: triangle and
// support counts)
//
// A long entry is intersected by probing the elements of its shorter list in
// a shared-memory bitmap of its longer list's whole row, so the longer list
// is read once per group of entries sharing it instead of once per entry:
// entries whose A(i,:) is longer are grouped by i, those whose B(j,:) is
// longer by j (key nrows + j).  The result of PLUS_PAIR is the number of
// matches, which needs neither values nor an order.  Groups with fewer than
// D3_GMIN entries, and rows whose column span does not fit the bitmap, stay
// on the merge path.
// ---------------------------------------------------------------------------

static constexpr int D3_GMIN = 8;              // smallest group worth a bitmap
static constexpr int64_t D3_WCHUNK = 1 << 20;  // probes per bitmap work item
static constexpr int D3_HKEY = 256;             // key rows up to this long: warp hash
static constexpr int D3_HSLOTS = 512;           // slots of a warp's hash table
static constexpr int64_t D3_HCHUNK = 1 << 16;   // probes per warp-hash work item
static constexpr int D3_HWARPS = 8;             // warps (tables) per hash block
static constexpr int D3_BM_THREADS = 1024;
static constexpr int D3_LONG = 4096;          // longer lists go to the shared table
static constexpr int D3_PROBE_UNROLL = 4;     // probe loads in flight per lane
static constexpr int D3_SEG = 512;            // probes per shared long-list segment
static constexpr int D3_TABLE = 1024;         // long lists registered per item

// a grouped entry as the bitmap kernel reads it: its probed list and where
// its result goes
struct __align__(16) D3Rec { int32_t s0, len, pm, j; };

// a work item: every nit-th entry of key's group, from the t-th; its key row
// (offsets rp0..rp1, first column lo) and lanes per entry 2^lg
struct __align__(16) D3Item { int32_t key, t, nit, m_item, rp0, rp1, lo, lg; int64_t g0;
                               int32_t hi, pad; };

template <class SR> struct IsCount {
    static constexpr bool value = SR::add_op == OP_PLUS && SR::mult_op == OP_PAIR &&
        std::is_integral<typename SR::z_t>::value &&
        !std::is_same<typename SR::z_t, bool>::value;
};

// group size kept (0 below D3_GMIN), as int64 for the offsets scan
__global__ void k_d3_gsize(const int32_t *__restrict__ gcnt, int64_t nkeys,
                           int64_t *__restrict__ gsz)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < nkeys; t += stride) {
        const int32_t c = gcnt[t];
        gsz[t] = c >= D3_GMIN ? c : 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) gsz[nkeys] = 0;    // the scan's last input
}

// route every queued entry to its group's bucket or to the merge list
__global__ void __launch_bounds__(256)
k_d3_route(const D3Work *__restrict__ queue, const int *__restrict__ qlen_p,
           const int64_t *__restrict__ gsz, const int64_t *__restrict__ goff,
           int32_t *__restrict__ gfill, unsigned long long *__restrict__ gwork,
           D3Rec *__restrict__ bucket, int32_t nrows, int32_t *__restrict__ merge_sel,
           int *__restrict__ merge_len)
{
    const int lane = threadIdx.x & 31;
    const int qlen = *qlen_p;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
         base < qlen; base += nw * 32) {
        const int w = (int)(base + lane);
        bool grouped = false, merge = false;
        int32_t key = -1;
        unsigned long long work = 0;
        D3Rec rec{0, 0, 0, 0};
        if (w < qlen) {
            const D3Work e = queue[w];
            key = e.pad;
            grouped = key >= 0 && gsz[key] > 0;
            merge = !grouped;
            // probes: the other list's elements (the shorter one)
            const bool by_row = key < nrows;
            rec = by_row ? D3Rec{e.b0, e.b1 - e.b0, e.pm, e.j}
                         : D3Rec{e.a0, e.a1 - e.a0, e.pm, e.j};
            work = (unsigned long long)rec.len;
        }
        const unsigned gm = __ballot_sync(0xffffffffu, grouped);
        if (grouped) {
            const unsigned same = __match_any_sync(gm, key);
            const int leader = __ffs(same) - 1;
            // the leader reserves slots and adds the work of its lanes (the
            // work only balances items: each lane's share is capped at 2^26)
            const unsigned wsum = __reduce_add_sync(same, (unsigned)min(work, 1ull << 26));
            int slot0 = 0;
            if (lane == leader) {
                slot0 = atomicAdd(&gfill[key], __popc(same));
                atomicAdd(&gwork[key], (unsigned long long)wsum);
            }
            slot0 = __shfl_sync(same, slot0, leader);
            bucket[goff[key] + slot0 + __popc(same & ((1u << lane) - 1))] = rec;
        }
        const unsigned mm = __ballot_sync(0xffffffffu, merge);
        if (mm) {
            int mbase = 0;
            if (lane == 0) mbase = atomicAdd(merge_len, __popc(mm));
            mbase = __shfl_sync(0xffffffffu, mbase, 0);
            if (merge) merge_sel[mbase + __popc(mm & ((1u << lane) - 1))] = w;
        }
    }
}

// work items per group.  A group whose key row has at most D3_HKEY entries
// goes to the warp-hash kernel (items of about D3_HCHUNK probes), a longer
// key row to the block-bitmap kernel (items of about D3_WCHUNK probes); at
// most one item per 32 entries, so items never outnumber nkeys + entries/32.
__global__ void k_d3_item_count(const int64_t *__restrict__ gsz,
                                const unsigned long long *__restrict__ gwork,
                                int64_t nkeys, int32_t nrows,
                                const int32_t *__restrict__ Ap,
                                const int32_t *__restrict__ Bp,
                                int64_t *__restrict__ nit_big, int64_t *__restrict__ nit_small)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    if (t == 0) { nit_big[nkeys] = 0; nit_small[nkeys] = 0; }    // the scans' last inputs
    for (; t < nkeys; t += stride) {
        const int64_t g = gsz[t];
        int64_t nb = 0, ns = 0;
        if (g > 0) {
            const bool by_row = t < nrows;
            const int32_t r = by_row ? (int32_t)t : (int32_t)(t - nrows);
            const int32_t klen = by_row ? Ap[r + 1] - Ap[r] : Bp[r + 1] - Bp[r];
            const bool small = klen <= D3_HKEY;
            int64_t n = 1 + (int64_t)(gwork[t] / (small ? D3_HCHUNK : D3_WCHUNK));
            const int64_t mx = g / 32 > 1 ? g / 32 : 1;
            if (n > mx) n = mx;
            if (small) ns = n; else nb = n;
        }
        nit_big[t] = nb;
        nit_small[t] = ns;
    }
}

__global__ void k_d3_item_fill(const int64_t *__restrict__ ioff, int64_t nkeys,
                               const int64_t *__restrict__ goff,
                               const unsigned long long *__restrict__ gwork, int32_t nrows,
                               const int32_t *__restrict__ Ap, const int32_t *__restrict__ Aj,
                               const int32_t *__restrict__ Bp, const int32_t *__restrict__ Bj,
                               D3Item *__restrict__ items)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < nkeys; t += stride) {
        const int64_t o = ioff[t], n = ioff[t + 1] - o;
        if (n == 0) continue;
        const bool by_row = t < nrows;
        const int32_t r = by_row ? (int32_t)t : (int32_t)(t - nrows);
        const int32_t rp0 = by_row ? Ap[r] : Bp[r], rp1 = by_row ? Ap[r + 1] : Bp[r + 1];
        const int32_t lo = by_row ? Aj[rp0] : Bj[rp0];
        const int32_t hi = by_row ? Aj[rp1 - 1] : Bj[rp1 - 1];
        const int64_t g0 = goff[t], gn = goff[t + 1] - g0;
        // lanes per entry: a power of two near an eighth of the mean list
        // length, so a lane's D3_PROBE_UNROLL loads are mostly in use and
        // short lists of a skewed group leave few lanes idle (half and a
        // quarter of the mean, and a sixteenth, measured slower)
        const unsigned long long mean = gwork[t] / (unsigned long long)gn;
        int lg = 0;
        while (lg < 5 && (8ull << lg) < mean) lg++;
        for (int64_t q = 0; q < n; q++)
            items[o + q] = D3Item{(int32_t)t, (int32_t)q, (int32_t)n,
                                  (int32_t)((gn - q + n - 1) / n), rp0, rp1, lo, lg, g0,
                                  hi, 0};
    }
}

// One block per SM, persistent: take an item, set the bits of its key row
// (A(i,:) or B(j,:), relative to the row's first column) in shared memory,
// then count, for every entry of the item, the elements of its other
// (trimmed) list that hit the bitmap, in two phases:
//   A. each warp splits into groups of G lanes (G a power of two near half
//      the group's mean probes per entry, so short lists do not waste
//      lanes); groups take the item's entries one at a time from a shared
//      counter and stride over their list; a list longer than D3_LONG is
//      instead registered in a shared table (up to D3_TABLE entries) as
//      segments of D3_SEG probes;
//   B. all warps take the segments from a shared counter, 32 probes per step,
//      and add their hits to the entry's shared count; then the table's
//      entries are written.
// If the table is full, the group that owns the entry finishes it itself.
// The bits are cleared again from the row before the next item.
template <class SR>
__global__ void __launch_bounds__(D3_BM_THREADS, 1)
k_dot3_bitmap_count(const D3Item *__restrict__ items, const int64_t *__restrict__ nitems_p,
                    int *__restrict__ inext, const D3Rec *__restrict__ bucket,
                    int32_t nrows, const int32_t *__restrict__ Aj,
                    const int32_t *__restrict__ Bj,
                    uint32_t bm_words, int32_t *__restrict__ Cj,
                    typename SR::z_t *__restrict__ Cx,
                    unsigned long long *__restrict__ nzombies)
{
    using Z = typename SR::z_t;
    extern __shared__ __align__(16) uint32_t bm[];
    __shared__ int s_item, s_next, s_gnext;
    __shared__ D3Item s_I;                        // the next item, fetched ahead
    __shared__ unsigned long long s_tbl;          // (segments << 32) | entries
    __shared__ int32_t t_start[D3_TABLE], t_rem[D3_TABLE], t_seg0[D3_TABLE];
    __shared__ int32_t t_cnt[D3_TABLE], t_pm[D3_TABLE], t_j[D3_TABLE];
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t nbits = bm_words * 32u;
    for (uint32_t q = tid; q < bm_words; q += blockDim.x) bm[q] = 0;
    const int64_t nitems = *nitems_p;
    unsigned long long zc = 0;
    // hits among S[b0 + t] for t = first, first + step, ... < n
    // (D3_PROBE_UNROLL predicated loads issued together per step, the tail included;
    // a skipped slot reads as lo - 1, which is never a bit of the row)
    auto probes = [&](const int32_t *S, int32_t b0, int32_t first, int32_t step, int32_t n,
                      int32_t lo) -> int {
        int c = 0;
        for (int32_t t = first; t < n; t += D3_PROBE_UNROLL * step) {
            int32_t x[D3_PROBE_UNROLL];
            #pragma unroll
            for (int u = 0; u < D3_PROBE_UNROLL; u++) {
                const int32_t q = t + u * step;
                x[u] = q < n ? S[b0 + q] : lo - 1;
            }
            #pragma unroll
            for (int u = 0; u < D3_PROBE_UNROLL; u++) {
                const uint32_t k = (uint32_t)(x[u] - lo);
                c += (k < nbits) ? (int)((bm[k >> 5] >> (k & 31)) & 1u) : 0;
            }
        }
        return c;
    };
    if (tid == 0) {
        s_item = atomicAdd(inext, 1);
        if (s_item < nitems) s_I = items[s_item];
    }
    while (true) {
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const D3Item I = s_I;
        __syncthreads();
        if (tid == 0) { s_next = 0; s_gnext = 0; s_tbl = 0; }
        const bool by_row = I.key < nrows;
        const int32_t *J = by_row ? Aj : Bj;
        const int32_t *S = by_row ? Bj : Aj;     // the probed lists
        const int32_t rp0 = I.rp0, rp1 = I.rp1, lo = I.lo;
        // set the key row's bits: four loads in flight per thread
        {
            const int32_t nt = (int32_t)blockDim.x;
            int32_t q = rp0 + tid;
            for (; q + 3 * nt < rp1; q += 4 * nt) {
                const uint32_t k0 = (uint32_t)(J[q] - lo), k1 = (uint32_t)(J[q + nt] - lo);
                const uint32_t k2 = (uint32_t)(J[q + 2 * nt] - lo);
                const uint32_t k3 = (uint32_t)(J[q + 3 * nt] - lo);
                atomicOr(&bm[k0 >> 5], 1u << (k0 & 31));
                atomicOr(&bm[k1 >> 5], 1u << (k1 & 31));
                atomicOr(&bm[k2 >> 5], 1u << (k2 & 31));
                atomicOr(&bm[k3 >> 5], 1u << (k3 & 31));
            }
            for (; q < rp1; q += nt) {
                const uint32_t k = (uint32_t)(J[q] - lo);
                atomicOr(&bm[k >> 5], 1u << (k & 31));
            }
        }
        const int64_t g0 = I.g0;
        const int32_t m_item = I.m_item;
        const int lg = I.lg;
        const int G = 1 << lg, gi = lane >> lg, gl = lane & (G - 1);
        const int groups = 32 >> lg;
        __syncthreads();
        // fetch the next item while this one runs
        if (tid == 0) {
            s_item = atomicAdd(inext, 1);
            if (s_item < nitems) s_I = items[s_item];
        }
        // phase A: the next chunk's records are fetched while this chunk
        // probes, so their load latency overlaps the probes'
        int c_next = 0;
        if (lane == 0) c_next = atomicAdd(&s_next, groups);
        c_next = __shfl_sync(0xffffffffu, c_next, 0);
        D3Rec e_next{0, 0, 0, 0};
        if (c_next + gi < m_item) e_next = bucket[g0 + I.t + (int64_t)I.nit * (c_next + gi)];
        while (true) {
            const int c0 = c_next;
            if (c0 >= m_item) break;
            const int32_t rr = c0 + gi;
            const int32_t s0 = e_next.s0, len = rr < m_item ? e_next.len : 0;
            const int32_t pm = e_next.pm, j = e_next.j;
            if (lane == 0) c_next = atomicAdd(&s_next, groups);
            c_next = __shfl_sync(0xffffffffu, c_next, 0);
            if (c_next + gi < m_item) e_next = bucket[g0 + I.t + (int64_t)I.nit * (c_next + gi)];
            // a long list goes to the table (its group's first lane registers
            // it); the group keeps it only if the table is full
            unsigned slot = 0xffffffffu;
            if (len > D3_LONG && gl == 0) {
                const unsigned long long nseg =
                    (unsigned long long)((len + D3_SEG - 1) / D3_SEG);
                const unsigned long long old = atomicAdd(&s_tbl, (nseg << 32) | 1ull);
                slot = (unsigned)(old & 0xffffffffull);
                if (slot < (unsigned)D3_TABLE) {
                    t_start[slot] = s0;
                    t_rem[slot] = len;
                    t_seg0[slot] = (int32_t)(old >> 32);
                    t_cnt[slot] = 0;
                    t_pm[slot] = pm;
                    t_j[slot] = j;
                }
            }
            slot = __shfl_sync(0xffffffffu, slot, gi << lg);
            const bool own = rr < m_item && slot >= (unsigned)D3_TABLE;
            int cnt = own ? probes(S, s0, gl, G, len, lo) : 0;
            for (int o = G >> 1; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o, G);
            if (own && gl == 0) {
                if (cnt) { Cj[pm] = j; Cx[pm] = (Z)cnt; }
                else { Cj[pm] = flip(j); zc++; }
            }
        }
        __syncthreads();
        // phase B
        const unsigned long long tb = s_tbl;
        const int ntab = (int)min((unsigned long long)D3_TABLE, tb & 0xffffffffull);
        if (ntab > 0) {
            const int total = t_seg0[ntab - 1] + (t_rem[ntab - 1] + D3_SEG - 1) / D3_SEG;
            while (true) {
                int g = 0;
                if (lane == 0) g = atomicAdd(&s_gnext, 1);
                g = __shfl_sync(0xffffffffu, g, 0);
                if (g >= total) break;
                // table entry holding segment g: last with t_seg0 <= g
                int a = 0, b = ntab;
                while (b - a > 1) {
                    const int mid = (a + b) >> 1;
                    if (t_seg0[mid] <= g) a = mid; else b = mid;
                }
                const int32_t off = (g - t_seg0[a]) * D3_SEG;
                const int32_t n = min(D3_SEG, t_rem[a] - off);
                const int c = (int)__reduce_add_sync(
                    0xffffffffu, (unsigned)probes(S, t_start[a] + off, lane, 32, n, lo));
                if (lane == 0 && c) atomicAdd(&t_cnt[a], c);
            }
        }
        __syncthreads();
        for (int q = tid; q < ntab; q += blockDim.x) {
            const int c = t_cnt[q];
            const int32_t pm = t_pm[q], j = t_j[q];
            if (c) { Cj[pm] = j; Cx[pm] = (Z)c; }
            else { Cj[pm] = flip(j); zc++; }
        }
        __syncthreads();
        // clear: zero the row's word range with 16-byte stores when that is
        // cheaper than revisiting the row's entries
        const uint32_t span_words = (uint32_t)(I.hi - lo) / 32u + 1u;
        if (span_words <= 4u * (uint32_t)(rp1 - rp0)) {
            uint4 *b4 = reinterpret_cast<uint4 *>(bm);
            const uint32_t n4 = (span_words + 3u) / 4u;
            for (uint32_t q = tid; q < n4; q += blockDim.x) b4[q] = make_uint4(0, 0, 0, 0);
        } else {
            for (int32_t q = rp0 + tid; q < rp1; q += blockDim.x) {
                const uint32_t k = (uint32_t)(J[q] - lo);
                bm[k >> 5] = 0;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) zc += __shfl_down_sync(0xffffffffu, zc, o);
    if (lane == 0 && zc) atomicAdd(nzombies, zc);
}

// One warp per work item whose key row is short (at most D3_HKEY entries):
// the key row's columns go into the warp's own shared-memory hash table
// (D3_HSLOTS slots, open addressing, at most half full), then the warp's
// lanes, in groups of 2^lg per entry, probe the item's entries' other lists
// against it.  No block-wide barrier: the many small groups of a skewed
// graph run side by side, 8 tables (16 KB) per block.
__device__ __forceinline__ uint32_t d3_hash(int32_t k)
{
    return ((uint32_t)k * 0x9E3779B1u) >> (32 - 9);       // 2^9 = D3_HSLOTS
}

template <class SR>
__global__ void __launch_bounds__(D3_HWARPS * 32)
k_dot3_hash_count(const D3Item *__restrict__ items, const int64_t *__restrict__ nitems_p,
                  int *__restrict__ inext, const D3Rec *__restrict__ bucket,
                  int32_t nrows, const int32_t *__restrict__ Aj,
                  const int32_t *__restrict__ Bj, int32_t *__restrict__ Cj,
                  typename SR::z_t *__restrict__ Cx,
                  unsigned long long *__restrict__ nzombies)
{
    using Z = typename SR::z_t;
    __shared__ int32_t tab_all[D3_HWARPS][D3_HSLOTS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t *tab = tab_all[w];
    for (int q = lane; q < D3_HSLOTS; q += 32) tab[q] = -1;
    __syncwarp();
    const int64_t nitems = *nitems_p;
    unsigned long long zc = 0;
    auto has = [&](int32_t k) -> int {
        uint32_t h = d3_hash(k);
        while (true) {
            const int32_t v = tab[h];
            if (v == k) return 1;
            if (v < 0) return 0;
            h = (h + 1) & (D3_HSLOTS - 1);
        }
    };
    while (true) {
        int it = 0;
        if (lane == 0) it = atomicAdd(inext, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        const D3Item I = items[it];
        const bool by_row = I.key < nrows;
        const int32_t *J = by_row ? Aj : Bj;
        const int32_t *S = by_row ? Bj : Aj;
        for (int32_t q = I.rp0 + lane; q < I.rp1; q += 32) {
            const int32_t k = J[q];
            uint32_t h = d3_hash(k);
            while (atomicCAS(&tab[h], -1, k) != -1) h = (h + 1) & (D3_HSLOTS - 1);
        }
        __syncwarp();
        const int lg = I.lg, G = 1 << lg, gi = lane >> lg, gl = lane & (G - 1);
        const int groups = 32 >> lg;
        // the next chunk's records load while this chunk probes; four
        // predicated loads per step (a skipped slot looks up -2, never a key)
        D3Rec e_next{0, 0, 0, 0};
        if (gi < I.m_item) e_next = bucket[I.g0 + I.t + (int64_t)I.nit * gi];
        for (int32_t c0 = 0; c0 < I.m_item; c0 += groups) {
            const int32_t rr = c0 + gi;
            const int32_t s0 = e_next.s0, len = rr < I.m_item ? e_next.len : 0;
            const int32_t pm = e_next.pm, j = e_next.j;
            if (rr + groups < I.m_item)
                e_next = bucket[I.g0 + I.t + (int64_t)I.nit * (rr + groups)];
            int cnt = 0;
            for (int32_t t = gl; t < len; t += 4 * G) {
                int32_t x[4];
                #pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int32_t q = t + u * G;
                    x[u] = q < len ? S[s0 + q] : -2;
                }
                #pragma unroll
                for (int u = 0; u < 4; u++) cnt += x[u] >= 0 ? has(x[u]) : 0;
            }
            for (int o = G >> 1; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o, G);
            if (rr < I.m_item && gl == 0) {
                if (cnt) { Cj[pm] = j; Cx[pm] = (Z)cnt; }
                else { Cj[pm] = flip(j); zc++; }
            }
        }
        __syncwarp();
        for (int q = lane; q < D3_HSLOTS; q += 32) tab[q] = -1;
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) zc += __shfl_down_sync(0xffffffffu, zc, o);
    if (lane == 0 && zc) atomicAdd(nzombies, zc);
}

static constexpr int64_t D3_BM_MIN_ENTRIES = 1 << 16;   // mask entries

// Words of the shared-memory bitmap: enough for every column index (plus one
// word of slack) when that fits beside the kernel's static shared memory,
// else the most that fits (rows spanning more columns stay on the merge
// path).  0 disables the bitmap path.
template <class SR>
static uint32_t bitmap_words(int64_t ncols)
{
    static int64_t avail = -1;
    if (avail < 0) {
        const void *fn = (const void *)k_dot3_bitmap_count<SR>;
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
    // a multiple of 4 words: the clear writes 16-byte blocks
    const int64_t need = ((ncols + 31) / 32 + 1 + 3) & ~(int64_t)3;
    const int64_t cap = avail & ~(int64_t)3;
    const int64_t w = need < cap ? need : cap;
    return w >= 1024 || w == need ? (uint32_t)w : 0;
}

template <class SR>
static int dot3_launch(DevCSR &C, const DevCSR &M, bool mask_struct,
                       const DevCSR &A, const DevCSR &B, cudaStream_t s)
{
    using Z = typename SR::z_t;
    const int64_t mnz = M.nnz;
    C.nrows = M.nrows; C.ncols = M.ncols; C.nnz = mnz; C.type = 0; C.iso = false;
    C.p = (int32_t *)dalloc((size_t)(M.nrows + 1) * 4, s);
    C.j = (int32_t *)dalloc((size_t)(mnz ? mnz : 1) * 4, s);
    C.x = dalloc((size_t)(mnz ? mnz : 1) * sizeof(Z), s);
    // the bitmap path: counting semirings on masks large enough to pay for it
    const int64_t nkeys = M.nrows + B.nrows;
    uint32_t bm_words = 0;
    if constexpr (IsCount<SR>::value) {
        if (mnz >= D3_BM_MIN_ENTRIES && nkeys < INT32_MAX) bm_words = bitmap_words<SR>(A.ncols);
    }
    // the work queue, the counters and the bitmap path's arrays in one
    // allocation; the counters, group sizes, fill cursors and work sums come
    // first and adjacent, so that one memset clears them
    int *counter = nullptr;
    D3Work *queue = nullptr;
    int32_t *gcnt = nullptr, *gfill = nullptr, *merge_sel = nullptr;
    D3Rec *bucket = nullptr;
    int64_t *gsz = nullptr, *goff = nullptr, *nit = nullptr, *ioff = nullptr, *ws = nullptr;
    int64_t *nit_s = nullptr, *ioff_s = nullptr;
    D3Item *items_s = nullptr;
    unsigned long long *gwork = nullptr;
    D3Item *items = nullptr;
    Carve cv(s);
    auto layout = [&]() {
        counter = cv.take<int>(16);
        if (bm_words) {
            gcnt = cv.take<int32_t>(nkeys);
            gfill = cv.take<int32_t>(nkeys);
            gwork = cv.take<unsigned long long>(nkeys);
        }
        queue = cv.take<D3Work>(mnz ? mnz : 1);
        if (bm_words) {
            gsz = cv.take<int64_t>(nkeys + 1);
            goff = cv.take<int64_t>(nkeys + 1);
            nit = cv.take<int64_t>(nkeys + 1);
            ioff = cv.take<int64_t>(nkeys + 1);
            nit_s = cv.take<int64_t>(nkeys + 1);
            ioff_s = cv.take<int64_t>(nkeys + 1);
            items_s = cv.take<D3Item>(nkeys + mnz / 32 + 1);
            items = cv.take<D3Item>(nkeys + mnz / 32 + 1);
            bucket = cv.take<D3Rec>(mnz);
            merge_sel = cv.take<int32_t>(mnz);
            ws = cv.take<int64_t>((int64_t)scan_ws_elems(nkeys + 1));
        }
    };
    layout();
    const bool got = cv.alloc();
    layout();
    struct Release { Carve &c; ~Release() { dfree(c.base, c.s); } } release{cv};
    if (!C.p || !C.j || !C.x || !got) {
        dev_free(C, s); return OUT_OF_MEMORY;
    }
    cudaMemcpyAsync(C.p, M.p, (size_t)(M.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
    const char *zero_end = bm_words ? (const char *)(gwork + nkeys) : (const char *)(counter + 16);
    cudaMemsetAsync(counter, 0, (size_t)(zero_end - (const char *)counter), s);
    int *qlen = counter, *qnext = counter + 1, *merge_len = counter + 2, *inext = counter + 3;
    unsigned long long *zc = (unsigned long long *)((char *)counter + 32);
    if (mnz > 0 && M.nrows > 0) {
        const int nsm = runtime().num_sms;
        int64_t warps_needed = (mnz + 31) / 32;
        int64_t blocks = (warps_needed + 7) / 8;
        if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
        const int ps = prof_begin("dot3", s);
        k_dot3_classify<SR><<<(unsigned)blocks, 256, 0, s>>>(
            M.p, M.j, mask_struct ? nullptr : M.x, M.type, mask_struct, mnz, M.nrows,
            A.p, A.j, A.x, A.iso, B.p, B.j, B.x, B.iso, C.j, (Z *)C.x,
            queue, qlen, zc, gcnt, bm_words * 32u);
        if (bm_words) {
            const int kb = (int)std::min<int64_t>((nkeys + 255) / 256, (int64_t)nsm * 8);
            k_d3_gsize<<<kb, 256, 0, s>>>(gcnt, nkeys, gsz);
            scan_exclusive_i64_ws(gsz, goff, nkeys + 1, ws, s);
            k_d3_route<<<(unsigned)blocks, 256, 0, s>>>(queue, qlen, gsz, goff, gfill, gwork,
                                                       bucket, (int32_t)M.nrows, merge_sel,
                                                       merge_len);
            k_d3_item_count<<<kb, 256, 0, s>>>(gsz, gwork, nkeys, (int32_t)M.nrows, A.p, B.p,
                                               nit, nit_s);
            scan_exclusive_i64_ws(nit, ioff, nkeys + 1, ws, s);
            k_d3_item_fill<<<kb, 256, 0, s>>>(ioff, nkeys, goff, gwork, (int32_t)M.nrows,
                                              A.p, A.j, B.p, B.j, items);
            scan_exclusive_i64_ws(nit_s, ioff_s, nkeys + 1, ws, s);
            k_d3_item_fill<<<kb, 256, 0, s>>>(ioff_s, nkeys, goff, gwork, (int32_t)M.nrows,
                                              A.p, A.j, B.p, B.j, items_s);
            if constexpr (IsCount<SR>::value)
                k_dot3_hash_count<SR><<<nsm * 8, D3_HWARPS * 32, 0, s>>>(
                    items_s, ioff_s + nkeys, inext + 1, bucket, (int32_t)M.nrows, A.j, B.j,
                    C.j, (Z *)C.x, zc);
            if constexpr (IsCount<SR>::value)
                k_dot3_bitmap_count<SR><<<nsm, D3_BM_THREADS, (size_t)bm_words * 4, s>>>(
                    items, ioff + nkeys, inext, bucket, (int32_t)M.nrows, A.j, B.j,
                    bm_words, C.j, (Z *)C.x, zc);
            k_dot3_intersect<SR><<<nsm * 8, 256, 0, s>>>(
                queue, merge_sel, merge_len, qnext, A.j, A.x, A.iso, B.j, B.x, B.iso,
                C.j, (Z *)C.x, zc);
        } else {
            k_dot3_intersect<SR><<<nsm * 8, 256, 0, s>>>(
                queue, nullptr, qlen, qnext, A.j, A.x, A.iso, B.j, B.x, B.iso, C.j,
                (Z *)C.x, zc);
        }
        prof_end(ps, s);
    }
    unsigned long long hz = 0;
    cudaError_t e = readback(&hz, zc, 8, s);
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
    int *qlen = (int *)scratch, *qnext = qlen + 1;
    unsigned long long *zc = (unsigned long long *)((char *)scratch + 32);
    D3Work *queue = (D3Work *)((char *)scratch + NOALLOC_HEAD);
    cudaError_t e = cudaMemsetAsync(scratch, 0, NOALLOC_HEAD, s);
    if (e != cudaSuccess) return cuda_to_info(e);
    if (mnz > 0 && nrows > 0) {
        const int nsm = runtime().num_sms;
        int64_t blocks = ((mnz + 31) / 32 + 7) / 8;
        if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
        k_dot3_classify<SR><<<(unsigned)blocks, 256, 0, s>>>(
            Mp, Mj, nullptr, T_BOOL, true, mnz, nrows, Ap, Aj, Ax, a_iso,
            Bp, Bj, Bx, b_iso, Cj, (Z *)Cx, queue, qlen, zc, nullptr, 0u);
        k_dot3_intersect<SR><<<nsm * 8, 256, 0, s>>>(
            queue, nullptr, qlen, qnext, Aj, Ax, a_iso, Bj, Bx, b_iso, Cj, (Z *)Cx, zc);
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
    if (mnz > NOALLOC_MAX_ENTRIES || nrows >= INT32_MAX || ncols >= INT32_MAX) {
        fprintf(stderr, "grb_b200_dot3_noalloc: %lld mask entries exceed the fixed "
                "scratch capacity of %lld entries\n", (long long)mnz,
                (long long)NOALLOC_MAX_ENTRIES);
        return INVALID_VALUE;
    }
    int info = init_device();
    if (info != SUCCESS) return info;
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
