// grb_common.cuh: shared device definitions for the B200 semiring SpGEMM path.
//
// Device matrices are CSR with int32 row offsets and column indices (every
// supported problem has n, nnz < 2^31); the host boundary narrows the
// reference's int64 arrays on upload and widens them on download.
//
// Type codes and operator opcodes are the reference's GB_Type_code and
// GB_Opcode values (Source/builtin/include/GB_opaque.h:28-42, 209-247), so a
// caller inside SuiteSparse:GraphBLAS can pass type->code / op->opcode as is.

#pragma once
#include <cstdint>
#include <cstddef>
#include <cmath>
#include <type_traits>
#include <cuda_runtime.h>

namespace grb {

// ---- GrB_Info values (Include/GraphBLAS.h:358-381) ----
enum Info : int {
    SUCCESS = 0, NO_VALUE = 1, NULL_POINTER = -2, INVALID_VALUE = -3,
    DOMAIN_MISMATCH = -5, DIMENSION_MISMATCH = -6, NOT_IMPLEMENTED = -8,
    PANIC = -101, OUT_OF_MEMORY = -102, INVALID_OBJECT = -104
};

// ---- type codes (GB_Type_code) ----
enum TypeCode : int { T_BOOL = 1, T_INT32 = 6, T_UINT32 = 7, T_INT64 = 8,
                      T_UINT64 = 9, T_FP32 = 10, T_FP64 = 11 };

// ---- binary operator opcodes (GB_Opcode) ----
enum Op : int {
    OP_NOP = 0, OP_FIRST = 72, OP_SECOND = 73, OP_ANY = 74, OP_PAIR = 75,
    OP_MIN = 76, OP_MAX = 77, OP_PLUS = 78, OP_MINUS = 79, OP_RMINUS = 80,
    OP_TIMES = 81, OP_DIV = 82, OP_LOR = 91, OP_LAND = 92, OP_LXOR = 93,
    OP_EQ = 102, OP_FIRSTI = 115, OP_FIRSTI1 = 116, OP_FIRSTJ = 117,
    OP_FIRSTJ1 = 118, OP_SECONDI = 119, OP_SECONDI1 = 120, OP_SECONDJ = 121,
    OP_SECONDJ1 = 122
};

inline size_t type_size(int t)
{
    switch (t) {
        case T_BOOL: return 1;
        case T_INT32: case T_UINT32: case T_FP32: return 4;
        case T_INT64: case T_UINT64: case T_FP64: return 8;
        default: return 0;
    }
}

// zombie encoding of a column index (Source/math/include/GB_zombie.h:37)
__host__ __device__ inline int32_t flip(int32_t j) { return -j - 2; }
__host__ __device__ inline bool is_zombie(int32_t j) { return j < 0; }

// device CSR matrix (row-major vectors)
struct DevCSR {
    int64_t nrows = 0, ncols = 0, nnz = 0;
    int32_t *p = nullptr;   // nrows+1
    int32_t *j = nullptr;   // nnz (zombies hold flip(j))
    void *x = nullptr;      // nnz values, or one value if iso, or null (pattern)
    int type = T_BOOL;
    bool iso = false;
    int64_t nzombies = 0;
};

// ---------------------------------------------------------------------------
// semiring definitions, one per (add monoid, multiply op, type)
// ---------------------------------------------------------------------------

template <int OP> struct is_positional {
    static constexpr bool value = (OP >= OP_FIRSTI && OP <= OP_SECONDJ1);
};

// The multiply op on operands a = A(i,k), b = B(k,j).  Floating point
// products and sums use explicit round-to-nearest intrinsics so the compiler
// cannot contract them into an FMA: the reference computes z = a*b and z + t
// as separately rounded operations.
template <int MULT, typename Z> struct Mult;

#define GRB_MULT(OPC, EXPR, NEEDA, NEEDB)                                     \
    template <typename Z> struct Mult<OPC, Z> {                               \
        static constexpr bool needs_a = NEEDA, needs_b = NEEDB;               \
        __device__ __forceinline__ static Z f(Z a, Z b, int64_t i, int64_t k, \
                                              int64_t j) { return EXPR; } };

template <typename Z> __device__ __forceinline__ Z rn_add(Z a, Z b) { return (Z)(a + b); }
template <> __device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
template <typename Z> __device__ __forceinline__ Z rn_mul(Z a, Z b) { return (Z)(a * b); }
template <> __device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ int32_t rn_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
template <> __device__ __forceinline__ int64_t rn_add(int64_t a, int64_t b) { return (int64_t)((uint64_t)a + (uint64_t)b); }
template <> __device__ __forceinline__ int32_t rn_mul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
template <> __device__ __forceinline__ int64_t rn_mul(int64_t a, int64_t b) { return (int64_t)((uint64_t)a * (uint64_t)b); }
template <> __device__ __forceinline__ bool rn_add(bool a, bool b) { return a || b; }
template <> __device__ __forceinline__ bool rn_mul(bool a, bool b) { return a && b; }

template <typename Z> __device__ __forceinline__ Z op_min(Z a, Z b) { return a < b ? a : b; }
template <typename Z> __device__ __forceinline__ Z op_max(Z a, Z b) { return a > b ? a : b; }
template <> __device__ __forceinline__ float op_min(float a, float b) { return fminf(a, b); }
template <> __device__ __forceinline__ float op_max(float a, float b) { return fmaxf(a, b); }
template <> __device__ __forceinline__ double op_min(double a, double b) { return fmin(a, b); }
template <> __device__ __forceinline__ double op_max(double a, double b) { return fmax(a, b); }

GRB_MULT(OP_TIMES,   rn_mul<Z>(a, b), true, true)
GRB_MULT(OP_PLUS,    rn_add<Z>(a, b), true, true)
GRB_MULT(OP_MIN,     op_min<Z>(a, b), true, true)
GRB_MULT(OP_MAX,     op_max<Z>(a, b), true, true)
GRB_MULT(OP_FIRST,   a, true, false)
GRB_MULT(OP_SECOND,  b, false, true)
GRB_MULT(OP_PAIR,    (Z)1, false, false)
GRB_MULT(OP_LAND,    (Z)((a != (Z)0) && (b != (Z)0)), true, true)
GRB_MULT(OP_LOR,     (Z)((a != (Z)0) || (b != (Z)0)), true, true)
GRB_MULT(OP_FIRSTI,  (Z)i, false, false)
GRB_MULT(OP_FIRSTJ,  (Z)k, false, false)
GRB_MULT(OP_SECONDI, (Z)k, false, false)
GRB_MULT(OP_SECONDJ, (Z)j, false, false)
#undef GRB_MULT

// The additive monoid.
//   add(z,t):    the monoid's operator, used by the dot-product fold
//                (GB_MULTADD / GB_ADD of the factory kernels)
//   update(z,t): the saxpy coarse-task update Hx[i] += t (GB_UPDATE), which
//                for floating MIN/MAX skips NaN and keeps z when z <= t
//   exact:       true when the result does not depend on the order of the
//                terms (integer wrap-around +,*; min/max; logical ops), so
//                parallel atomic accumulation is bit-exact
template <int ADD, typename Z> struct Monoid;

template <typename Z> struct Monoid<OP_PLUS, Z> {
    static constexpr bool exact = !(std::is_floating_point<Z>::value);
    static constexpr bool any = false;
    __device__ __forceinline__ static Z identity() { return (Z)0; }
    __device__ __forceinline__ static Z add(Z z, Z t) { return rn_add<Z>(z, t); }
    __device__ __forceinline__ static Z update(Z z, Z t) { return rn_add<Z>(z, t); }
};
template <typename Z> struct Monoid<OP_TIMES, Z> {
    static constexpr bool exact = !(std::is_floating_point<Z>::value);
    static constexpr bool any = false;
    __device__ __forceinline__ static Z identity() { return (Z)1; }
    __device__ __forceinline__ static Z add(Z z, Z t) { return rn_mul<Z>(z, t); }
    __device__ __forceinline__ static Z update(Z z, Z t) { return rn_mul<Z>(z, t); }
};
template <typename Z> struct Monoid<OP_MIN, Z> {
    static constexpr bool exact = true;
    static constexpr bool any = false;
    __device__ __forceinline__ static Z identity() {
        if constexpr (std::is_floating_point<Z>::value) return (Z)INFINITY;
        else if constexpr (std::is_same<Z, int32_t>::value) return (Z)INT32_MAX;
        else if constexpr (std::is_same<Z, bool>::value) return true;
        else return (Z)INT64_MAX;
    }
    __device__ __forceinline__ static Z add(Z z, Z t) { return op_min<Z>(z, t); }
    __device__ __forceinline__ static Z update(Z z, Z t) {
        if constexpr (std::is_floating_point<Z>::value) {
            // GB_UPDATE of GB_AxB__min_plus_fp32.c:22
            if (!isnan((double)t) && !(z <= t)) z = t;
            return z;
        }
        return t < z ? t : z;
    }
};
template <typename Z> struct Monoid<OP_MAX, Z> {
    static constexpr bool exact = true;
    static constexpr bool any = false;
    __device__ __forceinline__ static Z identity() {
        if constexpr (std::is_floating_point<Z>::value) return (Z)(-INFINITY);
        else if constexpr (std::is_same<Z, int32_t>::value) return (Z)INT32_MIN;
        else if constexpr (std::is_same<Z, bool>::value) return false;
        else return (Z)INT64_MIN;
    }
    __device__ __forceinline__ static Z add(Z z, Z t) { return op_max<Z>(z, t); }
    __device__ __forceinline__ static Z update(Z z, Z t) {
        if constexpr (std::is_floating_point<Z>::value) {
            if (!isnan((double)t) && !(z >= t)) z = t;
            return z;
        }
        return t > z ? t : z;
    }
};
template <typename Z> struct Monoid<OP_ANY, Z> {
    // saxpy: the last contribution in ascending k wins (GB_UPDATE z = t);
    // dot3: the first match ends the dot product (terminal monoid)
    static constexpr bool exact = false;
    static constexpr bool any = true;
    __device__ __forceinline__ static Z identity() { return (Z)0; }
    __device__ __forceinline__ static Z add(Z z, Z t) { return t; }
    __device__ __forceinline__ static Z update(Z z, Z t) { return t; }
};
template <typename Z> struct Monoid<OP_LOR, Z> {
    static constexpr bool exact = true;
    static constexpr bool any = false;
    __device__ __forceinline__ static Z identity() { return (Z)0; }
    __device__ __forceinline__ static Z add(Z z, Z t) { return (Z)(z || t); }
    __device__ __forceinline__ static Z update(Z z, Z t) { return (Z)(z || t); }
};
template <typename Z> struct Monoid<OP_LAND, Z> {
    static constexpr bool exact = true;
    static constexpr bool any = false;
    __device__ __forceinline__ static Z identity() { return (Z)1; }
    __device__ __forceinline__ static Z add(Z z, Z t) { return (Z)(z && t); }
    __device__ __forceinline__ static Z update(Z z, Z t) { return (Z)(z && t); }
};

template <int ADD, int MULT, typename Z> struct Semiring {
    using z_t = Z;
    using M = Monoid<ADD, Z>;
    using F = Mult<MULT, Z>;
    static constexpr int add_op = ADD, mult_op = MULT;
    static constexpr bool needs_a = F::needs_a, needs_b = F::needs_b;
    // ANY with a multiplier whose value is k (FIRSTJ / SECONDI): "last k
    // wins" equals "max k", computable in any order
    static constexpr bool any_max_k = M::any && (MULT == OP_FIRSTJ || MULT == OP_SECONDI);
    // ANY with a multiplier whose value does not depend on k: every term is
    // equal, so any order gives the same result
    static constexpr bool any_const = M::any &&
        (MULT == OP_PAIR || MULT == OP_FIRSTI || MULT == OP_SECONDJ);
    static constexpr bool order_free = M::exact || any_max_k || any_const;
};

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------

// first position p in [lo,hi) with a[p] >= key
__device__ __forceinline__ int32_t lower_bound(const int32_t *a, int32_t lo,
                                               int32_t hi, int32_t key)
{
    while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// the largest r in [0, n] with a[r] <= key (a nondecreasing, a[0] <= key),
// found by the 32 lanes of a warp together: each step probes 32 evenly
// spaced entries at once and keeps the gap that holds key, so a million
// entries take four dependent loads instead of twenty.  All lanes call it
// with the same arguments and get the same result.
template <typename T, typename I>
__device__ __forceinline__ I warp_last_le(const T *__restrict__ a, I n, T key, int lane)
{
    I lo = 0, hi = n;                              // a[lo] <= key; the answer is in [lo, hi]
    while (lo < hi) {
        const I step = (hi - lo + 31) / 32;
        const I p = lo + (I)(lane + 1) * step;
        const bool le = p <= hi && a[p] <= key;
        const int k = __popc(__ballot_sync(0xffffffffu, le));
        const I nhi = lo + (I)(k + 1) * step - 1;
        lo = lo + (I)k * step;
        hi = nhi < hi ? nhi : hi;
    }
    return lo;
}

// first position p in [lo,hi) with a[p] > key
__device__ __forceinline__ int32_t upper_bound(const int32_t *a, int32_t lo,
                                               int32_t hi, int32_t key)
{
    while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (a[mid] <= key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <typename T> __device__ __forceinline__ T ld_val(const void *x, int64_t p, bool iso)
{
    return reinterpret_cast<const T *>(x)[iso ? 0 : p];
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// warp shuffles for every value type (bool travels as int)
template <typename T> __device__ __forceinline__ T shfl(T v, int src)
{ return __shfl_sync(0xffffffffu, v, src); }
template <> __device__ __forceinline__ bool shfl(bool v, int src)
{ return __shfl_sync(0xffffffffu, (int)v, src) != 0; }
template <typename T> __device__ __forceinline__ T shfl_down(T v, int o)
{ return __shfl_down_sync(0xffffffffu, v, o); }
template <> __device__ __forceinline__ bool shfl_down(bool v, int o)
{ return __shfl_down_sync(0xffffffffu, (int)v, o) != 0; }

}  // namespace grb
