// grb_runtime.h: host-side runtime of the B200 SpGEMM library (C++).
//
// One process drives one device.  Device memory comes from the stream-ordered
// pool (cudaMallocAsync) with a release threshold that keeps freed blocks
// cached, so repeated calls do not return memory to the driver.  Every public
// call runs on a stream taken from a small pool and synchronises before it
// returns, as the reference's GPU gateway does (CUDA/GB_cuda_AxB_dot3.cpp:54,
// one stream per call, synchronised at the end).

#pragma once
#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>
#include "grb_common.cuh"

namespace grb {

struct Runtime {
    int device = 0;
    int num_sms = 148;
    size_t smem_optin = 0;        // max dynamic shared memory per block
    bool ready = false;
};

Runtime &runtime();

// initialise the device (idempotent); returns an Info code.  Sets the
// release threshold of the device's default memory pool to "never".
int init_device();

// the current device's SM count (cached), touching no other device state
int device_sm_count(int *nsm);

// stream pool: acquire/release a non-blocking stream
cudaStream_t stream_acquire();
void stream_release(cudaStream_t s);

// a caller-chosen stream for this host thread (nullptr: use the pool)
void set_thread_stream(cudaStream_t s);
cudaStream_t thread_stream();

// kernel timing with CUDA events on the launching stream (off by default):
// prof_begin/prof_end bracket a launch; prof_flush, called after the stream
// is synchronised, adds the elapsed time to the kernel's running total
void prof_enable(bool on);
void prof_select(const char *name, int every);   // name null: every kernel
bool prof_on();
int prof_begin(const char *name, cudaStream_t s);
void prof_end(int slot, cudaStream_t s);
void prof_flush();
void prof_reset();
bool prof_read(const char *name, double *ms, int64_t *count);

// stream-ordered allocation; returns nullptr on failure (and records it)
void *dalloc(size_t bytes, cudaStream_t s);
void dfree(void *p, cudaStream_t s);

// A scratch buffer owned by a stream, kept between calls (work on the stream
// is ordered, so the stream's calls can share it without a synchronisation),
// for streams the library owns: the pool's, and those a component enables
// (and releases before destroying the stream).  stream_scratch grows it to
// at least min_bytes (the old buffer is released in stream order) and gives
// its size in *bytes; nullptr if the allocation fails or the stream has no
// scratch (a caller's stream: the caller then allocates for the call).
void stream_scratch_enable(cudaStream_t s);
bool stream_scratch_enabled(cudaStream_t s);
void *stream_scratch(cudaStream_t s, size_t min_bytes, size_t *bytes);
size_t stream_scratch_size(cudaStream_t s);
void stream_scratch_release(cudaStream_t s);

// copy `bytes` (at most a few KB) from the device after the stream's work,
// synchronising the stream; returns its error
cudaError_t readback(void *dst, const void *src, size_t bytes, cudaStream_t s);

// host-side allocation fault injection (the reference's malloc_debug
// counter, Source/global/GB_Global.c:83-93): when armed with n > 0, the n-th
// following device allocation fails.  0 disarms.
void set_alloc_fail_countdown(int64_t n);

// map a CUDA error to the reference's convention (CUDA/include/
// GB_cuda_error.hpp:22-35): out of memory -> OUT_OF_MEMORY, else PANIC
int cuda_to_info(cudaError_t e);

// One device allocation carved into 256-byte aligned pieces.  The caller
// lays its buffers out twice with the same take() calls: a sizing pass
// (take() returns null), then, after alloc(), the pass that hands out the
// pieces.  One allocation and one free replace one pair per buffer: the
// stream-ordered allocator's host cost dominates small calls.
struct Carve {
    cudaStream_t s;
    char *base = nullptr;
    size_t off = 0;
    explicit Carve(cudaStream_t st) : s(st) {}
    template <typename T> T *take(size_t count) {
        const size_t o = (off + 255) & ~(size_t)255;
        off = o + count * sizeof(T);
        return base ? reinterpret_cast<T *>(base + o) : nullptr;
    }
    bool alloc() {
        base = (char *)dalloc(off ? off : 16, s);
        off = 0;
        return base != nullptr;
    }
};

// A call's scratch block: the stream's scratch buffer when the library owns
// the stream (kept between calls, so a call of the same size allocates
// nothing), else an allocation for this call, released with the block.
struct CallBlock {
    cudaStream_t s;
    char *base = nullptr;
    bool own = false;
    explicit CallBlock(cudaStream_t st) : s(st) {}
    bool get(size_t bytes)
    {
        if (bytes == 0) bytes = 16;
        if (stream_scratch_enabled(s)) {
            base = (char *)stream_scratch(s, bytes, nullptr);
            own = false;
        } else {
            base = (char *)dalloc(bytes, s);
            own = true;
        }
        return base != nullptr;
    }
    ~CallBlock() { if (own) dfree(base, s); }
};

// scratch buffers that live for one call on one stream
struct Scratch {
    cudaStream_t s;
    void *ptrs[64];
    int n = 0;
    bool failed = false;
    explicit Scratch(cudaStream_t st) : s(st) {}
    template <typename T> T *get(size_t count) {
        if (n >= 64) { failed = true; return nullptr; }
        void *p = dalloc(count * sizeof(T) + 16, s);
        if (!p) { failed = true; return nullptr; }
        ptrs[n++] = p;
        return reinterpret_cast<T *>(p);
    }
    ~Scratch() { for (int i = 0; i < n; i++) dfree(ptrs[i], s); }
};

// ---- device matrix management ----
void dev_free(DevCSR &A, cudaStream_t s);

// upload a host CSR (int64 p/i as in GB_matrix.h) into a DevCSR (int32)
int dev_upload(DevCSR &A, int64_t nrows, int64_t ncols, const int64_t *p,
               const int64_t *i, const void *x, int type, bool iso,
               cudaStream_t s);

// download a DevCSR to host int64 arrays allocated with `alloc`; zombies are
// kept as flipped indices when keep_zombies, else they are removed
typedef void *(*alloc_fn)(size_t);
int dev_download(const DevCSR &A, int64_t **p, int64_t **i, void **x,
                 bool keep_zombies, alloc_fn alloc, cudaStream_t s);

// structural copy of a valued mask: entries whose value is false dropped
int dev_mask_to_struct(DevCSR &out, const DevCSR &M, cudaStream_t s);

// remove zombies in place (GB_wait's zombie pruning), producing a clean CSR
int dev_prune_zombies(DevCSR &A, cudaStream_t s);

// upload from the caller's int64 CSR with checks on the device (offsets from
// 0 to nnz, never decreasing; indices in [0, ncols); rows given out of order
// are sorted, duplicates rejected): INVALID_OBJECT when the arrays are not a
// matrix (GrB_Matrix_import's secure import)
int dev_import(DevCSR &A, int64_t nrows, int64_t ncols, const int64_t *p,
               const int64_t *i, const void *x, int type, cudaStream_t s);

// copy the live entries into the caller's arrays (nrows+1 offsets, then the
// live indices and values; iso values expanded); synchronises s
int dev_download_to(const DevCSR &A, int64_t *p, int64_t *i, void *x, cudaStream_t s);

// copy every entry (zombies kept as flipped indices) into the caller's
// arrays (nrows+1 offsets, nnz indices, and nnz values unless x is null;
// iso values expanded); synchronises s
int dev_copy_out(const DevCSR &A, int64_t *p, int64_t *i, void *x, cudaStream_t s);

// ---- scans ----
// exclusive scan of n int64 values in place; out[n] receives the total when
// `with_total`.  `in` and `out` may alias.
int scan_exclusive_i64(const int64_t *in, int64_t *out, int64_t n,
                       cudaStream_t s);
int scan_exclusive_i32_to_i64(const int32_t *in, int64_t *out, int64_t n,
                              cudaStream_t s);
// allocation-free variant: ws holds scan_ws_elems(n) int64 values
size_t scan_ws_elems(int64_t n);
static constexpr int64_t SCAN_SINGLE_MAX = 8192;
// Arrays of at most SCAN_SINGLE_MAX elements are scanned by one launch of one
// block.  total (device, may be null) receives the sum of all n inputs;
// out32 (may be null) receives the offsets narrowed to int32 as well.
void scan_exclusive_i64_ws(const int64_t *in, int64_t *out, int64_t n, int64_t *ws,
                           cudaStream_t s, int64_t *total = nullptr,
                           int32_t *out32 = nullptr);

// The same exclusive scan as one launch for any length (decoupled
// look-back; up to 8192 values it is the single-block scan).  ws holds
// scan_lb_ws_elems(n) words that are zero before the first use; every
// scan leaves them zero again.  *err (may be null) is set if a tile's wait
// for its predecessors passes its bound.  in may equal out.
size_t scan_lb_ws_elems(int64_t n);
void scan_exclusive_lb(const int64_t *in, int64_t *out, int64_t n, unsigned long long *ws,
                       cudaStream_t s, int64_t *total = nullptr, int32_t *out32 = nullptr,
                       int *err = nullptr);
// The same over n + 1 values taken from int32 counts: value i is cnt[i]
// where keep[i] is non-zero (every i when keep is null), else 0, and value n
// is 0 (row counts to row offsets, rows outside every bin counting 0).
// Always the look-back kernel.
void scan_exclusive_lb_counts(const int32_t *cnt, const int8_t *keep, int64_t n,
                              int64_t *out, unsigned long long *ws, cudaStream_t s,
                              int64_t *total, int32_t *out32, int *err);

// ---- operations (device matrices) ----

struct SemiringCode { int add, mult, type; };

// C<M> = A*B' by dot products over M's pattern (Source/mxm/GB_AxB_dot3.c:37).
// C gets M's pattern with zombies for empty dot products.  live_sum (may be
// null) receives the sum of C's live entries for the counting semirings
// (PLUS_PAIR on integers; wrapping int64 adds), 0 for the others.
int dot3(DevCSR &C, const DevCSR &M, bool mask_struct, const DevCSR &A,
         const DevCSR &B, SemiringCode sr, cudaStream_t s, int64_t *live_sum = nullptr);

// C<M> = A*B row by row (Source/mxm/GB_AxB_saxpy3.c:119); M may be null.
// Output rows are sorted, no zombies.
int saxpy3(DevCSR &C, const DevCSR *M, bool mask_comp, bool mask_struct,
           const DevCSR &A, const DevCSR &B, SemiringCode sr, cudaStream_t s);

// s = reduce(A) with a monoid over live entries (zombies skipped)
// (Source/reduce/GB_reduce_to_scalar.c:41); result written to host *out
int reduce_scalar(void *out, const DevCSR &A, int monoid, cudaStream_t s);

// C<M,replace> = accum(C,T)  (Source/mask/GB_accum_mask.c:126)
int accum_mask(DevCSR &C, const DevCSR &T, const DevCSR *M, bool mask_comp,
               bool mask_struct, bool replace, int accum, cudaStream_t s);

// B = A' (Source/transpose/GB_transpose_cast.c:18)
int transpose(DevCSR &B, const DevCSR &A, cudaStream_t s);

// w<m> = A*u, u and w sparse 1-by-n rows (GrB_mxv, Source/mxm/GrB_mxv.c:18)
int mxv(DevCSR &w, const DevCSR *mask, bool mask_comp, bool mask_struct,
        const DevCSR &A, const DevCSR &u, SemiringCode sr, cudaStream_t s);

// supported semiring?  (declines with NO_VALUE otherwise)
bool semiring_supported(SemiringCode sr);

}  // namespace grb
