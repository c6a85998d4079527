// grb_runtime.cu: device init, stream pool, stream-ordered memory, CSR
// upload/download, scans and zombie pruning for the B200 SpGEMM library.

#include <mutex>
#include <string>
#include <vector>
#include <atomic>
#include <cstring>
#include <cstdio>
#include "grb_runtime.h"
#include "grb_lookback.cuh"

namespace grb {

static Runtime g_rt;
static std::mutex g_mu;
static std::vector<cudaStream_t> g_streams;
static std::atomic<int64_t> g_fail_countdown{0};

Runtime &runtime() { return g_rt; }

int cuda_to_info(cudaError_t e)
{
    if (e == cudaSuccess) return SUCCESS;
    if (e == cudaErrorMemoryAllocation) return OUT_OF_MEMORY;
    return PANIC;
}

// The device's SM count, read once per process, without the pool setting
// that init_device makes: callers that must leave the device's memory state
// alone (the allocation-free entry point) use this instead.
int device_sm_count(int *nsm)
{
    static std::atomic<int> cached[128];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 128) { cudaGetLastError(); return PANIC; }
    int v = cached[dev].load();
    if (v <= 0) {
        e = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || v <= 0) { cudaGetLastError(); return PANIC; }
        cached[dev].store(v);
    }
    *nsm = v;
    return SUCCESS;
}

int init_device()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_rt.ready) return SUCCESS;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) { cudaGetLastError(); return PANIC; }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return PANIC;
    g_rt.device = dev;
    g_rt.num_sms = prop.multiProcessorCount;
    g_rt.smem_optin = prop.sharedMemPerBlockOptin;
    // keep freed pool memory cached instead of returning it to the driver
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thresh = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh);
    }
    g_rt.ready = true;
    return SUCCESS;
}

cudaStream_t stream_acquire()
{
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_streams.empty()) {
            cudaStream_t s = g_streams.back();
            g_streams.pop_back();
            return s;
        }
    }
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return nullptr;
    stream_scratch_enable(s);      // the pool's streams live as long as the library
    return s;
}

void stream_release(cudaStream_t s)
{
    if (!s) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_streams.push_back(s);
}

void set_alloc_fail_countdown(int64_t n) { g_fail_countdown.store(n); }

// per-stream scratch buffers
struct StreamScratch { cudaStream_t s; void *p; size_t bytes; };
static std::mutex g_scratch_mu;
static std::vector<StreamScratch> g_scratch;

void stream_scratch_enable(cudaStream_t s)
{
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    for (auto &x : g_scratch)
        if (x.s == s) return;
    g_scratch.push_back({s, nullptr, 0});
}

bool stream_scratch_enabled(cudaStream_t s)
{
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    for (auto &x : g_scratch)
        if (x.s == s) return true;
    return false;
}

void *stream_scratch(cudaStream_t s, size_t min_bytes, size_t *bytes)
{
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    StreamScratch *e = nullptr;
    for (auto &x : g_scratch)
        if (x.s == s) { e = &x; break; }
    if (!e) { if (bytes) *bytes = 0; return nullptr; }
    if (e->bytes < min_bytes || !e->p) {
        dfree(e->p, s);
        e->p = nullptr;
        e->bytes = 0;
        size_t want = min_bytes < 4096 ? 4096 : min_bytes;
        void *p = dalloc(want, s);
        if (!p) { if (bytes) *bytes = 0; return nullptr; }
        e->p = p;
        e->bytes = want;
    }
    if (bytes) *bytes = e->bytes;
    return e->p;
}

size_t stream_scratch_size(cudaStream_t s)
{
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    for (auto &x : g_scratch)
        if (x.s == s) return x.p ? x.bytes : 0;
    return 0;
}

void stream_scratch_release(cudaStream_t s)
{
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    for (size_t k = 0; k < g_scratch.size(); k++) {
        if (g_scratch[k].s != s) continue;
        dfree(g_scratch[k].p, s);
        g_scratch[k] = g_scratch.back();
        g_scratch.pop_back();
        return;
    }
}

static thread_local cudaStream_t t_stream = nullptr;
void set_thread_stream(cudaStream_t s) { t_stream = s; }
cudaStream_t thread_stream() { return t_stream; }

// ---------------------------------------------------------------------------
// kernel timing
// ---------------------------------------------------------------------------

struct ProfPending { const char *name; cudaEvent_t a, b; int dev; };
struct ProfTotal { const char *name; double ms; int64_t count; };
struct ProfEvent { cudaEvent_t e; int dev; };
static std::atomic<bool> g_prof{false};
static std::mutex g_prof_mu;
static std::vector<ProfPending> g_pending;
static std::vector<ProfTotal> g_totals;
// events are kept for reuse (creating two per range would cost more host
// time than the launches the range brackets)
static std::vector<ProfEvent> g_free_events;
// the kernel whose ranges are recorded (empty: all) and one range in every
static std::string g_prof_name;
static int g_prof_every = 1;
static uint64_t g_prof_seen = 0;

void prof_select(const char *name, int every)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_name = name ? name : "";
    g_prof_every = every < 1 ? 1 : every;
    g_prof_seen = 0;
}

bool prof_on() { return g_prof.load(); }

// an event of device dev from the pool, or a new one; g_prof_mu held
static cudaEvent_t prof_event(int dev)
{
    for (size_t q = g_free_events.size(); q-- > 0;) {
        if (g_free_events[q].dev == dev) {
            const cudaEvent_t e = g_free_events[q].e;
            g_free_events.erase(g_free_events.begin() + q);
            return e;
        }
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); e = nullptr; }
    return e;
}

// Turning ranges on fills the current device's share of the pool to 256
// events, so that ranges opened in a timed loop create none.
void prof_enable(bool on)
{
    if (on) {
        int dev = 0;
        cudaGetDevice(&dev);
        std::lock_guard<std::mutex> lk(g_prof_mu);
        int have = 0;
        for (const ProfEvent &e : g_free_events) have += e.dev == dev;
        for (; have < 256; have++) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); break; }
            g_free_events.push_back({e, dev});
        }
    }
    g_prof.store(on);
}

int prof_begin(const char *name, cudaStream_t s)
{
    if (!g_prof.load()) return -1;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof_name.empty() && g_prof_name != name) return -1;
    if (g_prof_seen++ % (uint64_t)g_prof_every != 0) return -1;
    ProfPending p{name, prof_event(dev), prof_event(dev), dev};
    if (!p.a || !p.b) {
        if (p.a) g_free_events.push_back({p.a, dev});
        if (p.b) g_free_events.push_back({p.b, dev});
        return -1;
    }
    cudaEventRecord(p.a, s);
    g_pending.push_back(p);
    return (int)g_pending.size() - 1;
}

void prof_end(int slot, cudaStream_t s)
{
    if (slot < 0) return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (slot < (int)g_pending.size()) cudaEventRecord(g_pending[slot].b, s);
}

void prof_flush()
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto &p : g_pending) {
        float ms = 0.0f;
        cudaEventSynchronize(p.b);
        if (cudaEventElapsedTime(&ms, p.a, p.b) != cudaSuccess) { cudaGetLastError(); ms = 0; }
        bool found = false;
        for (auto &t : g_totals)
            if (strcmp(t.name, p.name) == 0) { t.ms += ms; t.count++; found = true; break; }
        if (!found) g_totals.push_back({p.name, (double)ms, 1});
        g_free_events.push_back({p.a, p.dev});
        g_free_events.push_back({p.b, p.dev});
    }
    g_pending.clear();
}

void prof_reset()
{
    prof_flush();
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_totals.clear();
}

bool prof_read(const char *name, double *ms, int64_t *count)
{
    prof_flush();
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto &t : g_totals)
        if (strcmp(t.name, name) == 0) { *ms = t.ms; *count = t.count; return true; }
    *ms = 0; *count = 0;
    return false;
}

void *dalloc(size_t bytes, cudaStream_t s)
{
    int64_t c = g_fail_countdown.load();
    if (c > 0) {
        int64_t left = g_fail_countdown.fetch_sub(1) - 1;
        if (left == 0) return nullptr;          // injected failure
    }
    if (bytes == 0) bytes = 16;
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, s);
    if (e != cudaSuccess) { cudaGetLastError(); return nullptr; }
    return p;
}

void dfree(void *p, cudaStream_t s)
{
    if (p) cudaFreeAsync(p, s);
}

// The few bytes a call reads back (bin counts, totals, zombie counts) go
// through a page-locked, device-mapped buffer of the calling host thread,
// written by a one-block kernel queued behind the call's last kernel: a
// kernel that follows a kernel on the same stream starts within a
// microsecond or two, where a copy-engine transfer first waits for the
// compute engine's completion (several microseconds more per read).
static constexpr size_t READBACK_MAX = 4096;

__global__ void k_readback(const unsigned char *__restrict__ src, unsigned char *dst,
                           uint32_t bytes)
{
    const bool words = ((((uintptr_t)src) | ((uintptr_t)dst) | bytes) & 3) == 0;
    if (words) {
        const uint32_t *s4 = reinterpret_cast<const uint32_t *>(src);
        uint32_t *d4 = reinterpret_cast<uint32_t *>(dst);
        for (uint32_t q = threadIdx.x; q < bytes / 4; q += blockDim.x) d4[q] = s4[q];
    } else {
        for (uint32_t q = threadIdx.x; q < bytes; q += blockDim.x) dst[q] = src[q];
    }
    __threadfence_system();
}

// A thread takes a buffer from a shared pool on first use and puts it back
// when it exits, so the worker threads a server starts for each replay reuse
// the same few buffers (page-locking memory, and unlocking it, is slow).
struct ReadbackPage { void *host = nullptr, *dev = nullptr; };
static std::mutex g_rb_mu;
static std::vector<ReadbackPage> g_rb_pool;

struct ReadbackBuffer {
    ReadbackPage pg;
    ~ReadbackBuffer() {
        if (pg.host) {
            std::lock_guard<std::mutex> lk(g_rb_mu);
            g_rb_pool.push_back(pg);
        }
    }
};

cudaError_t readback(void *dst, const void *src, size_t bytes, cudaStream_t s)
{
    thread_local ReadbackBuffer rb;
    ReadbackPage &pg = rb.pg;
    if (!pg.host && bytes <= READBACK_MAX) {
        {
            std::lock_guard<std::mutex> lk(g_rb_mu);
            if (!g_rb_pool.empty()) {
                pg = g_rb_pool.back();
                g_rb_pool.pop_back();
            }
        }
        if (!pg.host) {
            void *h = nullptr, *d = nullptr;
            if (cudaHostAlloc(&h, READBACK_MAX, cudaHostAllocMapped | cudaHostAllocPortable) !=
                cudaSuccess) {
                cudaGetLastError();
            } else if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
                cudaGetLastError();
                cudaFreeHost(h);
            } else {
                pg.host = h;
                pg.dev = d;
            }
        }
    }
    // a copy refused at submission leaves nothing for the synchronise to
    // report, so its own status is checked first (the bytes are not read)
    if (!pg.host || bytes > READBACK_MAX) {
        const cudaError_t c = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
        if (c != cudaSuccess) return c;
        return cudaStreamSynchronize(s);
    }
    if (bytes == 0) return cudaStreamSynchronize(s);
    k_readback<<<1, 128, 0, s>>>((const unsigned char *)src, (unsigned char *)pg.dev,
                                 (uint32_t)bytes);
    const cudaError_t c = cudaGetLastError();
    if (c != cudaSuccess) return c;
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) memcpy(dst, pg.host, bytes);
    return e;
}

void dev_free(DevCSR &A, cudaStream_t s)
{
    dfree(A.p, s); dfree(A.j, s); dfree(A.x, s);
    A.p = nullptr; A.j = nullptr; A.x = nullptr;
    A.nnz = 0; A.nzombies = 0;
}

// ---------------------------------------------------------------------------
// narrowing / widening copies
// ---------------------------------------------------------------------------

__global__ void k_narrow(const int64_t *__restrict__ in, int32_t *__restrict__ out,
                         int64_t n)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < n; t += stride) out[t] = (int32_t)in[t];
}

__global__ void k_widen(const int32_t *__restrict__ in, int64_t *__restrict__ out,
                        int64_t n)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < n; t += stride) out[t] = (int64_t)in[t];
}

static inline int grid_for(int64_t n, int threads)
{
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)runtime().num_sms * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

int dev_upload(DevCSR &A, int64_t nrows, int64_t ncols, const int64_t *p,
               const int64_t *i, const void *x, int type, bool iso,
               cudaStream_t s)
{
    int64_t nnz = p[nrows];
    if (nrows >= INT32_MAX || ncols >= INT32_MAX || nnz >= INT32_MAX)
        return NO_VALUE;
    A.nrows = nrows; A.ncols = ncols; A.nnz = nnz; A.type = type; A.iso = iso;
    A.nzombies = 0;
    size_t ts = type_size(type);
    // stage int64 arrays through one device buffer (the stream's scratch
    // buffer when the library owns the stream), then narrow on the device
    int64_t stage_n = (nrows + 1 > nnz) ? nrows + 1 : nnz;
    const bool shared = stream_scratch_enabled(s);
    int64_t *stage = shared ? (int64_t *)stream_scratch(s, (size_t)stage_n * 8, nullptr)
                            : (int64_t *)dalloc((size_t)stage_n * 8, s);
    A.p = (int32_t *)dalloc((size_t)(nrows + 1) * 4, s);
    A.j = (int32_t *)dalloc((size_t)(nnz ? nnz : 1) * 4, s);
    A.x = nullptr;
    if (x) A.x = dalloc(iso ? ts : (size_t)(nnz ? nnz : 1) * ts, s);
    if (!stage || !A.p || !A.j || (x && !A.x)) {
        if (!shared) dfree(stage, s);
        dev_free(A, s);
        return OUT_OF_MEMORY;
    }
    cudaMemcpyAsync(stage, p, (size_t)(nrows + 1) * 8, cudaMemcpyHostToDevice, s);
    k_narrow<<<grid_for(nrows + 1, 256), 256, 0, s>>>(stage, A.p, nrows + 1);
    if (nnz > 0) {
        cudaMemcpyAsync(stage, i, (size_t)nnz * 8, cudaMemcpyHostToDevice, s);
        k_narrow<<<grid_for(nnz, 256), 256, 0, s>>>(stage, A.j, nnz);
    }
    if (x) cudaMemcpyAsync(A.x, x, iso ? ts : (size_t)nnz * ts,
                           cudaMemcpyHostToDevice, s);
    if (!shared) dfree(stage, s);
    return cuda_to_info(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// import with checks, and export into the caller's arrays
// ---------------------------------------------------------------------------

// narrow with a range check: flag |= bit for a value outside [lo, hi], or,
// for offsets (monotone), a value above its successor
__global__ void k_narrow_check(const int64_t *__restrict__ in, int32_t *__restrict__ out,
                               int64_t n, int64_t lo, int64_t hi, bool monotone,
                               unsigned *__restrict__ flag, unsigned bit)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    bool bad = false;
    for (; t < n; t += stride) {
        const int64_t v = in[t];
        bad |= v < lo || v > hi || (monotone && t + 1 < n && in[t + 1] < v);
        out[t] = (int32_t)v;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, bit);
}

// bit p[r] of `starts` marks the first entry of every non-empty row r
__global__ void k_row_starts(const int32_t *__restrict__ Ap, int64_t nrows, int64_t nnz,
                             unsigned *__restrict__ starts)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t q = Ap[r];
        // offsets not yet known to be valid stay inside the bitmap
        if (q >= 0 && q < Ap[r + 1] && q < nnz) atomicOr(&starts[q >> 5], 1u << (q & 31));
    }
}

// flag |= bit when an entry that does not start a row is not above the one
// before it (rows not strictly increasing), flat and coalesced over entries
__global__ void k_check_rows(const int32_t *__restrict__ Aj, int64_t nnz,
                             const unsigned *__restrict__ starts,
                             unsigned *__restrict__ flag, unsigned bit)
{
    bool bad = false;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; q < nnz;
         q += (int64_t)gridDim.x * blockDim.x) {
        if (!((starts[q >> 5] >> (q & 31)) & 1u)) bad |= Aj[q - 1] >= Aj[q];
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, bit);
}

// are the rows of A strictly increasing?  (flag bit set when not)
static void check_rows(const DevCSR &A, unsigned *starts, unsigned *flag, unsigned bit,
                       cudaStream_t s)
{
    cudaMemsetAsync(starts, 0, (size_t)((A.nnz + 31) / 32) * 4, s);
    k_row_starts<<<grid_for(A.nrows, 256), 256, 0, s>>>(A.p, A.nrows, A.nnz, starts);
    k_check_rows<<<grid_for(A.nnz, 256), 256, 0, s>>>(A.j, A.nnz, starts, flag, bit);
}

int dev_import(DevCSR &A, int64_t nrows, int64_t ncols, const int64_t *p,
               const int64_t *i, const void *x, int type, cudaStream_t s)
{
    if (nrows < 0 || ncols < 0) return INVALID_VALUE;
    const int64_t nnz = p[nrows];
    if (p[0] != 0 || nnz < 0) return INVALID_OBJECT;
    if (nrows >= INT32_MAX || ncols >= INT32_MAX || nnz >= INT32_MAX) return NO_VALUE;
    A = DevCSR();
    A.nrows = nrows; A.ncols = ncols; A.nnz = nnz; A.type = type; A.iso = false;
    const size_t ts = type_size(type);
    // the staging array, the error flag and the row-start bitmap in one
    // block (the stream's scratch buffer when the stream keeps one)
    Carve cv(s);
    int64_t *stage = nullptr;
    unsigned *flag = nullptr, *starts = nullptr;
    auto layout = [&]() {
        flag = cv.take<unsigned>(1);
        starts = cv.take<unsigned>((nnz + 31) / 32 + 1);
        stage = cv.take<int64_t>((nrows + 1 > nnz) ? nrows + 1 : nnz);
    };
    layout();
    CallBlock blk(s);
    const bool got = blk.get(cv.off);
    cv.base = blk.base;
    cv.off = 0;
    layout();
    A.p = (int32_t *)dalloc((size_t)(nrows + 1) * 4, s);
    A.j = (int32_t *)dalloc((size_t)(nnz ? nnz : 1) * 4, s);
    A.x = dalloc((size_t)(nnz ? nnz : 1) * ts, s);
    if (!got || !A.p || !A.j || !A.x) { dev_free(A, s); return OUT_OF_MEMORY; }
    cudaMemsetAsync(flag, 0, 4, s);
    cudaMemcpyAsync(stage, p, (size_t)(nrows + 1) * 8, cudaMemcpyHostToDevice, s);
    k_narrow_check<<<grid_for(nrows + 1, 256), 256, 0, s>>>(stage, A.p, nrows + 1, 0, nnz,
                                                            true, flag, 1u);
    if (nnz > 0) {
        cudaMemcpyAsync(stage, i, (size_t)nnz * 8, cudaMemcpyHostToDevice, s);
        k_narrow_check<<<grid_for(nnz, 256), 256, 0, s>>>(stage, A.j, nnz, 0, ncols - 1,
                                                          false, flag, 2u);
        cudaMemcpyAsync(A.x, x, (size_t)nnz * ts, cudaMemcpyHostToDevice, s);
    }
    unsigned hflag = 0;
    cudaMemcpyAsync(&hflag, flag, 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { dev_free(A, s); return cuda_to_info(e); }
    if (hflag) { dev_free(A, s); return INVALID_OBJECT; }
    if (nnz == 0) return SUCCESS;
    check_rows(A, starts, flag, 4u, s);
    cudaMemcpyAsync(&hflag, flag, 4, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { dev_free(A, s); return cuda_to_info(e); }
    if (hflag == 0) return SUCCESS;
    // rows given out of order: (A')' has every row sorted
    DevCSR T, B;
    int info = transpose(T, A, s);
    if (info == SUCCESS) info = transpose(B, T, s);
    dev_free(T, s);
    dev_free(A, s);
    if (info != SUCCESS) { dev_free(B, s); return info; }
    A = B;
    // a sorted row with two equal indices holds a duplicate: not a matrix
    cudaMemsetAsync(flag, 0, 4, s);
    check_rows(A, starts, flag, 4u, s);
    cudaMemcpyAsync(&hflag, flag, 4, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess || hflag) {
        dev_free(A, s);
        return e != cudaSuccess ? cuda_to_info(e) : INVALID_OBJECT;
    }
    return SUCCESS;
}

template <typename T>
__global__ void k_fill_value(T *__restrict__ out, const T *__restrict__ v, int64_t n)
{
    const T x = *v;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        out[t] = x;
}

// every entry of A as it is (zombies keep their flipped indices) into the
// caller's arrays: nrows+1 offsets, nnz indices and, when x is given, nnz
// values (iso values expanded); synchronises s
int dev_copy_out(const DevCSR &A, int64_t *p, int64_t *i, void *x, cudaStream_t s)
{
    const size_t ts = type_size(A.type);
    const int64_t nnz = A.nnz;
    // the widening stage (and the expanded iso values) in one block: the
    // stream's scratch buffer when the stream keeps one
    const bool expand = x && A.x && A.iso && nnz > 0;
    Carve cv(s);
    int64_t *stage = nullptr;
    char *ex = nullptr;
    auto layout = [&]() {
        stage = cv.take<int64_t>((A.nrows + 1 > nnz) ? A.nrows + 1 : nnz);
        if (expand) ex = cv.take<char>((size_t)nnz * ts);
    };
    layout();
    CallBlock blk(s);
    if (!blk.get(cv.off)) return OUT_OF_MEMORY;
    cv.base = blk.base;
    cv.off = 0;
    layout();
    k_widen<<<grid_for(A.nrows + 1, 256), 256, 0, s>>>(A.p, stage, A.nrows + 1);
    cudaMemcpyAsync(p, stage, (size_t)(A.nrows + 1) * 8, cudaMemcpyDeviceToHost, s);
    if (nnz > 0) {
        k_widen<<<grid_for(nnz, 256), 256, 0, s>>>(A.j, stage, nnz);
        cudaMemcpyAsync(i, stage, (size_t)nnz * 8, cudaMemcpyDeviceToHost, s);
        if (x && A.x) {
            if (ex) {
                // iso values are expanded, one per entry
                switch (ts) {
                    case 1: k_fill_value<uint8_t><<<grid_for(nnz, 256), 256, 0, s>>>(
                                (uint8_t *)ex, (const uint8_t *)A.x, nnz); break;
                    case 4: k_fill_value<uint32_t><<<grid_for(nnz, 256), 256, 0, s>>>(
                                (uint32_t *)ex, (const uint32_t *)A.x, nnz); break;
                    default: k_fill_value<uint64_t><<<grid_for(nnz, 256), 256, 0, s>>>(
                                (uint64_t *)ex, (const uint64_t *)A.x, nnz); break;
                }
                cudaMemcpyAsync(x, ex, (size_t)nnz * ts, cudaMemcpyDeviceToHost, s);
            } else {
                cudaMemcpyAsync(x, A.x, (size_t)nnz * ts, cudaMemcpyDeviceToHost, s);
            }
        }
    }
    return cuda_to_info(cudaStreamSynchronize(s));
}

int dev_download_to(const DevCSR &A0, int64_t *p, int64_t *i, void *x, cudaStream_t s)
{
    if (A0.nzombies == 0) return dev_copy_out(A0, p, i, x, s);
    // prune a private copy so the caller's matrix is untouched
    DevCSR B = A0;
    const size_t ts = type_size(A0.type);
    B.p = (int32_t *)dalloc((size_t)(A0.nrows + 1) * 4, s);
    B.j = (int32_t *)dalloc((size_t)(A0.nnz ? A0.nnz : 1) * 4, s);
    B.x = nullptr;
    if (A0.x) B.x = dalloc(A0.iso ? ts : (size_t)(A0.nnz ? A0.nnz : 1) * ts, s);
    if (!B.p || !B.j || (A0.x && !B.x)) { dev_free(B, s); return OUT_OF_MEMORY; }
    cudaMemcpyAsync(B.p, A0.p, (size_t)(A0.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(B.j, A0.j, (size_t)A0.nnz * 4, cudaMemcpyDeviceToDevice, s);
    if (A0.x) cudaMemcpyAsync(B.x, A0.x, A0.iso ? ts : (size_t)A0.nnz * ts,
                              cudaMemcpyDeviceToDevice, s);
    int info = dev_prune_zombies(B, s);
    if (info == SUCCESS) info = dev_copy_out(B, p, i, x, s);
    dev_free(B, s);
    cudaStreamSynchronize(s);
    return info;
}

// ---------------------------------------------------------------------------
// exclusive scans (three passes: block totals, scan of totals, block scans)
// ---------------------------------------------------------------------------

static constexpr int SCAN_THREADS = 512;
static constexpr int SCAN_ITEMS = 8;
static constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__global__ void k_scan_totals(const T *__restrict__ in, int64_t n,
                              int64_t *__restrict__ totals)
{
    __shared__ int64_t warp_sums[SCAN_THREADS / 32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    int64_t sum = 0;
    for (int it = 0; it < SCAN_ITEMS; it++) {
        int64_t idx = base + (int64_t)it * SCAN_THREADS + threadIdx.x;
        if (idx < n) sum += (int64_t)in[idx];
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x < 32) {
        int64_t v = threadIdx.x < SCAN_THREADS / 32 ? warp_sums[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) totals[blockIdx.x] = v;
    }
}

// scan one tile per block; offsets[b] is the exclusive prefix of the tile;
// total / out32 as in scan_exclusive_i64_ws
template <typename T>
__global__ void k_scan_tiles(const T *__restrict__ in, int64_t *__restrict__ out,
                             int64_t n, const int64_t *__restrict__ offsets,
                             int64_t *__restrict__ total = nullptr,
                             int32_t *__restrict__ out32 = nullptr)
{
    __shared__ int64_t warp_sums[SCAN_THREADS / 32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int64_t v[SCAN_ITEMS];
    int64_t local = 0;
    #pragma unroll
    for (int it = 0; it < SCAN_ITEMS; it++) {
        int64_t idx = base + it;
        v[it] = idx < n ? (int64_t)in[idx] : 0;
        local += v[it];
    }
    // warp inclusive scan of per-thread totals
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t inc = local;
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < SCAN_THREADS / 32 ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_THREADS / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    int64_t prefix = offsets[blockIdx.x] + (warp > 0 ? warp_sums[warp - 1] : 0) +
                     (inc - local);
    #pragma unroll
    for (int it = 0; it < SCAN_ITEMS; it++) {
        int64_t idx = base + it;
        if (idx < n) {
            out[idx] = prefix;
            if (out32) out32[idx] = (int32_t)prefix;
        }
        prefix += v[it];
        if (total && idx == n - 1) *total = prefix;
    }
}

// the whole scan in one block of 1024 threads, tile after tile with a running
// carry (in may equal out: every tile is read before it is written).  A warp
// owns 256 consecutive values as 8 rows of 32: loads and stores are
// coalesced, each row is scanned with shuffles and carried into the next.
static constexpr int SCAN1_THREADS = 1024;
static constexpr int SCAN1_ROWS = 8;
static constexpr int SCAN1_TILE = SCAN1_THREADS * SCAN1_ROWS;

template <typename T>
__global__ void __launch_bounds__(SCAN1_THREADS)
k_scan_single(const T *in, int64_t *out, int64_t n, int64_t *__restrict__ total,
              int32_t *__restrict__ out32)
{
    __shared__ int64_t warp_sums[SCAN1_THREADS / 32];
    __shared__ int64_t tile_sum;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t carry = 0;
    for (int64_t tile = 0; tile < n; tile += SCAN1_TILE) {
        const int64_t base = tile + (int64_t)warp * (32 * SCAN1_ROWS) + lane;
        int64_t v[SCAN1_ROWS];
        #pragma unroll
        for (int r = 0; r < SCAN1_ROWS; r++) {
            const int64_t idx = base + r * 32;
            v[r] = idx < n ? (int64_t)in[idx] : 0;
        }
        // inclusive scan of the warp's 256 values, row by row
        int64_t run = 0;
        #pragma unroll
        for (int r = 0; r < SCAN1_ROWS; r++) {
            int64_t x = v[r];
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            v[r] = run + x - v[r];                  // exclusive within the warp
            run += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) warp_sums[warp] = run;
        __syncthreads();
        if (warp == 0) {
            const int64_t own = warp_sums[lane];
            int64_t w = own;
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w - own;              // exclusive prefix of each warp
        }
        __syncthreads();
        const int64_t wbase = carry + warp_sums[warp];
        #pragma unroll
        for (int r = 0; r < SCAN1_ROWS; r++) {
            const int64_t idx = base + r * 32;
            if (idx < n) {
                const int64_t o = wbase + v[r];
                out[idx] = o;
                if (out32) out32[idx] = (int32_t)o;
            }
        }
        // the tile's sum: the last warp's prefix plus its own run
        if (warp == SCAN1_THREADS / 32 - 1 && lane == 0) tile_sum = warp_sums[warp] + run;
        __syncthreads();
        carry += tile_sum;
    }
    if (total && threadIdx.x == 0) *total = carry;
}

template <typename T>
static int scan_impl(const T *in, int64_t *out, int64_t n, cudaStream_t s)
{
    if (n <= 0) return SUCCESS;
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    int64_t *totals = (int64_t *)dalloc((size_t)(nb + 1) * 8, s);
    if (!totals) return OUT_OF_MEMORY;
    k_scan_totals<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, totals);
    int info = SUCCESS;
    if (nb > 1) info = scan_impl<int64_t>(totals, totals, nb, s);
    else cudaMemsetAsync(totals, 0, 8, s);
    if (info == SUCCESS)
        k_scan_tiles<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, totals);
    dfree(totals, s);
    if (info != SUCCESS) return info;
    return cuda_to_info(cudaGetLastError());
}

int scan_exclusive_i64(const int64_t *in, int64_t *out, int64_t n, cudaStream_t s)
{
    return scan_impl<int64_t>(in, out, n, s);
}

// the same scan with caller-provided workspace (no allocation, no host sync:
// usable inside CUDA graph capture)
size_t scan_ws_elems(int64_t n)
{
    size_t tot = 0;
    while (n > 1) {
        int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
        tot += (size_t)nb + 1;
        if (nb <= 1) break;
        n = nb;
    }
    return tot + 2;
}

template <typename T>
static void scan_ws_impl(const T *in, int64_t *out, int64_t n, int64_t *ws, cudaStream_t s,
                         int64_t *total = nullptr, int32_t *out32 = nullptr)
{
    if (n <= 0) return;
    if (n <= SCAN_SINGLE_MAX) {
        k_scan_single<T><<<1, SCAN1_THREADS, 0, s>>>(in, out, n, total, out32);
        return;
    }
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    int64_t *totals = ws;
    k_scan_totals<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, totals);
    scan_ws_impl<int64_t>(totals, totals, nb, ws + nb + 1, s);
    k_scan_tiles<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, totals, total, out32);
}

void scan_exclusive_i64_ws(const int64_t *in, int64_t *out, int64_t n, int64_t *ws,
                           cudaStream_t s, int64_t *total, int32_t *out32)
{
    scan_ws_impl<int64_t>(in, out, n, ws, s, total, out32);
}

// ---------------------------------------------------------------------------
// single-pass scans: the look-back kernel of grb_lookback.cuh
// ---------------------------------------------------------------------------

size_t scan_lb_ws_elems(int64_t n) { return lb_ws_elems(n); }

// value i of the scan: an int64 array
struct LbLoadI64 {
    const int64_t *in;
    __device__ int64_t operator()(int64_t i) const { return in[i]; }
};

// value i of the scan: cnt[i] where keep[i] (every i when keep is null), 0
// elsewhere and at i = n
struct LbLoadCounts {
    const int32_t *cnt;
    const int8_t *keep;
    int64_t n;
    __device__ int64_t operator()(int64_t i) const
    {
        if (i >= n) return 0;
        // both loads issued before either is used
        const int32_t c = cnt[i];
        const int8_t k = keep ? keep[i] : (int8_t)1;
        return k ? (int64_t)c : 0;
    }
};

void scan_exclusive_lb(const int64_t *in, int64_t *out, int64_t n, unsigned long long *ws,
                       cudaStream_t s, int64_t *total, int32_t *out32, int *err)
{
    if (n <= 0) return;
    if (n <= SCAN_SINGLE_MAX) {
        k_scan_single<int64_t><<<1, SCAN1_THREADS, 0, s>>>(in, out, n, total, out32);
        return;
    }
    const int64_t ntiles = (n + LB_TILE - 1) / LB_TILE;
    k_scan_lookback<LbLoadI64><<<(unsigned)ntiles, LB_THREADS, 0, s>>>(LbLoadI64{in}, out, n,
                                                                      ws, total, out32, err);
}

void scan_exclusive_lb_counts(const int32_t *cnt, const int8_t *keep, int64_t n,
                              int64_t *out, unsigned long long *ws, cudaStream_t s,
                              int64_t *total, int32_t *out32, int *err)
{
    const int64_t ntiles = (n + 1 + LB_TILE - 1) / LB_TILE;
    k_scan_lookback<LbLoadCounts><<<(unsigned)ntiles, LB_THREADS, 0, s>>>(
        LbLoadCounts{cnt, keep, n}, out, n + 1, ws, total, out32, err);
}

int scan_exclusive_i32_to_i64(const int32_t *in, int64_t *out, int64_t n,
                              cudaStream_t s)
{
    return scan_impl<int32_t>(in, out, n, s);
}

// ---------------------------------------------------------------------------
// zombie pruning and download
// ---------------------------------------------------------------------------

// live entries per row (one warp per row)
__global__ void k_count_live(const int32_t *__restrict__ Ap,
                             const int32_t *__restrict__ Aj, int64_t nrows,
                             int64_t *__restrict__ cnt)
{
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int lane = threadIdx.x & 31;
    for (int64_t r = warp; r < nrows; r += nwarps) {
        int32_t lo = Ap[r], hi = Ap[r + 1];
        int32_t c = 0;
        for (int32_t p = lo + lane; p < hi; p += 32) c += (Aj[p] >= 0);
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) cnt[r] = c;
    }
}

// copy live entries of each row to their new positions (order preserved)
__global__ void k_compact_live(const int32_t *__restrict__ Ap,
                               const int32_t *__restrict__ Aj,
                               const char *__restrict__ Ax, size_t ts, bool iso,
                               int64_t nrows, const int64_t *__restrict__ newp,
                               int32_t *__restrict__ Bj, char *__restrict__ Bx)
{
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int lane = threadIdx.x & 31;
    for (int64_t r = warp; r < nrows; r += nwarps) {
        int32_t lo = Ap[r], hi = Ap[r + 1];
        int64_t w = newp[r];
        for (int32_t base = lo; base < hi; base += 32) {
            int32_t p = base + lane;
            bool live = (p < hi) && (Aj[p] >= 0);
            unsigned m = __ballot_sync(0xffffffffu, live);
            if (live) {
                int64_t q = w + __popc(m & ((1u << lane) - 1));
                Bj[q] = Aj[p];
                if (Ax && !iso) {
                    for (size_t b = 0; b < ts; b++) Bx[q * ts + b] = Ax[(int64_t)p * ts + b];
                }
            }
            w += __popc(m);
        }
    }
}

__global__ void k_i64_to_i32(const int64_t *__restrict__ in, int32_t *__restrict__ out,
                             int64_t n)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; t < n; t += stride) out[t] = (int32_t)in[t];
}

int dev_prune_zombies(DevCSR &A, cudaStream_t s)
{
    if (A.nzombies == 0) return SUCCESS;
    size_t ts = type_size(A.type);
    int64_t *cnt = (int64_t *)dalloc((size_t)(A.nrows + 1) * 8, s);
    if (!cnt) return OUT_OF_MEMORY;
    int threads = 256;
    int grid = grid_for(A.nrows * 32, threads);
    k_count_live<<<grid, threads, 0, s>>>(A.p, A.j, A.nrows, cnt);
    cudaMemsetAsync(cnt + A.nrows, 0, 8, s);
    int info = scan_exclusive_i64(cnt, cnt, A.nrows + 1, s);
    if (info != SUCCESS) { dfree(cnt, s); return info; }
    int64_t live = A.nnz - A.nzombies;
    int32_t *Bj = (int32_t *)dalloc((size_t)(live ? live : 1) * 4, s);
    char *Bx = nullptr;
    if (A.x && !A.iso) Bx = (char *)dalloc((size_t)(live ? live : 1) * ts, s);
    int32_t *Bp = (int32_t *)dalloc((size_t)(A.nrows + 1) * 4, s);
    if (!Bj || !Bp || (A.x && !A.iso && !Bx)) {
        dfree(cnt, s); dfree(Bj, s); dfree(Bx, s); dfree(Bp, s);
        return OUT_OF_MEMORY;
    }
    k_compact_live<<<grid, threads, 0, s>>>(A.p, A.j, (const char *)A.x, ts,
                                            A.iso, A.nrows, cnt, Bj, Bx);
    k_i64_to_i32<<<grid_for(A.nrows + 1, 256), 256, 0, s>>>(cnt, Bp, A.nrows + 1);
    dfree(cnt, s);
    dfree(A.p, s); dfree(A.j, s);
    if (A.x && !A.iso) { dfree(A.x, s); A.x = Bx; }
    A.p = Bp; A.j = Bj; A.nnz = live; A.nzombies = 0;
    return cuda_to_info(cudaGetLastError());
}

// entries of a valued mask whose value is false become zombies
__global__ void k_mask_false_to_zombie(const int32_t *__restrict__ Mj,
                                       const void *__restrict__ Mx, int mtype,
                                       int64_t n, int32_t *__restrict__ Oj,
                                       unsigned long long *__restrict__ nz)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long c = 0;
    for (; t < n; t += stride) {
        bool v;
        switch (mtype) {
            case T_BOOL: v = ((const uint8_t *)Mx)[t] != 0; break;
            case T_INT32: case T_UINT32: v = ((const uint32_t *)Mx)[t] != 0; break;
            case T_FP32: v = ((const float *)Mx)[t] != 0.0f; break;
            case T_FP64: v = ((const double *)Mx)[t] != 0.0; break;
            default: v = ((const uint64_t *)Mx)[t] != 0; break;
        }
        int32_t j = Mj[t];
        if (j >= 0 && !v) { Oj[t] = flip(j); c++; }
        else Oj[t] = j;
    }
    if (c) atomicAdd(nz, c);
}

int dev_mask_to_struct(DevCSR &out, const DevCSR &M, cudaStream_t s)
{
    out = DevCSR();
    out.nrows = M.nrows; out.ncols = M.ncols; out.nnz = M.nnz; out.type = T_BOOL;
    out.p = (int32_t *)dalloc((size_t)(M.nrows + 1) * 4, s);
    out.j = (int32_t *)dalloc((size_t)(M.nnz ? M.nnz : 1) * 4, s);
    unsigned long long *nz = (unsigned long long *)dalloc(8, s);
    if (!out.p || !out.j || !nz) { dev_free(out, s); dfree(nz, s); return OUT_OF_MEMORY; }
    cudaMemcpyAsync(out.p, M.p, (size_t)(M.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(nz, 0, 8, s);
    if (M.iso) {
        // iso mask: all true or all false
        uint64_t v = 0;
        cudaMemcpyAsync(&v, M.x, type_size(M.type), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        bool t;
        if (M.type == T_FP32) { float f; memcpy(&f, &v, 4); t = f != 0.0f; }
        else if (M.type == T_FP64) { double d; memcpy(&d, &v, 8); t = d != 0.0; }
        else t = v != 0;
        if (t) {
            cudaMemcpyAsync(out.j, M.j, (size_t)M.nnz * 4, cudaMemcpyDeviceToDevice, s);
            out.nzombies = M.nzombies;
        } else {
            dfree(out.j, s);
            out.j = (int32_t *)dalloc(4, s);
            cudaMemsetAsync(out.p, 0, (size_t)(M.nrows + 1) * 4, s);
            out.nnz = 0;
            out.nzombies = 0;
        }
        dfree(nz, s);
        return cuda_to_info(cudaStreamSynchronize(s));
    }
    if (M.nnz > 0)
        k_mask_false_to_zombie<<<grid_for(M.nnz, 256), 256, 0, s>>>(M.j, M.x, M.type, M.nnz, out.j, nz);
    unsigned long long h = 0;
    cudaMemcpyAsync(&h, nz, 8, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    dfree(nz, s);
    if (e != cudaSuccess) { dev_free(out, s); return cuda_to_info(e); }
    out.nzombies = (int64_t)h + M.nzombies;
    return dev_prune_zombies(out, s);
}

int dev_download(const DevCSR &A0, int64_t **p, int64_t **i, void **x,
                 bool keep_zombies, alloc_fn alloc, cudaStream_t s)
{
    DevCSR A = A0;              // shallow copy
    bool owned = false;
    if (!keep_zombies && A.nzombies > 0) {
        // prune into a private copy so the caller's matrix is untouched
        DevCSR B = A0;
        size_t ts = type_size(A0.type);
        B.p = (int32_t *)dalloc((size_t)(A0.nrows + 1) * 4, s);
        B.j = (int32_t *)dalloc((size_t)(A0.nnz ? A0.nnz : 1) * 4, s);
        B.x = nullptr;
        if (A0.x) B.x = dalloc(A0.iso ? ts : (size_t)(A0.nnz ? A0.nnz : 1) * ts, s);
        if (!B.p || !B.j || (A0.x && !B.x)) { dev_free(B, s); return OUT_OF_MEMORY; }
        cudaMemcpyAsync(B.p, A0.p, (size_t)(A0.nrows + 1) * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(B.j, A0.j, (size_t)A0.nnz * 4, cudaMemcpyDeviceToDevice, s);
        if (A0.x) cudaMemcpyAsync(B.x, A0.x, A0.iso ? ts : (size_t)A0.nnz * ts,
                                  cudaMemcpyDeviceToDevice, s);
        int info = dev_prune_zombies(B, s);
        if (info != SUCCESS) { dev_free(B, s); return info; }
        A = B; owned = true;
    }
    size_t ts = type_size(A.type);
    int64_t nnz = A.nnz;
    *p = (int64_t *)alloc((size_t)(A.nrows + 1) * 8);
    *i = (int64_t *)alloc((size_t)(nnz ? nnz : 1) * 8);
    *x = nullptr;
    if (A.x) *x = alloc(A.iso ? ts : (size_t)(nnz ? nnz : 1) * ts);
    int64_t *stage = (int64_t *)dalloc((size_t)((A.nrows + 1 > nnz ? A.nrows + 1 : nnz)) * 8, s);
    if (!*p || !*i || (A.x && !*x) || !stage) {
        dfree(stage, s);
        if (owned) dev_free(A, s);
        return OUT_OF_MEMORY;
    }
    k_widen<<<grid_for(A.nrows + 1, 256), 256, 0, s>>>(A.p, stage, A.nrows + 1);
    cudaMemcpyAsync(*p, stage, (size_t)(A.nrows + 1) * 8, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    if (nnz > 0) {
        k_widen<<<grid_for(nnz, 256), 256, 0, s>>>(A.j, stage, nnz);
        cudaMemcpyAsync(*i, stage, (size_t)nnz * 8, cudaMemcpyDeviceToHost, s);
    }
    if (A.x) cudaMemcpyAsync(*x, A.x, A.iso ? ts : (size_t)nnz * ts,
                             cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    dfree(stage, s);
    if (owned) dev_free(A, s);
    return cuda_to_info(e);
}

}  // namespace grb
