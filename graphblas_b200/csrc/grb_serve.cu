// grb_serve.cu: a request server over device-resident graphs.
//
// The reference has no server; this answers the "serving" use of the path:
// triangle counts (C<L> = L*U', plus_pair, then a sum: dot3 + reduce), SSSP
// relaxation steps (w = u'*A with min_plus fp32: saxpy3 on a one-row u) and
// products C = A*B (plus_times fp64: saxpy3) against graphs uploaded once.
//
// Continuous batching: `nslots` worker threads, each with its own CUDA
// stream, take admitted requests as they finish their previous one, so
// requests that arrive while others run join the running set at once and
// their kernels overlap on the device.  Admission is by HBM footprint: every
// request's device memory need is estimated from its symbolic size (mask
// entries for dot3, min(flops, ncols) per row for saxpy3) before it runs; a
// request waits while the running set's footprint plus its own exceeds the
// budget, and one that can never fit is rejected.  Latency = completion time
// minus arrival time (the open-loop replay submits each request at its
// arrival time on a steady clock).
//
// Requests of the same kind on the same graph that wait together are fused:
// a worker that takes an SSSP step also takes the other waiting SSSP steps
// on that graph (up to max_group, as the budget allows) and runs them as one
// product W = U min.+ S whose rows are their frontiers - row r of W is
// exactly request r's vxm, because the product is computed row by row - so
// small requests share one symbolic phase, one set of launches and one host
// synchronisation.  Each request's checksum is the sum of its own row taken
// in a fixed order, the same whether it ran alone or fused.  A fused product
// that fails (a device allocation, say) is retried request by request, so
// one request's failure never fails the others it was fused with.

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>
#include <algorithm>
#include "../../include/grb_b200.h"
#include "grb_saxpy3.h"

using namespace grb;
using Clock = std::chrono::steady_clock;

namespace {

enum Kind { K_TRICOUNT = 1, K_SSSP = 2, K_MXM = 3 };

struct Graph {
    int kind;                 // what it serves
    DevCSR S;                 // the matrix (weights for SSSP / values for MXM)
    DevCSR L, U;              // triangle counting: strict lower / upper
    int64_t mxm_cap = 0;      // symbolic output capacity of S*S (entries)
};

struct Req {
    int64_t id;
    int kind;
    int graph;
    // SSSP frontier (indices, fp32 distances)
    std::vector<int64_t> ui;
    std::vector<float> ux;
    double t_arrival = 0, t_start = 0, t_done = 0;
    int64_t footprint = 0;
    int status = 0;
    // results
    int64_t count = 0;                // triangles, or nnz of the result
    double checksum = 0;              // sum of the result's values (device)
    std::vector<int64_t> rp, ri;      // result pattern (SSSP: 1-row; MXM: CSR)
    std::vector<uint8_t> rx;          // result values (raw bytes)
};

}  // namespace

struct grb_b200_server_s {
    int nslots = 1;
    int64_t budget = 0;
    std::vector<Graph> graphs;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Req *> pending;
    std::vector<Req *> all;
    std::vector<std::thread> workers;
    bool stopping = false;
    int64_t in_use = 0, peak_use = 0;
    int64_t admitted = 0, rejected = 0, completed = 0, failed = 0;
    int active = 0, peak_active = 0;
    int max_group = 64;               // SSSP steps fused into one product, at most
    int64_t fused_runs = 0, fused_requests = 0;
    int largest_group = 1;
    Clock::time_point t0;
    bool keep_results = true;
};

namespace {

double now_s(const grb_b200_server_s *S)
{
    return std::chrono::duration<double>(Clock::now() - S->t0).count();
}

int64_t footprint(const grb_b200_server_s *S, const Req *r)
{
    const Graph &g = S->graphs[r->graph];
    switch (r->kind) {
        case K_TRICOUNT:
            // C values + indices + the dot3 work queue, per mask entry
            return g.L.nnz * (8 + 4 + 32) + 4 * (g.L.nrows + 1) + (1 << 20);
        case K_SSSP:
            // dense accumulator and flags (heavy row) or the slot arrays
            return g.S.ncols * (8 + 4 + 4 + 4) + (int64_t)r->ui.size() * 8 + (1 << 20);
        case K_MXM:
            // slot capacity of the output (temp + final) plus per-row plans
            return g.mxm_cap * (4 + 8) * 2 + g.S.nrows * 48 + (1 << 20);
    }
    return 1 << 20;
}

// per-row sums of an fp32 CSR (one warp per row: lane-strided partial sums in
// index order, then a fixed shuffle tree), so a row's sum depends only on the
// row; out[r] as double
__global__ void k_row_sums_fp32(const int32_t *__restrict__ p, const float *__restrict__ x,
                                int64_t nrows, double *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows;
         r += nw) {
        float acc = 0.0f;
        for (int32_t q = p[r] + lane; q < p[r + 1]; q += 32) acc = __fadd_rn(acc, x[q]);
        for (int o = 16; o > 0; o >>= 1) acc = __fadd_rn(acc, __shfl_down_sync(0xffffffffu, acc, o));
        if (lane == 0) out[r] = (double)acc;
    }
}

// SSSP steps on one graph, fused: W = U min.+ S with one row of U per request
int run_sssp_group(grb_b200_server_s *S, std::vector<Req *> &grp, cudaStream_t s)
{
    const Graph &g = S->graphs[grp[0]->graph];
    const int64_t k = (int64_t)grp.size();
    std::vector<int64_t> up(k + 1, 0), ui;
    std::vector<float> ux;
    for (int64_t q = 0; q < k; q++) {
        ui.insert(ui.end(), grp[q]->ui.begin(), grp[q]->ui.end());
        ux.insert(ux.end(), grp[q]->ux.begin(), grp[q]->ux.end());
        up[q + 1] = (int64_t)ui.size();
    }
    DevCSR U, W;
    int info = dev_upload(U, k, g.S.nrows, up.data(), ui.empty() ? nullptr : ui.data(),
                          ux.empty() ? nullptr : ux.data(), T_FP32, false, s);
    if (info == SUCCESS) {
        SemiringCode sr{OP_MIN, OP_PLUS, T_FP32};
        info = saxpy3(W, nullptr, false, true, U, g.S, sr, s);
    }
    std::vector<int64_t> wp(k + 1, 0);
    std::vector<double> sums(k, 0.0);
    if (info == SUCCESS) {
        double *d_sums = (double *)dalloc((size_t)k * 8, s);
        if (!d_sums) info = OUT_OF_MEMORY;
        if (info == SUCCESS) {
            if (W.nnz > 0)
                k_row_sums_fp32<<<(unsigned)((k + 7) / 8), 256, 0, s>>>(W.p, (const float *)W.x,
                                                                      k, d_sums);
            else
                cudaMemsetAsync(d_sums, 0, (size_t)k * 8, s);
            std::vector<int32_t> wp32(k + 1);
            cudaMemcpyAsync(wp32.data(), W.p, (size_t)(k + 1) * 4, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(sums.data(), d_sums, (size_t)k * 8, cudaMemcpyDeviceToHost, s);
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) info = cuda_to_info(e);
            for (int64_t q = 0; q <= k; q++) wp[q] = wp32[q];
            dfree(d_sums, s);
        }
    }
    if (info == SUCCESS && S->keep_results && W.nnz > 0) {
        int64_t *p = nullptr, *i = nullptr;
        void *x = nullptr;
        info = dev_download(W, &p, &i, &x, false, malloc, s);
        if (info == SUCCESS) {
            for (int64_t q = 0; q < k; q++) {
                Req *r = grp[q];
                const int64_t lo = p[q], hi = p[q + 1];
                r->rp = {0, hi - lo};
                r->ri.assign(i + lo, i + hi);
                r->rx.assign((uint8_t *)x + lo * 4, (uint8_t *)x + hi * 4);
            }
        }
        free(p); free(i); free(x);
    } else if (info == SUCCESS && S->keep_results) {
        for (Req *r : grp) { r->rp = {0, 0}; r->ri.clear(); r->rx.clear(); }
    }
    for (int64_t q = 0; q < k; q++) {
        grp[q]->count = wp[q + 1] - wp[q];
        grp[q]->checksum = sums[q];
    }
    dev_free(U, s);
    dev_free(W, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (info == SUCCESS && e != cudaSuccess) info = cuda_to_info(e);
    return info;
}

int run_request(grb_b200_server_s *S, Req *r, cudaStream_t s)
{
    const Graph &g = S->graphs[r->graph];
    int info = SUCCESS;
    if (r->kind == K_TRICOUNT) {
        DevCSR C;
        SemiringCode sr{OP_PLUS, OP_PAIR, T_INT64};
        info = dot3(C, g.L, true, g.L, g.U, sr, s);
        if (info == SUCCESS) {
            int64_t n = 0;
            info = reduce_scalar(&n, C, OP_PLUS, s);
            r->count = n;
            r->checksum = (double)n;
        }
        dev_free(C, s);
    } else if (r->kind == K_SSSP) {
        // one relaxation step, w = u' min.+ S (fp32, u sparse): a group of one
        std::vector<Req *> one{r};
        return run_sssp_group(S, one, s);
    } else {
        DevCSR C;
        SemiringCode sr{OP_PLUS, OP_TIMES, T_FP64};
        info = saxpy3(C, nullptr, false, true, g.S, g.S, sr, s);
        if (info == SUCCESS) {
            r->count = C.nnz;
            double sum = 0;
            info = reduce_scalar(&sum, C, OP_PLUS, s);
            r->checksum = sum;
        }
        if (info == SUCCESS) {
            if (S->keep_results) {
                int64_t *p = nullptr, *i = nullptr;
                void *x = nullptr;
                info = dev_download(C, &p, &i, &x, false, malloc, s);
                if (info == SUCCESS) {
                    r->rp.assign(p, p + C.nrows + 1);
                    r->ri.assign(i, i + C.nnz);
                    r->rx.assign((uint8_t *)x, (uint8_t *)x + C.nnz * 8);
                }
                free(p); free(i); free(x);
            }
        }
        dev_free(C, s);
    }
    cudaError_t e = cudaStreamSynchronize(s);
    if (info == SUCCESS && e != cudaSuccess) info = cuda_to_info(e);
    return info;
}

void worker_main(grb_b200_server_s *S, int dev)
{
    cudaSetDevice(dev);
    cudaStream_t s;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    stream_scratch_enable(s);
    std::vector<Req *> grp;
    while (true) {
        Req *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            // admit the oldest pending request once its footprint fits
            S->cv.wait(lk, [&] {
                if (S->stopping && S->pending.empty()) return true;
                if (S->pending.empty()) return false;
                const Req *h = S->pending.front();
                return S->in_use + h->footprint <= S->budget;
            });
            if (S->pending.empty()) break;
            r = S->pending.front();
            S->pending.pop_front();
            grp.assign(1, r);
            int64_t fp = r->footprint;
            if (r->kind == K_SSSP) {
                // the other waiting SSSP steps on the same graph join it
                for (auto it = S->pending.begin();
                     it != S->pending.end() && (int)grp.size() < S->max_group;) {
                    Req *q = *it;
                    if (q->kind == K_SSSP && q->graph == r->graph &&
                        S->in_use + fp + q->footprint <= S->budget) {
                        grp.push_back(q);
                        fp += q->footprint;
                        it = S->pending.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
            S->in_use += fp;
            S->peak_use = std::max(S->peak_use, S->in_use);
            S->admitted += (int64_t)grp.size();
            S->active += (int)grp.size();
            S->peak_active = std::max(S->peak_active, S->active);
        }
        const double t_start = now_s(S);
        for (Req *q : grp) q->t_start = t_start;
        if (grp.size() > 1) {
            const int status = run_sssp_group(S, grp, s);
            const double t_done = now_s(S);
            for (Req *q : grp) {
                q->status = status;
                q->t_done = t_done;
            }
            if (status != SUCCESS) {
                // retried one by one: a member's own failure stays its own
                for (Req *q : grp) {
                    q->status = run_request(S, q, s);
                    q->t_done = now_s(S);
                }
            }
        } else {
            r->status = run_request(S, r, s);
            r->t_done = now_s(S);
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (grp.size() > 1) {
                S->fused_runs++;
                S->fused_requests += (int64_t)grp.size();
                S->largest_group = std::max(S->largest_group, (int)grp.size());
            }
            for (Req *q : grp) {
                S->in_use -= q->footprint;
                S->active--;
                if (q->status == SUCCESS) S->completed++;
                else S->failed++;
            }
        }
        S->cv.notify_all();
    }
    cudaStreamSynchronize(s);
    stream_scratch_release(s);
    cudaStreamDestroy(s);
}

// requests [r0, r1) have arrived: queued together, under one lock
void submit(grb_b200_server_s *S, Req *const *r0, Req *const *r1)
{
    for (Req *const *q = r0; q < r1; q++) (*q)->footprint = footprint(S, *q);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (Req *const *q = r0; q < r1; q++) {
            Req *r = *q;
            S->all.push_back(r);
            if (r->footprint > S->budget) {
                r->status = OUT_OF_MEMORY;          // can never fit: rejected
                r->t_start = r->t_done = r->t_arrival;
                S->rejected++;
                continue;
            }
            S->pending.push_back(r);
        }
    }
    S->cv.notify_all();
}

}  // namespace

extern "C" {

int grb_b200_server_create(grb_b200_server *Sp, int nslots, int64_t hbm_budget_bytes,
                           bool keep_results)
{
    if (!Sp) return NULL_POINTER;
    if (nslots < 1 || nslots > 64 || hbm_budget_bytes <= 0) return INVALID_VALUE;
    int info = init_device();
    if (info != SUCCESS) return info;
    grb_b200_server_s *S = new grb_b200_server_s();
    S->nslots = nslots;
    S->budget = hbm_budget_bytes;
    S->keep_results = keep_results;
    S->t0 = Clock::now();
    *Sp = S;
    return SUCCESS;
}

int grb_b200_server_add_graph(grb_b200_server S, int kind, int64_t n, const int64_t *p,
                              const int64_t *i, const void *x, int *graph_id)
{
    if (!S || !p || !i || !graph_id) return NULL_POINTER;
    if (kind < K_TRICOUNT || kind > K_MXM) return INVALID_VALUE;
    cudaStream_t s = stream_acquire();
    Graph g;
    g.kind = kind;
    int info = SUCCESS;
    if (kind == K_TRICOUNT) {
        // split into strict lower / upper triangles on the host once
        std::vector<int64_t> Lp(n + 1), Up(n + 1), Li, Ui;
        Li.reserve(p[n] / 2 + 1);
        Ui.reserve(p[n] / 2 + 1);
        for (int64_t r = 0; r < n; r++) {
            Lp[r] = (int64_t)Li.size();
            Up[r] = (int64_t)Ui.size();
            for (int64_t q = p[r]; q < p[r + 1]; q++) {
                if (i[q] < r) Li.push_back(i[q]);
                else if (i[q] > r) Ui.push_back(i[q]);
            }
        }
        Lp[n] = (int64_t)Li.size();
        Up[n] = (int64_t)Ui.size();
        info = dev_upload(g.L, n, n, Lp.data(), Li.data(), nullptr, T_BOOL, true, s);
        if (info == SUCCESS)
            info = dev_upload(g.U, n, n, Up.data(), Ui.data(), nullptr, T_BOOL, true, s);
    } else {
        const int t = (kind == K_SSSP) ? T_FP32 : T_FP64;
        info = dev_upload(g.S, n, n, p, i, x, t, false, s);
        if (info == SUCCESS && kind == K_MXM) {
            // symbolic size of S*S: sum over rows of min(flops, n)
            int64_t cap = 0;
            for (int64_t r = 0; r < n; r++) {
                int64_t f = 0;
                for (int64_t q = p[r]; q < p[r + 1]; q++) f += p[i[q] + 1] - p[i[q]];
                cap += std::min(f, n);
            }
            g.mxm_cap = cap;
        }
    }
    cudaError_t e = cudaStreamSynchronize(s);
    stream_release(s);
    if (info == SUCCESS && e != cudaSuccess) info = cuda_to_info(e);
    if (info != SUCCESS) return info;
    std::lock_guard<std::mutex> lk(S->mu);
    S->graphs.push_back(std::move(g));
    *graph_id = (int)S->graphs.size() - 1;
    return SUCCESS;
}

// A graph given as a serialized blob (GxB_Matrix_serialize's format, any
// compression): decoded on the host, then uploaded as add_graph does
int grb_b200_server_add_graph_blob(grb_b200_server S, int kind, const void *blob,
                                   size_t blob_size, int *graph_id)
{
    if (!S || !blob || !graph_id) return NULL_POINTER;
    if (kind < K_TRICOUNT || kind > K_MXM) return INVALID_VALUE;
    const int want = kind == K_SSSP ? T_FP32 : (kind == K_MXM ? T_FP64 : 0);
    int64_t nrows = 0, ncols = 0, *p = nullptr, *i = nullptr;
    void *x = nullptr;
    int type = 0;
    bool iso = false;
    int info = grb_b200_blob_decode(blob, blob_size, want, &nrows, &ncols, &type, &p, &i, &x,
                                    &iso);
    if (info != SUCCESS) return info;
    if (nrows != ncols) info = DIMENSION_MISMATCH;
    void *xs = x;
    if (info == SUCCESS && want != 0 && iso) {
        // the server's graphs hold one value per entry
        const size_t ts = type_size(type);
        const int64_t nnz = p[nrows];
        xs = malloc((size_t)(nnz ? nnz : 1) * ts);
        if (!xs) info = OUT_OF_MEMORY;
        else for (int64_t q = 0; q < nnz; q++) memcpy((char *)xs + q * ts, x, ts);
    }
    if (info == SUCCESS)
        info = grb_b200_server_add_graph(S, kind, nrows, p, i, want ? xs : nullptr, graph_id);
    if (xs != x) free(xs);
    free(p); free(i); free(x);
    return info;
}

// Replay an open-loop trace: request k (kind[k] on graph[k]) arrives at
// t_arrival[k] seconds after the call; SSSP requests take their frontier from
// (fp[k]..fp[k+1]) of fi/fx.  Returns when every request finished.
int grb_b200_server_replay(grb_b200_server S, int64_t nreq, const int *kind,
                           const int *graph, const double *t_arrival,
                           const int64_t *fp, const int64_t *fi, const float *fx)
{
    if (!S || !kind || !graph || !t_arrival) return NULL_POINTER;
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (Req *r : S->all) delete r;
        S->all.clear();
        S->pending.clear();
        S->stopping = false;
        S->in_use = S->peak_use = 0;
        S->admitted = S->rejected = S->completed = S->failed = 0;
        S->active = S->peak_active = 0;
        S->fused_runs = S->fused_requests = 0;
        S->largest_group = 1;
    }
    for (int64_t k = 0; k < nreq; k++)
        if (graph[k] < 0 || graph[k] >= (int)S->graphs.size() ||
            S->graphs[graph[k]].kind != kind[k])
            return INVALID_VALUE;
    S->t0 = Clock::now();
    for (int w = 0; w < S->nslots; w++) S->workers.emplace_back(worker_main, S, dev);
    std::vector<Req *> reqs((size_t)nreq);
    for (int64_t k = 0; k < nreq; k++) {
        Req *r = new Req();
        r->id = k;
        r->kind = kind[k];
        r->graph = graph[k];
        if (r->kind == K_SSSP && fp && fi && fx) {
            r->ui.assign(fi + fp[k], fi + fp[k + 1]);
            r->ux.assign(fx + fp[k], fx + fp[k + 1]);
        }
        r->t_arrival = t_arrival[k];
        reqs[k] = r;
    }
    for (int64_t k = 0; k < nreq;) {
        // open loop: wait for the arrival time, never for the server; then
        // queue every request that has arrived by now (in arrival order)
        const auto due = S->t0 + std::chrono::duration_cast<Clock::duration>(
                                     std::chrono::duration<double>(t_arrival[k]));
        std::this_thread::sleep_until(due);
        const double now = now_s(S);
        int64_t e = k + 1;
        while (e < nreq && t_arrival[e] <= now) e++;
        submit(S, reqs.data() + k, reqs.data() + e);
        k = e;
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv.notify_all();
    for (auto &t : S->workers) t.join();
    S->workers.clear();
    return SUCCESS;
}

// Per-request outcome: status, count (triangles or result nnz), checksum (sum
// of the result's values, reduced on the device, so it is there whether or
// not results are kept), latency (done - arrival), queueing delay (start -
// arrival).
int grb_b200_server_request(grb_b200_server S, int64_t k, int *status, int64_t *count,
                            double *checksum, double *latency_s, double *wait_s)
{
    if (!S) return NULL_POINTER;
    if (k < 0 || k >= (int64_t)S->all.size()) return INVALID_VALUE;
    const Req *r = nullptr;
    for (const Req *q : S->all) if (q->id == k) { r = q; break; }
    if (!r) return INVALID_VALUE;
    if (status) *status = r->status;
    if (count) *count = r->count;
    if (checksum) *checksum = r->checksum;
    if (latency_s) *latency_s = r->t_done - r->t_arrival;
    if (wait_s) *wait_s = r->t_start - r->t_arrival;
    return SUCCESS;
}

// Copy out a kept result (SSSP: 1-row CSR with fp32 values; MXM: CSR with
// fp64 values).  Sizes in *np, *ni; pass NULL buffers to query sizes.
int grb_b200_server_result(grb_b200_server S, int64_t k, int64_t *p, int64_t *i,
                           void *x, int64_t *np_, int64_t *ni)
{
    if (!S || !np_ || !ni) return NULL_POINTER;
    const Req *r = nullptr;
    for (const Req *q : S->all) if (q->id == k) { r = q; break; }
    if (!r) return INVALID_VALUE;
    *np_ = (int64_t)r->rp.size();
    *ni = (int64_t)r->ri.size();
    if (p) memcpy(p, r->rp.data(), r->rp.size() * 8);
    if (i) memcpy(i, r->ri.data(), r->ri.size() * 8);
    if (x) memcpy(x, r->rx.data(), r->rx.size());
    return SUCCESS;
}

int grb_b200_server_stats(grb_b200_server S, int64_t *admitted, int64_t *rejected,
                          int64_t *completed, int64_t *failed, int64_t *peak_bytes,
                          int *peak_active, double *makespan_s)
{
    if (!S) return NULL_POINTER;
    std::lock_guard<std::mutex> lk(S->mu);
    if (admitted) *admitted = S->admitted;
    if (rejected) *rejected = S->rejected;
    if (completed) *completed = S->completed;
    if (failed) *failed = S->failed;
    if (peak_bytes) *peak_bytes = S->peak_use;
    if (peak_active) *peak_active = S->peak_active;
    if (makespan_s) {
        double t = 0;
        for (const Req *r : S->all) t = std::max(t, r->t_done);
        *makespan_s = t;
    }
    return SUCCESS;
}

int grb_b200_server_set_fusion(grb_b200_server S, int max_group)
{
    if (!S) return NULL_POINTER;
    if (max_group < 1 || max_group > 4096) return INVALID_VALUE;
    std::lock_guard<std::mutex> lk(S->mu);
    S->max_group = max_group;
    return SUCCESS;
}

int grb_b200_server_fusion_stats(grb_b200_server S, int64_t *fused_runs,
                                 int64_t *fused_requests, int *largest_group)
{
    if (!S) return NULL_POINTER;
    std::lock_guard<std::mutex> lk(S->mu);
    if (fused_runs) *fused_runs = S->fused_runs;
    if (fused_requests) *fused_requests = S->fused_requests;
    if (largest_group) *largest_group = S->largest_group;
    return SUCCESS;
}

int grb_b200_server_free(grb_b200_server *Sp)
{
    if (!Sp || !*Sp) return SUCCESS;
    grb_b200_server_s *S = *Sp;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv.notify_all();
    for (auto &t : S->workers) t.join();
    cudaStream_t s = stream_acquire();
    for (Graph &g : S->graphs) { dev_free(g.S, s); dev_free(g.L, s); dev_free(g.U, s); }
    cudaStreamSynchronize(s);
    stream_release(s);
    for (Req *r : S->all) delete r;
    delete S;
    *Sp = nullptr;
    return SUCCESS;
}

}  // extern "C"
