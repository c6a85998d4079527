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
        // one relaxation step: w = u' min.+ S (fp32), u sparse
        DevCSR u, w;
        const int64_t nu = (int64_t)r->ui.size();
        std::vector<int64_t> up = {0, nu};
        info = dev_upload(u, 1, g.S.nrows, up.data(), r->ui.data(), r->ux.data(), T_FP32,
                          false, s);
        if (info == SUCCESS) {
            SemiringCode sr{OP_MIN, OP_PLUS, T_FP32};
            info = saxpy3(w, nullptr, false, true, u, g.S, sr, s);
        }
        if (info == SUCCESS) {
            r->count = w.nnz;
            float sum = 0;
            info = reduce_scalar(&sum, w, OP_PLUS, s);
            r->checksum = sum;
        }
        if (info == SUCCESS) {
            if (S->keep_results) {
                int64_t *p = nullptr, *i = nullptr;
                void *x = nullptr;
                info = dev_download(w, &p, &i, &x, false, malloc, s);
                if (info == SUCCESS) {
                    r->rp.assign(p, p + 2);
                    r->ri.assign(i, i + w.nnz);
                    r->rx.assign((uint8_t *)x, (uint8_t *)x + w.nnz * 4);
                }
                free(p); free(i); free(x);
            }
        }
        dev_free(u, s);
        dev_free(w, s);
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
            S->in_use += r->footprint;
            S->peak_use = std::max(S->peak_use, S->in_use);
            S->admitted++;
            S->active++;
            S->peak_active = std::max(S->peak_active, S->active);
        }
        r->t_start = now_s(S);
        r->status = run_request(S, r, s);
        r->t_done = now_s(S);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->in_use -= r->footprint;
            S->active--;
            if (r->status == SUCCESS) S->completed++;
            else S->failed++;
        }
        S->cv.notify_all();
    }
    cudaStreamDestroy(s);
}

void submit(grb_b200_server_s *S, Req *r)
{
    r->footprint = footprint(S, r);
    std::lock_guard<std::mutex> lk(S->mu);
    S->all.push_back(r);
    if (r->footprint > S->budget) {
        r->status = OUT_OF_MEMORY;          // can never fit: rejected
        r->t_start = r->t_done = r->t_arrival;
        S->rejected++;
        return;
    }
    S->pending.push_back(r);
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
    }
    for (int64_t k = 0; k < nreq; k++)
        if (graph[k] < 0 || graph[k] >= (int)S->graphs.size() ||
            S->graphs[graph[k]].kind != kind[k])
            return INVALID_VALUE;
    S->t0 = Clock::now();
    for (int w = 0; w < S->nslots; w++) S->workers.emplace_back(worker_main, S, dev);
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
        // open loop: wait for the arrival time, never for the server
        const auto due = S->t0 + std::chrono::duration_cast<Clock::duration>(
                                     std::chrono::duration<double>(t_arrival[k]));
        std::this_thread::sleep_until(due);
        submit(S, r);
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
