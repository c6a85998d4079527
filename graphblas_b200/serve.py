"""The request server (grb_b200_server_*, include/grb_b200.h) from Python.

``Server`` wraps a server handle; ``make_trace`` builds the serving workload:
an open-loop Poisson stream of mixed requests on device-resident graphs -
triangle counts on R-MAT graphs of scale 10-16 (plus_pair, dot3), SSSP
relaxation steps (min_plus fp32 vxm) and products C = A*A (plus_times fp64) on
Erdos-Renyi matrices with n log-uniform in [1024, 65536] and 4-16 entries per
row.  ``BenchServe`` is bench.py --config serve.
"""

import ctypes
import math
import os

import numpy as np

from . import lib as _lib, check, workloads as W

vp = ctypes.c_void_p
K_TRICOUNT, K_SSSP, K_MXM = 1, 2, 3


def _bind(L):
    if getattr(L, "_serve_bound", False):
        return L
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.grb_b200_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int64,
                                         ctypes.c_bool]
    L.grb_b200_server_add_graph.argtypes = [vp, ctypes.c_int, ctypes.c_int64, vp, vp, vp,
                                            ctypes.POINTER(ctypes.c_int)]
    L.grb_b200_server_replay.argtypes = [vp, ctypes.c_int64, vp, vp, vp, vp, vp, vp]
    L.grb_b200_server_request.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int),
                                          i64p, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double)]
    L.grb_b200_server_result.argtypes = [vp, ctypes.c_int64, vp, vp, vp, i64p, i64p]
    L.grb_b200_server_stats.argtypes = [vp, i64p, i64p, i64p, i64p, i64p,
                                        ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_double)]
    L.grb_b200_server_free.argtypes = [ctypes.POINTER(vp)]
    L.grb_b200_server_add_graph_blob.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t,
                                                  ctypes.POINTER(ctypes.c_int)]
    L.grb_b200_server_set_fusion.argtypes = [vp, ctypes.c_int]
    L.grb_b200_server_fusion_stats.argtypes = [vp, i64p, i64p, ctypes.POINTER(ctypes.c_int)]
    for n in ("create", "add_graph", "add_graph_blob", "replay", "request", "result",
              "stats", "free", "set_fusion", "fusion_stats"):
        getattr(L, "grb_b200_server_" + n).restype = ctypes.c_int
    L._serve_bound = True
    return L


class Server:
    """``fuse``: the most SSSP steps on one graph that run as one product when
    they wait together (1 = each request alone; None = the library's
    default, 64)."""

    def __init__(self, nslots=8, budget_bytes=40 << 30, keep_results=True, fuse=None):
        self.L = _bind(_lib())
        h = vp()
        check(self.L.grb_b200_server_create(ctypes.byref(h), nslots, budget_bytes,
                                            keep_results), "server_create")
        self.h = h
        self.kinds = []
        if fuse is not None:
            check(self.L.grb_b200_server_set_fusion(h, fuse), "server_set_fusion")

    def add_graph(self, kind, csr):
        gid = ctypes.c_int()
        x = None
        if kind == K_SSSP:
            x = np.ascontiguousarray(csr.x, np.float32)
        elif kind == K_MXM:
            x = np.ascontiguousarray(csr.x, np.float64)
        p = np.ascontiguousarray(csr.p, np.int64)
        i = np.ascontiguousarray(csr.i, np.int64)
        check(self.L.grb_b200_server_add_graph(self.h, kind, csr.nrows, p.ctypes.data,
                                               i.ctypes.data,
                                               None if x is None else x.ctypes.data,
                                               ctypes.byref(gid)), "server_add_graph")
        self.kinds.append(kind)
        return gid.value

    def add_graph_blob(self, kind, blob):
        """A resident graph from a serialized blob (GxB_Matrix_serialize's
        format, any compression)."""
        gid = ctypes.c_int()
        buf = ctypes.create_string_buffer(bytes(blob), max(len(blob), 1))
        check(self.L.grb_b200_server_add_graph_blob(self.h, kind, buf, len(blob),
                                                    ctypes.byref(gid)),
              "server_add_graph_blob")
        self.kinds.append(kind)
        return gid.value

    def replay(self, trace):
        kind = np.ascontiguousarray(trace["kind"], np.int32)
        graph = np.ascontiguousarray(trace["graph"], np.int32)
        t = np.ascontiguousarray(trace["t"], np.float64)
        fp = np.ascontiguousarray(trace["fp"], np.int64)
        fi = np.ascontiguousarray(trace["fi"], np.int64)
        fx = np.ascontiguousarray(trace["fx"], np.float32)
        check(self.L.grb_b200_server_replay(self.h, len(kind), kind.ctypes.data,
                                            graph.ctypes.data, t.ctypes.data, fp.ctypes.data,
                                            fi.ctypes.data, fx.ctypes.data), "server_replay")

    def request(self, k):
        st = ctypes.c_int()
        cnt = ctypes.c_int64()
        lat, wait, cs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(self.L.grb_b200_server_request(self.h, k, ctypes.byref(st), ctypes.byref(cnt),
                                             ctypes.byref(cs), ctypes.byref(lat),
                                             ctypes.byref(wait)))
        return dict(status=st.value, count=cnt.value, checksum=cs.value,
                    latency=lat.value, wait=wait.value)

    def result(self, k, kind):
        npp, ni = ctypes.c_int64(), ctypes.c_int64()
        check(self.L.grb_b200_server_result(self.h, k, None, None, None, ctypes.byref(npp),
                                            ctypes.byref(ni)))
        p = np.zeros(npp.value, np.int64)
        i = np.zeros(ni.value, np.int64)
        x = np.zeros(ni.value, np.float32 if kind == K_SSSP else np.float64)
        check(self.L.grb_b200_server_result(self.h, k, p.ctypes.data, i.ctypes.data,
                                            x.ctypes.data, ctypes.byref(npp),
                                            ctypes.byref(ni)))
        return p, i, x

    def stats(self):
        v = [ctypes.c_int64() for _ in range(5)]
        pa = ctypes.c_int()
        mk = ctypes.c_double()
        check(self.L.grb_b200_server_stats(self.h, *[ctypes.byref(a) for a in v],
                                           ctypes.byref(pa), ctypes.byref(mk)))
        fr, fq = ctypes.c_int64(), ctypes.c_int64()
        lg = ctypes.c_int()
        check(self.L.grb_b200_server_fusion_stats(self.h, ctypes.byref(fr), ctypes.byref(fq),
                                                  ctypes.byref(lg)))
        return dict(admitted=v[0].value, rejected=v[1].value, completed=v[2].value,
                    failed=v[3].value, peak_bytes=v[4].value, peak_active=pa.value,
                    makespan_s=mk.value, fused_runs=fr.value, fused_requests=fq.value,
                    largest_group=lg.value)

    def free(self):
        if self.h and self.h.value:
            self.L.grb_b200_server_free(ctypes.byref(self.h))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def make_graphs(seed=1, tc_scales=range(10, 17), n_sssp=3, n_mxm=6, mxm_nmax=65536):
    """The resident graph set of the serving workload."""
    graphs = []
    for s in tc_scales:
        graphs.append((K_TRICOUNT, W.rmat(s, 16, seed=seed + s)))
    rng = np.random.default_rng(seed)
    for k in range(n_sssp):
        S = W.rmat(12 + 2 * k, 16, seed=seed + 100 + k)
        w = (0.1 + 9.9 * rng.random(S.nnz)).astype(np.float32)
        graphs.append((K_SSSP, W.Csr(S.nrows, S.ncols, S.p, S.i, w)))
    lo, hi = math.log(1024), math.log(mxm_nmax)
    for k in range(n_mxm):
        n = int(round(math.exp(lo + (hi - lo) * W.unif01(seed + 7, k))))
        graphs.append((K_MXM, W.er_range(n, 4, 16, seed=seed + 200 + k)))
    return graphs


def make_trace(graphs, nreq=4000, rate=2000.0, seed=3):
    """Open-loop Poisson arrivals (mean `rate` per second), kinds uniform,
    graphs uniform within a kind; SSSP frontiers are random vertex subsets
    with fp32 distances."""
    rng = np.random.default_rng(seed)
    by_kind = {k: [g for g, (kk, _) in enumerate(graphs) if kk == k] for k in (1, 2, 3)}
    t = np.cumsum(rng.exponential(1.0 / rate, nreq))
    kind = rng.integers(1, 4, nreq).astype(np.int32)
    graph = np.array([by_kind[int(k)][rng.integers(len(by_kind[int(k)]))] for k in kind],
                     np.int32)
    fp = [0]
    fi, fx = [], []
    for k in range(nreq):
        if kind[k] == K_SSSP:
            n = graphs[graph[k]][1].nrows
            m = int(min(n, max(16, rng.integers(16, 4096))))
            idx = np.sort(rng.choice(n, m, replace=False)).astype(np.int64)
            fi.append(idx)
            fx.append((rng.random(m) * 50).astype(np.float32))
            fp.append(fp[-1] + m)
        else:
            fp.append(fp[-1])
    fi = np.concatenate(fi) if fi else np.zeros(1, np.int64)
    fx = np.concatenate(fx) if fx else np.zeros(1, np.float32)
    return {"t": t, "kind": kind, "graph": graph, "fp": np.array(fp, np.int64),
            "fi": fi, "fx": fx}


class BenchServe:
    """bench.py --config serve: req/s with p50/p99 latency."""
    metric, unit, dtype, kernel = "req/s", "req/s", "mixed", "dot3"

    def __init__(self, args):
        self.graphs = make_graphs(seed=args.seed)
        self.nreq = 4000
        self.trace = make_trace(self.graphs, nreq=self.nreq, rate=2000.0, seed=args.seed + 2)
        self.workload = "serve_poisson2000_tc_rmat10-16_sssp_minplus_fp32_mxm_er_fp64"
        self.alg_bytes = 0.0
        self.basis = ("per request: a triangle count reads L, U and the mask once and "
                      "writes C; an SSSP step reads its frontier and the rows of S it "
                      "touches and writes w; A*A reads A and the B row of every product "
                      "and writes C; over the replay's makespan, idle gaps included")

    def config(self):
        return dict(requests=self.nreq, rate_req_s=2000.0, slots=8,
                    hbm_budget_gb=40, **getattr(self, "lat", {}),
                    **getattr(self, "capacity", {}))

    def _server(self):
        # results stay on the device (counts and checksums come back), as a
        # caller chaining requests would use them
        S = Server(nslots=8, budget_bytes=40 << 30, keep_results=False)
        for kind, g in self.graphs:
            S.add_graph(kind, g)
        return S

    def dev_setup(self, gb):
        self.S = self._server()
        # capacity: the same requests all arriving at once (closed batch), so
        # the replay runs as fast as the server can take them
        burst = dict(self.trace)
        burst["t"] = np.zeros(self.nreq)
        self.S.replay(burst)
        st = self.S.stats()
        self.capacity = {"capacity_req_s": st["completed"] / max(st["makespan_s"], 1e-9),
                         "capacity_peak_concurrent": st["peak_active"],
                         "capacity_fused_requests": st["fused_requests"],
                         "capacity_largest_group": st["largest_group"]}
        # per-graph sizes for the bytes each request must move (4-byte
        # indices; fp32 / fp64 values): triangle count reads L, U and the
        # mask once and writes C; SSSP reads u and the rows of S it touches
        # and writes w; A*A reads A, the B rows of every product and writes C
        self.gstat = []
        for kind, g in self.graphs:
            deg = np.diff(g.p)
            if kind == K_TRICOUNT:
                nl = int(np.sum(g.i < np.repeat(np.arange(g.nrows), deg)))
                self.gstat.append({"tc": 8.0 * (g.nrows + 1) + 8.0 * nl + 16.0 * nl})
            elif kind == K_SSSP:
                self.gstat.append({"deg": deg})
            else:
                prods = float(np.sum(deg[g.i]))
                self.gstat.append({"mxm": 8.0 * (g.nrows + 1) + 12.0 * g.nnz + 12.0 * prods})

    def _request_bytes(self, S):
        tot = 0.0
        t = self.trace
        for k in range(self.nreq):
            g = int(t["graph"][k])
            st = self.gstat[g]
            cnt = S.request(k)["count"]
            if "tc" in st:
                tot += st["tc"]
            elif "deg" in st:
                lo, hi = t["fp"][k], t["fp"][k + 1]
                tot += 8.0 * (hi - lo) + 8.0 * float(np.sum(st["deg"][t["fi"][lo:hi]])) + 8.0 * cnt
            else:
                tot += st["mxm"] + 12.0 * cnt
        return tot

    def _latencies(self, S):
        lat = np.array([S.request(k)["latency"] for k in range(self.nreq)])
        st = S.stats()
        self.lat = {"p50_ms": float(np.percentile(lat, 50) * 1e3),
                    "p99_ms": float(np.percentile(lat, 99) * 1e3),
                    "admitted": st["admitted"], "rejected": st["rejected"],
                    "failed": st["failed"], "peak_hbm_gb": st["peak_bytes"] / 2**30,
                    "peak_concurrent": st["peak_active"],
                    "fused_runs": st["fused_runs"], "fused_requests": st["fused_requests"],
                    "makespan_s": st["makespan_s"]}
        return st

    def step_dev(self):
        self.S.replay(self.trace)
        st = self._latencies(self.S)
        # roofline over the whole replay: every request's bytes over the
        # makespan (idle gaps between arrivals included)
        self.alg_bytes = self._request_bytes(self.S)
        self.kernel_ms_override = 1e3 * st["makespan_s"]
        return st["completed"]

    def e2e_setup(self, torch):
        return 0, 0

    def step_e2e(self):
        S = self._server()
        S.replay(self.trace)
        st = S.stats()
        S.free()
        return st["completed"]

    def launches_per_step(self):
        # about 14 per request (a launch list of the first 300 requests of
        # this trace counts 4268): a saxpy3 product ~8 and an SSSP vxm step
        # ~14 (symbolic phase, heavy-row path, compaction, pack), a triangle
        # count 4 (small graphs) to 14 (bitmap path), plus the two-launch
        # device checksum reduction
        return 14 * self.nreq

    # the reference replays a bounded sample of the trace: its first requests,
    # with the same arrival times, through 8 host workers
    REF_SAMPLE = 400

    def _ref_trace(self):
        k = self.REF_SAMPLE
        t = self.trace
        return {"t": t["t"][:k], "kind": t["kind"][:k], "graph": t["graph"][:k],
                "fp": t["fp"][:k + 1], "fi": t["fi"], "fx": t["fx"]}

    def _ref_run(self, R, ncores, results=False):
        tr = self._ref_trace()
        per = max(1, ncores // 8)
        status, count, cs, lat, mk = R.serve(self.graphs, tr, 8, per)
        done = int((status == 0).sum())
        desc = ("first %d requests of the trace (same arrivals), 8 host workers x %d "
                "threads, p50 %.2f ms, p99 %.2f ms" %
                (self.REF_SAMPLE, per, 1e3 * np.percentile(lat, 50),
                 1e3 * np.percentile(lat, 99)))
        if results:
            return done, mk, desc, status, count, cs
        return done, mk, desc

    def cpu_baseline(self, R, ncores):
        """The reference replaying the trace's first requests, and the parity
        of those requests' results: counts (triangles, result entries) equal;
        checksums - sums of the result values, which the two libraries add
        in different orders - equal for triangle counts and within a
        recursive-summation bound (entries x eps x max(|sum|, entries)) for
        the fp32 SSSP and fp64 product results (their entries themselves
        are bit-identical to the reference's, as the serving tests check)."""
        done, mk, desc, status, count, cs = self._ref_run(R, ncores, results=True)
        bad = 0
        eps = {K_TRICOUNT: 0.0, K_SSSP: float(np.finfo(np.float32).eps),
               K_MXM: float(np.finfo(np.float64).eps)}
        for k in range(self.REF_SAMPLE):
            a = self.S.request(k)
            # n eps sum|x| bounds the order difference; |sum| stands in for
            # sum|x| with signed values' cancellation allowed for by n
            n = max(1, int(count[k]))
            tol = n * eps[int(self.trace["kind"][k])] * max(abs(cs[k]), float(n))
            if status[k] != 0 or a["status"] != 0 or a["count"] != int(count[k]):
                bad += 1
            elif abs(a["checksum"] - cs[k]) > tol:
                bad += 1
        parity = ("exact counts, checksums within the summation-order bound on the %d "
                  "replayed requests" % self.REF_SAMPLE if bad == 0 else
                  "MISMATCH: %d of %d requests differ" % (bad, self.REF_SAMPLE))
        return done / mk, desc, parity

    def reference_steps(self, R, steps, warmup):
        ncores = os.cpu_count() or 1
        for _ in range(warmup):
            self._ref_run(R, ncores)
        units, secs, desc = 0, 0.0, ""
        for _ in range(steps):
            done, mk, desc = self._ref_run(R, ncores)
            units += done
            secs += mk
        return units, secs, desc

    def free(self):
        self.S.free()
