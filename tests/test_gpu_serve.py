"""The request server: continuous batching over device-resident graphs.

* In the mix (8 slots, requests arriving faster than they finish, kernels of
  several requests overlapping on the device) every result equals the same
  request run alone (1 slot, no overlap), bit for bit, and matches the
  oracle (oracle/oracle.c).
* Admission: a request whose HBM footprint exceeds the budget is rejected
  with GrB_OUT_OF_MEMORY and the others still complete; the running set never
  holds more than the budget.
* Failure injection on the host: a device allocation that fails makes its
  request fail cleanly (GrB_OUT_OF_MEMORY) and the server carries on.
* Fusion: SSSP steps on one graph that wait together run as one product, one
  frontier per row; each result and checksum equals the request run alone,
  and a failure of the fused product is retried request by request.
"""

import numpy as np
import pytest

from graphblas_b200 import workloads as W
from tests.helpers import assert_exact

pytestmark = pytest.mark.gpu


def _graphs():
    from graphblas_b200.serve import make_graphs
    return make_graphs(seed=5, tc_scales=range(8, 11), n_sssp=1, n_mxm=2, mxm_nmax=3000)


def test_mixed_results_equal_alone_and_oracle(gpu, oracle):
    from graphblas_b200.serve import Server, make_trace, K_TRICOUNT, K_SSSP, K_MXM
    graphs = _graphs()
    trace = make_trace(graphs, nreq=180, rate=50000.0, seed=7)
    mix = Server(nslots=8, budget_bytes=8 << 30)
    for kind, g in graphs:
        mix.add_graph(kind, g)
    mix.replay(trace)
    st = mix.stats()
    assert st["completed"] == 180 and st["failed"] == 0 and st["rejected"] == 0
    assert st["peak_active"] > 1                     # requests overlapped
    alone = Server(nslots=1, budget_bytes=8 << 30, fuse=1)
    for kind, g in graphs:
        alone.add_graph(kind, g)
    slow = dict(trace)
    slow["t"] = np.arange(len(trace["t"])) * 1e-4    # one at a time, in order
    alone.replay(slow)
    assert alone.stats()["peak_active"] == 1
    assert alone.stats()["fused_runs"] == 0
    tri_cache = {}
    for k in range(180):
        kind = int(trace["kind"][k])
        g = graphs[int(trace["graph"][k])][1]
        a, b = mix.request(k), alone.request(k)
        assert a["status"] == 0 and b["status"] == 0
        assert a["count"] == b["count"]
        assert a["checksum"] == b["checksum"]
        if kind == K_TRICOUNT:
            gid = int(trace["graph"][k])
            if gid not in tri_cache:
                L, U = W.tril_triu(g)
                tri_cache[gid] = oracle.tricount(g.nrows, L.p, L.i, U.p, U.i)
            assert a["count"] == tri_cache[gid]
        else:
            ra, rb = mix.result(k, kind), alone.result(k, kind)
            assert_exact(ra, rb, "request %d mixed vs alone" % k)
            if k % 7 == 0:
                if kind == K_SSSP:
                    lo, hi = trace["fp"][k], trace["fp"][k + 1]
                    ui, ux = trace["fi"][lo:hi], trace["fx"][lo:hi]
                    u = (np.array([0, len(ui)], np.int64), ui, ux, 10)
                    want = oracle.saxpy(1, g.ncols, u, (g.p, g.i, g.x, 10), "MIN", "PLUS", 10)
                else:
                    want = oracle.saxpy(g.nrows, g.ncols, (g.p, g.i, g.x, 11),
                                        (g.p, g.i, g.x, 11), "PLUS", "TIMES", 11)
                assert_exact(ra, want, "request %d vs oracle" % k)
    mix.free()
    alone.free()


def test_admission_rejects_oversize_and_bounds_memory(gpu):
    from graphblas_b200.serve import Server, make_trace
    graphs = _graphs()
    trace = make_trace(graphs, nreq=60, rate=20000.0, seed=9)
    budget = 4 << 20                                  # 4 MiB: the big ones never fit
    S = Server(nslots=4, budget_bytes=budget)
    for kind, g in graphs:
        S.add_graph(kind, g)
    S.replay(trace)
    st = S.stats()
    assert st["rejected"] > 0
    assert st["completed"] + st["rejected"] + st["failed"] == 60
    assert st["completed"] > 0
    assert st["peak_bytes"] <= budget
    for k in range(60):
        r = S.request(k)
        assert r["status"] in (0, -102)
    S.free()


def test_injected_allocation_failure_is_isolated(gpu):
    from graphblas_b200.serve import Server, make_trace
    graphs = _graphs()
    trace = make_trace(graphs, nreq=40, rate=2000.0, seed=11)
    S = Server(nslots=1, budget_bytes=8 << 30, fuse=1)
    for kind, g in graphs:
        S.add_graph(kind, g)
    gpu.lib().grb_b200_debug_fail_alloc(3)            # the 3rd allocation fails
    S.replay(trace)
    gpu.lib().grb_b200_debug_fail_alloc(0)
    st = S.stats()
    assert st["failed"] == 1
    assert st["completed"] == 39
    statuses = [S.request(k)["status"] for k in range(40)]
    assert statuses.count(-102) == 1
    S.free()


def _sssp_burst(graphs, nreq, seed):
    """nreq SSSP steps on the first SSSP graph, all arriving at once."""
    from graphblas_b200.serve import make_trace, K_SSSP
    tr = make_trace(graphs, nreq=4 * nreq, rate=1e6, seed=seed)
    ks = [k for k in range(len(tr["kind"])) if tr["kind"][k] == K_SSSP][:nreq]
    gid = int(tr["graph"][ks[0]])
    ks = [k for k in ks if int(tr["graph"][k]) == gid]
    fp, fi, fx = [0], [], []
    for k in ks:
        lo, hi = tr["fp"][k], tr["fp"][k + 1]
        fi.append(tr["fi"][lo:hi])
        fx.append(tr["fx"][lo:hi])
        fp.append(fp[-1] + hi - lo)
    m = len(ks)
    return {"t": np.zeros(m), "kind": np.full(m, K_SSSP, np.int32),
            "graph": np.full(m, gid, np.int32), "fp": np.array(fp, np.int64),
            "fi": np.concatenate(fi), "fx": np.concatenate(fx)}, gid


def test_fused_sssp_equals_alone_and_oracle(gpu, oracle):
    from graphblas_b200.serve import Server, K_SSSP
    graphs = _graphs()
    burst, gid = _sssp_burst(graphs, 40, seed=13)
    m = len(burst["t"])
    assert m >= 8
    runs = {}
    for fuse in (1, 64):
        S = Server(nslots=1, budget_bytes=8 << 30, fuse=fuse)
        for kind, g in graphs:
            S.add_graph(kind, g)
        S.replay(burst)
        st = S.stats()
        assert st["completed"] == m and st["failed"] == 0
        if fuse == 1:
            assert st["fused_runs"] == 0
        else:
            # all arrive together, one worker: the first product takes them all
            assert st["largest_group"] == m and st["fused_requests"] == m
        runs[fuse] = ([S.request(k) for k in range(m)], [S.result(k, K_SSSP) for k in range(m)])
        S.free()
    g = graphs[gid][1]
    for k in range(m):
        a, b = runs[64][0][k], runs[1][0][k]
        assert a["count"] == b["count"] and a["checksum"] == b["checksum"]
        assert_exact(runs[64][1][k], runs[1][1][k], "request %d fused vs alone" % k)
        lo, hi = burst["fp"][k], burst["fp"][k + 1]
        u = (np.array([0, hi - lo], np.int64), burst["fi"][lo:hi], burst["fx"][lo:hi], 10)
        want = oracle.saxpy(1, g.ncols, u, (g.p, g.i, g.x, 10), "MIN", "PLUS", 10)
        assert_exact(runs[64][1][k], want, "request %d fused vs oracle" % k)


def test_fused_failure_is_retried_alone(gpu):
    from graphblas_b200.serve import Server, K_SSSP
    graphs = _graphs()
    burst, _ = _sssp_burst(graphs, 24, seed=17)
    m = len(burst["t"])
    S = Server(nslots=1, budget_bytes=8 << 30)
    for kind, g in graphs:
        S.add_graph(kind, g)
    gpu.lib().grb_b200_debug_fail_alloc(1)            # the fused product's first allocation
    S.replay(burst)
    gpu.lib().grb_b200_debug_fail_alloc(0)
    st = S.stats()
    assert st["largest_group"] == m
    assert st["failed"] == 0 and st["completed"] == m
    T = Server(nslots=1, budget_bytes=8 << 30, fuse=1)
    for kind, g in graphs:
        T.add_graph(kind, g)
    T.replay(burst)
    for k in range(m):
        a, b = S.request(k), T.request(k)
        assert a["status"] == 0 and a["count"] == b["count"] and a["checksum"] == b["checksum"]
        assert_exact(S.result(k, K_SSSP), T.result(k, K_SSSP), "request %d" % k)
    S.free()
    T.free()


def test_graphs_loaded_from_serialized_blobs(gpu):
    """Graphs registered from serialized blobs (the library's own writer, and
    the reference's ZSTD / LZ4 blobs where the reference is built here) serve
    the same results as the same graphs registered from CSR arrays."""
    from graphblas_b200 import grb
    from graphblas_b200.serve import Server, make_trace, K_SSSP, K_MXM
    from oracle import Reference, reference_available
    graphs = _graphs()
    trace = make_trace(graphs, nreq=60, rate=50000.0, seed=9)
    R = Reference(nthreads=2) if reference_available() else None
    csr, blob = Server(nslots=4, budget_bytes=8 << 30), Server(nslots=4, budget_bytes=8 << 30)
    for n, (kind, g) in enumerate(graphs):
        csr.add_graph(kind, g)
        t = {K_SSSP: 10, K_MXM: 11}.get(kind, 1)
        x = (np.ones(g.nnz, np.bool_) if t == 1 else
             np.ascontiguousarray(g.x, np.float32 if t == 10 else np.float64))
        if R is not None and n % 2 == 1:
            b = R.serialize(t, g.nrows, g.ncols, g.p, g.i, x, 2, n % 4 == 1,
                            1000 if n % 3 == 0 else 0)
        else:
            b = grb.blob_encode(g.nrows, g.ncols, t, g.p, g.i, x)
        blob.add_graph_blob(kind, b)
    for S in (csr, blob):
        S.replay(trace)
        assert S.stats()["completed"] == 60
    for k in range(60):
        a, b = csr.request(k), blob.request(k)
        assert a["status"] == 0 and b["status"] == 0
        assert a["count"] == b["count"] and a["checksum"] == b["checksum"]
    with pytest.raises(RuntimeError):
        g = graphs[0][1]
        wrong = grb.blob_encode(g.nrows, g.ncols, 8, g.p, g.i, np.ones(g.nnz, np.int64))
        blob.add_graph_blob(K_MXM, wrong)              # an int64 blob for an fp64 kind
    for S in (csr, blob):
        S.free()
