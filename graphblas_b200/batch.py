"""Batched products C_k = A_k * B_k through grb_b200_batch_* (include/grb_b200.h).

``Batch`` wraps one batch handle (block-diagonal upload, symbolic phase,
autotuning, CUDA-graph replay, result download).  ``BenchBatch`` is the
batched workload of bench.py: 4096 independent C_k = A_k*A_k with the min_plus
fp32 semiring, n_k log-uniform in [64, 8192], Poisson(6) entries per row.
"""

import ctypes
import time

import numpy as np

from . import lib as _lib, check, semiring, TYPES, NP_OF, workloads as W

vp = ctypes.c_void_p
_libc = ctypes.CDLL(None)
_libc.free.argtypes = [vp]


def _bind(L):
    if getattr(L, "_batch_bound", False):
        return L
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.grb_b200_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp, vp, vp, vp,
                                        vp, vp, vp, vp, vp, vp]
    L.grb_b200_batch_tune.argtypes = [vp, ctypes.c_bool, ctypes.POINTER(ctypes.c_double)]
    L.grb_b200_batch_run.argtypes = [vp, ctypes.c_bool]
    L.grb_b200_batch_enqueue.argtypes = [vp, vp]
    L.grb_b200_batch_info.argtypes = [vp, i64p, i64p, i64p, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_int)]
    L.grb_b200_batch_result.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                        ctypes.POINTER(vp), vp]
    L.grb_b200_batch_result_into.argtypes = [vp, vp, vp, vp, vp]
    L.grb_b200_batch_free.argtypes = [ctypes.POINTER(vp)]
    for n in ("create", "tune", "run", "enqueue", "info", "result", "result_into", "free"):
        getattr(L, "grb_b200_batch_" + n).restype = ctypes.c_int
    L._batch_bound = True
    return L


def concat(mats, dtype=None):
    """Concatenated CSR of a list of Csr (offsets continue across instances)."""
    rows = np.array([a.nrows for a in mats], np.int64)
    cols = np.array([a.ncols for a in mats], np.int64)
    nnz = np.array([a.nnz for a in mats], np.int64)
    eoff = np.concatenate([[0], np.cumsum(nnz)]).astype(np.int64)
    P = np.concatenate([a.p + eoff[k] for k, a in enumerate(mats)]).astype(np.int64)
    J = np.concatenate([a.i for a in mats]).astype(np.int64) if nnz.sum() else np.zeros(1, np.int64)
    X = None
    if mats[0].x is not None:
        X = np.concatenate([a.x for a in mats])
        if dtype is not None:
            X = X.astype(dtype)
    return rows, cols, P, J, X


class Batch:
    def __init__(self, mats, sr, bmats=None, concatenated=None):
        self.L = _bind(_lib())
        self.sr = sr
        self.dt = NP_OF[sr.type]
        if concatenated is not None:
            rows, cols, P, J, X = concatenated
        else:
            rows, cols, P, J, X = concat(mats, self.dt)
        self.count = len(rows)
        self.rows = rows
        self._keep = [rows, cols, P, J, X]
        bp = bj = bx = bcols = None
        if bmats is not None:
            _, bcols, bp, bj, bx = concat(bmats, self.dt)
            self._keep += [bcols, bp, bj, bx]
        h = vp()
        d = lambda a: None if a is None else a.ctypes.data
        check(self.L.grb_b200_batch_create(ctypes.byref(h), self.count, d(rows), d(cols),
                                           d(P), d(J), d(X), d(bcols), d(bp), d(bj), d(bx),
                                           ctypes.byref(sr)), "batch_create")
        self.h = h

    def tune(self, use_cache=True):
        ms = ctypes.c_double()
        check(self.L.grb_b200_batch_tune(self.h, use_cache, ctypes.byref(ms)), "batch_tune")
        return ms.value

    def run(self, use_graph=True):
        check(self.L.grb_b200_batch_run(self.h, use_graph), "batch_run")

    def enqueue(self, stream=None):
        check(self.L.grb_b200_batch_enqueue(self.h, stream), "batch_enqueue")

    def info(self):
        r, n, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        nb, gk = ctypes.c_int(), ctypes.c_int()
        ms = ctypes.c_double()
        check(self.L.grb_b200_batch_info(self.h, ctypes.byref(r), ctypes.byref(n),
                                         ctypes.byref(c), ctypes.byref(nb), ctypes.byref(ms),
                                         ctypes.byref(gk)))
        return dict(total_rows=r.value, nnz=n.value, capacity=c.value, nbins=nb.value,
                    tuned_ms=ms.value, graph_kernels=gk.value)

    def result_arrays(self):
        """Concatenated results (P offsets per instance into J/X) and the
        per-instance entry counts, without splitting."""
        cp, cj, cx = vp(), vp(), vp()
        nnzk = np.zeros(self.count, np.int64)
        check(self.L.grb_b200_batch_result(self.h, ctypes.byref(cp), ctypes.byref(cj),
                                           ctypes.byref(cx), nnzk.ctypes.data), "batch_result")
        tot = int(nnzk.sum())
        P = _take(cp.value, int(np.sum(self.rows + 1)), np.int64)
        return P, _take(cj.value, tot, np.int64), _take(cx.value, tot, self.dt), nnzk

    def result_into(self, P, J, X, nnzk):
        """Results into caller buffers given as raw host addresses (P offsets
        per instance, J/X entries, nnzk per-instance entry counts)."""
        check(self.L.grb_b200_batch_result_into(self.h, P, J, X, nnzk), "batch_result_into")

    def result(self):
        """[(p, i, x)] per instance (local indices, sorted rows)."""
        cp, cj, cx = vp(), vp(), vp()
        nnzk = np.zeros(self.count, np.int64)
        check(self.L.grb_b200_batch_result(self.h, ctypes.byref(cp), ctypes.byref(cj),
                                           ctypes.byref(cx), nnzk.ctypes.data), "batch_result")
        nP = int(np.sum(self.rows + 1))
        tot = int(nnzk.sum())
        P = _take(cp.value, nP, np.int64)
        J = _take(cj.value, tot, np.int64)
        X = _take(cx.value, tot, self.dt)
        out = []
        po = 0
        for k in range(self.count):
            n = int(self.rows[k])
            p = P[po:po + n + 1]
            lo, hi = int(p[0]), int(p[-1])
            out.append((p - lo, J[lo:hi], X[lo:hi]))
            po += n + 1
        return out

    def free(self):
        if self.h and self.h.value:
            self.L.grb_b200_batch_free(ctypes.byref(self.h))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _take(ptr, n, dt):
    dt = np.dtype(dt)
    if not ptr:
        return np.zeros(0, dt)
    if n == 0:
        _libc.free(ptr)
        return np.zeros(0, dt)
    buf = (ctypes.c_char * (n * dt.itemsize)).from_address(ptr)
    out = np.frombuffer(buf, dtype=dt).copy()
    _libc.free(ptr)
    return out


class BenchBatch:
    """bench.py --config batch: 4096 C_k = A_k*A_k, min_plus fp32."""
    metric, unit, dtype, kernel = "GFLOP/s", "GFLOP/s", "fp32", "saxpy3_numeric"

    def __init__(self, args):
        self.count = 4096
        self.mats = W.batch_min_plus(count=self.count, seed=11 + args.seed)
        self.products = 0
        for a in self.mats:
            deg = np.diff(a.p)
            self.products += int(np.sum(deg[a.i]))
        self.flops = 2.0 * self.products
        self.workload = "batch4096_min_plus_fp32_n64-8192_poisson6"
        self.sizes = np.array([a.nrows for a in self.mats], np.int64)

    def config(self):
        return {"instances": self.count, "rows": int(self.sizes.sum()),
                "nnz_A": int(sum(a.nnz for a in self.mats)), "products": self.products,
                "tuned_ms": getattr(self, "tuned_ms", None),
                "per_call_gpu_ms": getattr(self, "per_call_ms", None),
                "speedup_vs_per_call_gpu": getattr(self, "speedup", None),
                "graph": True}

    def dev_setup(self, gb):
        self.gb = gb
        self.sr = semiring("MIN", "PLUS", "fp32")
        self.B = Batch(self.mats, self.sr)
        self.tuned_ms = self.B.tune(use_cache=False)
        # one eager run with kernel timing for the roofline line
        L = self.B.L
        L.grb_b200_profile_reset()
        L.grb_b200_profile_enable(True)
        self.B.run(use_graph=False)
        L.grb_b200_profile_enable(False)
        ms, cnt = ctypes.c_double(), ctypes.c_int64()
        L.grb_b200_profile(b"saxpy3_numeric", ctypes.byref(ms), ctypes.byref(cnt))
        self.kernel_ms_override = ms.value / max(cnt.value, 1)
        self.B.run(use_graph=True)
        self.graph_kernels = self.B.info()["graph_kernels"]
        nnz = self.B.info()["nnz"]
        # algorithmic bytes: A once (4 B index + 4 B value) + B rows per product
        # + C once, per the batched workload's per-instance figure summed
        nnzA = sum(a.nnz for a in self.mats)
        self.alg_bytes = (8.0 * nnzA + 4.0 * (self.sizes.sum() + self.count) +
                          8.0 * self.products + 8.0 * nnz + 4.0 * (self.sizes.sum() + self.count))
        self.basis = ("every instance's A once and C once (row offsets, 4-byte indices, "
                      "fp32 values) plus the B row of every product (index and value)")
        self.per_call_ms = self.time_per_call()
        self.speedup = None

    def time_per_call(self):
        """The plain path: one GrB_mxm per instance through the GraphBLAS API
        (device-resident inputs), over all instances of the batch; host
        clock around the loop (each call returns when its product is done),
        device synchronised on both sides."""
        from .grb import API
        import torch
        api = API()
        As = [api.matrix_from_csr(a) for a in self.mats]
        Cs = [api.matrix_new(10, a.nrows, a.ncols) for a in self.mats]
        for A, C in zip(As, Cs):            # warm (uploads the inputs)
            api.mxm(C, None, None, "GrB_MIN_PLUS_SEMIRING_FP32", A, A)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for A, C in zip(As, Cs):
            api.mxm(C, None, None, "GrB_MIN_PLUS_SEMIRING_FP32", A, A)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        for X in As + Cs:
            api.free(X)
        return 1e3 * dt

    def digests(self):
        """oracle.csr_digest of every instance's result (the batch's last
        run), for the comparison with the reference's own results."""
        from oracle import csr_digest
        return np.array([csr_digest(*r) for r in self.B.result()], np.uint64)

    def step_dev(self):
        self.B.run(use_graph=True)
        return self.flops / 1e9

    def e2e_setup(self, torch):
        # the batch as a caller holds it: concatenated arrays in page-locked
        # host memory, and page-locked arrays for the results
        rows, cols, P, J, X = concat(self.mats, np.float32)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        self.pin_in = [pin(rows), pin(cols), pin(P), pin(J), pin(X)]
        self.cat = tuple(t.numpy() for t in self.pin_in)
        nnz_c = max(self.B.info()["nnz"], 0)
        n_p = int(self.sizes.sum() + self.count)
        self.pin_out = [torch.empty(n_p, dtype=torch.int64).pin_memory(),
                        torch.empty(max(nnz_c, 1), dtype=torch.int64).pin_memory(),
                        torch.empty(max(nnz_c, 1), dtype=torch.float32).pin_memory()]
        self.nnzk = np.zeros(self.count, np.int64)
        nb = lambda t: int(t.numel() * t.element_size())
        return sum(nb(t) for t in self.pin_in[2:]), 8 * n_p + 12 * nnz_c

    def step_e2e(self):
        # upload + symbolic phase with the cached tuning choice + one numeric
        # pass (eager: a single run does not pay for a graph capture) + results
        B = Batch(None, self.sr, concatenated=self.cat)
        B.tune(use_cache=True)
        B.run(use_graph=False)
        B.result_into(*(t.data_ptr() for t in self.pin_out), self.nnzk.ctypes.data)
        B.free()
        return self.flops / 1e9

    def launches_per_step(self):
        return self.graph_kernels

    def finish(self, dev_ms_per_step):
        self.speedup = self.per_call_ms / dev_ms_per_step if dev_ms_per_step else None

    def _ref_inputs(self):
        rows, cols, P, J, X = concat(self.mats, np.float32)
        poff = np.concatenate([[0], np.cumsum(rows + 1)[:-1]]).astype(np.int64)
        ioff = P[poff]                        # first entry of each instance
        return rows, poff, ioff, P, J, X

    def cpu_baseline(self, R, ncores):
        """The reference's loop of GrB_mxm calls over all instances, and the
        parity of every instance: the digests of the reference's results
        against those of the batch's."""
        rows, poff, ioff, P, J, X = self._ref_inputs()
        nnz, secs, ref = R.batch_square(rows, poff, ioff, P, J, X, digests=True)
        got = self.digests()
        bad = int(np.sum(got != ref))
        parity = ("exact: all %d instances bit-identical to the reference" % self.count
                  if bad == 0 else "MISMATCH: %d of %d instances differ" % (bad, self.count))
        return (self.flops / 1e9 / secs,
                "all 4096 instances, one GrB_mxm each (%.2f s)" % secs, parity)

    def reference_steps(self, R, steps, warmup):
        rows, poff, ioff, P, J, X = self._ref_inputs()
        for _ in range(warmup):
            R.batch_square(rows, poff, ioff, P, J, X)
        tot = 0.0
        for _ in range(steps):
            _, secs = R.batch_square(rows, poff, ioff, P, J, X)
            tot += secs
        return self.flops / 1e9 * steps, tot, "all 4096 instances per step, one GrB_mxm each"

    def free(self):
        self.B.free()
