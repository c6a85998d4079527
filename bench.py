#!/usr/bin/env python
"""Benchmark of the B200 semiring SpGEMM path (SuiteSparse:GraphBLAS GrB_mxm).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config all|tc|saxpy|bfs|bfs_pushpull|batch|serve]

Workloads (seeded synthetic inputs of the graph500 / Erdos-Renyi shapes the
reference is measured on; no dataset is read):

  tc     (the headline) masked dot3 triangle counting, C<L> = L*U' with
         plus_pair int64 then a sum reduction, on a symmetrised R-MAT graph of
         scale 20, edge factor 16, (a,b,c,d) = (0.57,0.19,0.19,0.05),
         self-loops and duplicates removed.  One step = GrB_mxm + GrB_reduce
         over the whole graph; metric triangles/s.
  saxpy  C = A*B, plus_times fp64, A and B 16384x16384 Erdos-Renyi with 8
         uniform columns per row, values U[-1,1]; metric GFLOP/s (2 flops per
         product).
  bfs    level-synchronous BFS parents (GrB_vxm any_secondi int64 with a
         complemented structural mask and replace, then GrB_assign) on R-MAT
         scale 22, edge factor 16; metric TEPS (undirected edges / s).
  bfs_pushpull  the same traversal direction-optimising: levels with a large
         frontier pull (GrB_mxv max_secondi on S, its own transpose), the
         others push; the parents are the push-only traversal's, bit for bit.
  batch  4096 independent C_k = A_k*A_k, min_plus fp32, n_k log-uniform in
         [64, 8192], Poisson(6) entries per row; metric GFLOP/s.
  serve  an open-loop Poisson stream (2000 req/s) of mixed requests on
         device-resident graphs; metric req/s with p50/p99 latency.

The default (--config all) prints one line: the tc workload's figures at the
top level and the other five under "configs", each with its own value, e2e,
roofline, cpu_baseline and parity.

* value: device time with the inputs resident in HBM, CUDA events on the
  launching stream, L2 flushed (a 256 MB write) between steps, max over ranks.
* e2e: the same step through the public API from pinned host buffers, the
  host->device copies and the result read-back inside the timed region.
* roofline: bytes per launch of the dominant kernel (or kernel phase) over
  its event-timed duration, against the measured HBM copy bandwidth; the
  byte basis of each workload is named in the line ("basis").
* cpu_baseline: the reference library (oracle/_ref, SuiteSparse:GraphBLAS
  built from its own sources) on this host's cores, same inputs, with the
  parity of the device's result against the reference's ("parity").

--impl reference times the reference's CPU path alone and prints its line.
Multi-GPU (torchrun): every rank runs an independent replica (the path has no
exchange step); value = all ranks' units / the max step time.
"""

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
# the timed loop records the hot kernel's events around one launch in this many
PROF_EVERY = 4
sys.path.insert(0, ROOT)

from graphblas_b200 import workloads as W  # noqa: E402


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        ok = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in ok if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in ok if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in ok:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

def scan_launches(n, tile=4096, single=8192):
    """Kernel launches of the library's device scan of n values: one block
    scans up to 8192 values in one launch; longer arrays take a tile-sum
    launch and a tile-scan launch around the scan of the tile sums."""
    if n <= single:
        return 1
    nb = (n + tile - 1) // tile
    return 2 + scan_launches(nb, tile, single)


class TriCount:
    metric, unit, dtype, kernel = "triangles/s", "triangles/s", "int64", "dot3"

    def __init__(self, args):
        self.scale = args.scale or 20
        S = W.rmat(self.scale, 16, seed=args.seed)
        self.S = S
        self.L, self.U = W.tril_triu(S)
        n, nnz = S.nrows, self.L.nnz
        # compulsory bytes of one call (int32 offsets and indices in HBM):
        # L, U and the mask (L again, read by its own pass) once each, C
        # written once (offsets, indices, int64 counts)
        self.alg_bytes = 3.0 * (4.0 * (n + 1) + 4.0 * nnz) + 4.0 * (n + 1) + 12.0 * nnz
        self.basis = ("compulsory: L, U and the mask read once, C written once "
                      "(4-byte offsets and indices, 8-byte counts)")
        dL = np.diff(self.L.p).astype(np.float64)
        dU = np.diff(self.U.p).astype(np.float64)
        # the merge-equivalent figure: every mask entry merging its two rows
        self.merge_equiv_bytes = 4.0 * (np.sum(dL * dL) + np.sum(dU * dU)) + 16.0 * nnz
        self.workload = "tricount_rmat%d_ef16_dot3_plus_pair" % self.scale
        # DRAM bytes of one dot3 call at scale 20 (dram__bytes_read.sum +
        # dram__bytes_write.sum over its kernels, one ncu capture of this
        # workload at this size)
        self.traffic_per_launch = TC_TRAFFIC_RMAT20 if self.scale == 20 else None

    def config(self):
        return {"n": int(self.S.nrows), "nnz_L": int(self.L.nnz),
                "triangles": int(getattr(self, "ntri", -1))}

    def dev_setup(self, gb):
        self.gb = gb
        self.dL = gb.DMatrix.upload(self.L, "bool")
        self.dU = gb.DMatrix.upload(self.U, "bool")
        self.sr = gb.semiring("PLUS", "PAIR", "int64")

    def step_dev(self):
        gb = self.gb
        C = gb.dot3(self.dL, self.dL, self.dU, self.sr)
        n = int(gb.reduce(C, "PLUS", np.int64))
        C.free()
        self.ntri = n
        return n

    def e2e_setup(self, torch):
        self.pin = {k: torch.from_numpy(v).pin_memory() for k, v in
                    (("Lp", self.L.p), ("Li", self.L.i), ("Up", self.U.p), ("Ui", self.U.i))}
        return sum(int(t.numel() * t.element_size()) for t in self.pin.values()), 8

    def step_e2e(self):
        gb = self.gb
        L_ = gb.lib()
        hL, hU = ctypes.c_void_p(), ctypes.c_void_p()
        gb.check(L_.grb_b200_dmatrix_upload(ctypes.byref(hL), self.L.nrows, self.L.ncols,
                                            self.pin["Lp"].data_ptr(), self.pin["Li"].data_ptr(),
                                            None, 1, True))
        gb.check(L_.grb_b200_dmatrix_upload(ctypes.byref(hU), self.U.nrows, self.U.ncols,
                                            self.pin["Up"].data_ptr(), self.pin["Ui"].data_ptr(),
                                            None, 1, True))
        dl, du = gb.DMatrix(hL.value), gb.DMatrix(hU.value)
        C = gb.dot3(dl, dl, du, self.sr)
        n = int(gb.reduce(C, "PLUS", np.int64))
        for d in (C, dl, du):
            d.free()
        assert n == self.ntri
        return n

    def launches_per_step(self):
        # the counting path (masks of 1024+ entries): classify, plan, route,
        # the warp-hash and block-bitmap count kernels and the merge kernel;
        # the sum of C comes back with the call, so the reduction launches
        # nothing.  Smaller masks: classify and intersect, then the two
        # reduction launches.
        if self.L.nnz < 1024:
            return 4
        return 6

    def cpu_baseline(self, R, ncores):
        ntri, times = R.tricount(self.S.nrows, self.L.p, self.L.i, self.U.p, self.U.i, reps=5)
        t = float(np.median(times))
        parity = ("exact: %d triangles, the reference's count" % ntri if ntri == self.ntri
                  else "MISMATCH: reference %d, device %d" % (ntri, self.ntri))
        return (ntri / t, "whole graph, GrB_mxm + GrB_reduce, median of 5 (%.2f s)" % t,
                parity)

    def reference_steps(self, R, steps, warmup):
        for _ in range(warmup):
            R.tricount(self.S.nrows, self.L.p, self.L.i, self.U.p, self.U.i, reps=1)
        ntri, times = R.tricount(self.S.nrows, self.L.p, self.L.i, self.U.p, self.U.i,
                                 reps=steps)
        self.ntri = ntri
        return ntri * steps, float(np.sum(times)), "whole graph per step (GrB_mxm + GrB_reduce)"

    def free(self):
        for d in ("dL", "dU"):
            if hasattr(self, d):
                getattr(self, d).free()


class Saxpy:
    metric, unit, dtype, kernel = "GFLOP/s", "GFLOP/s", "fp64", "saxpy3_numeric"

    def __init__(self, args):
        n = 16384
        self.n = n
        self.A = W.er_fixed(n, n, 8, seed=args.seed + 1)
        self.B = W.er_fixed(n, n, 8, seed=args.seed + 2)
        deg = np.diff(self.B.p)
        self.products = int(np.sum(deg[self.A.i]))
        self.flops = 2.0 * self.products
        self.workload = "saxpy3_er16384_d8_plus_times_fp64"
        # DRAM bytes of the one-launch product kernel per launch (ncu capture
        # of this workload at this size: the inputs come from L2, the written
        # slots stay there)
        self.traffic_per_launch = 3.46e6

    def config(self):
        return {"n": self.n, "nnz_A": int(self.A.nnz), "products": self.products,
                "nnz_C": int(getattr(self, "nnz_c", -1))}

    def dev_setup(self, gb):
        from graphblas_b200.grb import API
        self.gb = gb
        self.api = API()
        self.Ag = self.api.matrix_from_csr(self.A)
        self.Bg = self.api.matrix_from_csr(self.B)
        self.Cg = self.api.matrix_new(11, self.n, self.n)
        self.api.mxm(self.Cg, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", self.Ag, self.Bg)
        self.nnz_c = self.api.nvals(self.Cg)
        # algorithmic bytes (4 B index, 8 B value): A once, B rows per product, C once
        self.alg_bytes = (4.0 * (self.n + 1) + 12.0 * self.A.nnz + 12.0 * self.products +
                          12.0 * self.nnz_c + 4.0 * (self.n + 1))
        self.basis = ("A once, the B row of every product, C once (4-byte indices, "
                      "8-byte values); the 27 MB problem fits in L2")

    def step_dev(self):
        self.api.mxm(self.Cg, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", self.Ag, self.Bg)
        return self.flops / 1e9

    def e2e_setup(self, torch):
        # the caller's arrays live in page-locked host memory; GrB_Matrix_import
        # copies them to HBM and GrB_Matrix_export copies C back
        def pin(a):
            return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        n, nc = self.n, self.nnz_c
        self.pin = {"Ap": pin(self.A.p), "Ai": pin(self.A.i), "Ax": pin(self.A.x),
                    "Bp": pin(self.B.p), "Bi": pin(self.B.i), "Bx": pin(self.B.x),
                    "Cp": torch.empty(n + 1, dtype=torch.int64).pin_memory(),
                    "Ci": torch.empty(nc, dtype=torch.int64).pin_memory(),
                    "Cx": torch.empty(nc, dtype=torch.float64).pin_memory()}
        nb = lambda k: int(self.pin[k].numel() * self.pin[k].element_size())
        return (sum(nb(k) for k in ("Ap", "Ai", "Ax", "Bp", "Bi", "Bx")),
                sum(nb(k) for k in ("Cp", "Ci", "Cx")))

    def step_e2e(self):
        api, P, n = self.api, self.pin, self.n
        A = api.matrix_import(11, n, n, P["Ap"].data_ptr(), P["Ai"].data_ptr(),
                              P["Ax"].data_ptr(), self.A.nnz)
        B = api.matrix_import(11, n, n, P["Bp"].data_ptr(), P["Bi"].data_ptr(),
                              P["Bx"].data_ptr(), self.B.nnz)
        C = api.matrix_new(11, n, n)
        api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, B)
        nv = api.matrix_export(C, 11, P["Cp"].data_ptr(), P["Ci"].data_ptr(),
                               P["Cx"].data_ptr(), n + 1, self.nnz_c)
        for X in (A, B, C):
            api.free(X)
        assert nv == self.nnz_c
        return self.flops / 1e9

    def launches_per_step(self):
        # the one-launch product kernel (products per row, slots,
        # expand-sort-compress, C's offsets and entries) and the read of
        # nnz(C)
        return 2

    def cpu_baseline(self, R, ncores):
        from oracle import csr_digest
        reps = 5
        args = (self.n, self.n, self.n, (self.A.p, self.A.i, self.A.x, 11),
                (self.B.p, self.B.i, self.B.x, 11), "PLUS", "TIMES", 11)
        ref = R.mxm(*args)
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            R.mxm(*args)
            times.append(time.perf_counter() - t0)
        t = float(np.median(times))
        got = self.api.matrix_to_csr(self.Cg, 11, self.n)
        same = csr_digest(*got) == csr_digest(*ref)
        parity = ("exact: C bit-identical to the reference's (%d entries)" % len(ref[1])
                  if same else "MISMATCH: C differs from the reference's")
        return (self.flops / 1e9 / t,
                "whole product, median of %d incl. CSR pack/unpack (%.1f ms)" % (reps, 1e3 * t),
                parity)

    def reference_steps(self, R, steps, warmup):
        for _ in range(warmup):
            R.mxm(self.n, self.n, self.n, (self.A.p, self.A.i, self.A.x, 11),
                  (self.B.p, self.B.i, self.B.x, 11), "PLUS", "TIMES", 11)
        tot = 0.0
        for _ in range(steps):
            t0 = time.perf_counter()
            R.mxm(self.n, self.n, self.n, (self.A.p, self.A.i, self.A.x, 11),
                  (self.B.p, self.B.i, self.B.x, 11), "PLUS", "TIMES", 11)
            tot += time.perf_counter() - t0
        return self.flops / 1e9 * steps, tot, "whole product per step (GrB_mxm + wait + CSR pack/unpack)"

    def free(self):
        if hasattr(self, "api"):
            for X in (self.Ag, self.Bg, self.Cg):
                self.api.free(X)


class Bfs:
    metric, unit, dtype, kernel = "TEPS", "edges/s", "int64", "saxpy3_numeric"

    def __init__(self, args):
        self.scale = args.scale or 22
        self.S = W.rmat(self.scale, 16, seed=args.seed)
        self.n = self.S.nrows
        deg = np.diff(self.S.p)
        self.src = int(np.argmax(deg > 0))          # first vertex with an edge
        self.edges = self.S.nnz // 2
        self.workload = "bfs_rmat%d_ef16_vxm_any_secondi" % self.scale

    def config(self):
        return {"n": int(self.n), "nnz_S": int(self.S.nnz), "source": self.src,
                "levels": int(getattr(self, "levels", -1)),
                "reached": int(getattr(self, "reached", -1))}

    def dev_setup(self, gb):
        from graphblas_b200.grb import API
        self.gb = gb
        self.api = API()
        self.Sg = self.api.matrix_from_csr(self.S, 1)
        # bytes of the whole traversal: every row once (8 B of row offsets and
        # 4 B per index, as if every vertex were reached) plus 8 B parent
        # writes
        self.alg_bytes = 8.0 * self.n + 4.0 * self.S.nnz + 8.0 * self.n
        self.basis = "S read once (offsets and indices), the parent vector written once"
        # DRAM bytes of the traversal's numeric launches (one per level): the
        # dense-row product kernel read and wrote 744 MB over a traversal in
        # one ncu capture at this size (the dense row itself stays in L2);
        # the other kernels of the level move little.  Per numeric launch:
        self.traffic_per_launch = 744e6 / 6 if self.scale == 22 else None

    def bfs(self, Sg):
        api = self.api
        n, src = self.n, self.src
        q = api.vector_from([src], [src], 8, n)
        p = api.vector_from([src], [src], 8, n)
        lev = 0
        while True:
            lev += 1
            api.vxm(q, p, None, "GxB_ANY_SECONDI_INT64", q, Sg, "GrB_DESC_RSC")
            if api.vnvals(q) == 0:
                break
            api.assign_all(p, q, None, q, n, "GrB_DESC_S")
        self.levels = lev
        return q, p

    def step_dev(self):
        q, p = self.bfs(self.Sg)
        self.reached = self.api.vnvals(p)
        self.api.vfree(q)
        self.api.vfree(p)
        return self.edges

    def parents(self):
        """The parent vector of one more traversal (untimed), dense."""
        q, p = self.bfs(self.Sg)
        idx, par = self.api.vector_to(p, 8)
        self.api.vfree(q)
        self.api.vfree(p)
        out = np.full(self.n, -1, np.int64)
        out[idx] = par
        return out

    def e2e_setup(self, torch):
        # S arrives from page-locked host memory through GrB_Matrix_import
        # (pattern values as bool ones); the parent vector goes back through
        # GrB_Vector_extractTuples
        def pin(a):
            return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        self.pin = {"Sp": pin(self.S.p), "Si": pin(self.S.i),
                    "Sx": pin(np.ones(self.S.nnz, np.bool_)),
                    "Pi": torch.empty(self.n, dtype=torch.int64).pin_memory(),
                    "Px": torch.empty(self.n, dtype=torch.int64).pin_memory()}
        nb = lambda k: int(self.pin[k].numel() * self.pin[k].element_size())
        return nb("Sp") + nb("Si") + nb("Sx"), 16 * int(getattr(self, "reached", self.n))

    def step_e2e(self):
        api, P = self.api, self.pin
        Sg = api.matrix_import(1, self.n, self.n, P["Sp"].data_ptr(), P["Si"].data_ptr(),
                               P["Sx"].data_ptr(), self.S.nnz)
        q, p = self.bfs(Sg)
        nv = api.vector_extract(p, 8, P["Pi"].data_ptr(), P["Px"].data_ptr(), self.n)
        for v in (q, p):
            api.vfree(v)
        api.free(Sg)
        assert nv == self.reached
        return self.edges

    def launches_per_step(self):
        # levels whose frontier makes the row heavy go straight to the dense
        # row: prep, product-index scan, products, compaction, row-offset
        # scan, pack (6); the first and last levels (small frontiers) take
        # the binned path first: flop counts, bins, slot scan, bin fill,
        # three bin kernels, row-offset scan, then the dense row (14); each
        # parent assign but the last level's is one union launch
        lev = max(getattr(self, "levels", 1), 1)
        return 2 * 14 + 6 * max(lev - 2, 0) + (lev - 1)

    def cpu_baseline(self, R, ncores):
        """The reference's traversal on all cores, timed (median of 3), and
        parity against the single-threaded reference (the max-parent rule of
        its ANY monoid is exact there)."""
        times = []
        for _ in range(3):
            _, secs, nlev = R.bfs(self.n, self.S.p, self.S.i, self.src)
            times.append(secs)
        t = float(np.median(times))
        nt = R.nthreads
        R.set_nthreads(1)
        ref, _, _ = R.bfs(self.n, self.S.p, self.S.i, self.src)
        R.set_nthreads(nt)
        got = self.parents()
        bad = int(np.sum(got != ref))
        parity = ("exact: all %d parents equal the single-threaded reference's" % self.n
                  if bad == 0 else "MISMATCH: %d parents differ" % bad)
        return (self.edges / t, "whole traversal, vxm + assign per level, median of 3 "
                "(%.3f s)" % t, parity)

    def reference_steps(self, R, steps, warmup):
        for _ in range(warmup):
            R.bfs(self.n, self.S.p, self.S.i, self.src)
        tot = 0.0
        for _ in range(steps):
            _, secs, _ = R.bfs(self.n, self.S.p, self.S.i, self.src)
            tot += secs
        return self.edges * steps, tot, "whole traversal per step"

    def free(self):
        if hasattr(self, "api"):
            self.api.free(self.Sg)


class BfsPushPull(Bfs):
    """The same traversal, direction-optimising: a level whose frontier holds
    more than n/32 vertices pulls - GrB_mxv(q, p, MAX_SECONDI, S, q, RSC),
    S being symmetric its own transpose, each unvisited vertex walking its
    row from the end to its largest frontier neighbour - and the others push
    as before.  Both directions pick the largest frontier neighbour, so the
    parents are those of the push-only traversal, bit for bit."""

    # the roofline covers the whole traversal (pull and push levels): the
    # traversal's algorithmic bytes over its device time
    kernel = "bfs_traversal"

    def __init__(self, args):
        super().__init__(args)
        self.workload = "bfs_rmat%d_ef16_push_pull_max_secondi" % self.scale

    def dev_setup(self, gb):
        super().dev_setup(gb)
        self.basis = ("S read once (offsets and indices), the parent vector written once, "
                      "over the whole traversal's device time")
        self.traffic_per_launch = None

    def finish(self, ms_per_step):
        self.kernel_ms_override = ms_per_step

    def bfs(self, Sg):
        api = self.api
        n, src = self.n, self.src
        q = api.vector_from([src], [src], 8, n)
        p = api.vector_from([src], [src], 8, n)
        lev = pulls = 0
        while True:
            lev += 1
            if api.vnvals(q) > n // 32:
                api.mxv(q, p, None, "GxB_MAX_SECONDI_INT64", Sg, q, "GrB_DESC_RSC")
                pulls += 1
            else:
                api.vxm(q, p, None, "GxB_ANY_SECONDI_INT64", q, Sg, "GrB_DESC_RSC")
            if api.vnvals(q) == 0:
                break
            api.assign_all(p, q, None, q, n, "GrB_DESC_S")
        self.levels, self.pull_levels = lev, pulls
        return q, p

    def config(self):
        c = super().config()
        c["pull_levels"] = int(getattr(self, "pull_levels", -1))
        return c

    def launches_per_step(self):
        # a pull level: two bitmap scatters, the row kernel, the scan over
        # the 32-row groups and the compaction (5); push levels as in the
        # push-only traversal; one union per parent update
        lev = max(getattr(self, "levels", 1), 1)
        pulls = max(getattr(self, "pull_levels", 0), 0)
        push = lev - pulls
        return 5 * pulls + 14 * min(push, 2) + 6 * max(push - 2, 0) + (lev - 1)


CONFIGS = {"tc": TriCount, "saxpy": Saxpy, "bfs": Bfs, "bfs_pushpull": BfsPushPull}
SUB_CONFIGS = ("saxpy", "bfs", "bfs_pushpull", "batch", "serve")

# DRAM bytes (read + write) of one triangle-count dot3 call at R-MAT scale 20,
# summed over its six kernels from one ncu capture of this workload at this
# size (dram__bytes_read.sum + dram__bytes_write.sum)
TC_TRAFFIC_RMAT20 = 2.98e9


def make_batch(args):
    from graphblas_b200 import batch as B
    return B.BenchBatch(args)


def make_serve(args):
    from graphblas_b200 import serve as S
    return S.BenchServe(args)


def workload_class(name):
    return CONFIGS.get(name) or {"batch": make_batch, "serve": make_serve}.get(name)


# ---------------------------------------------------------------------------
# harness
# ---------------------------------------------------------------------------

def reference_line(args, name, steps, warmup, R, ncores):
    """One workload on the reference's CPU path: its figures as a dict."""
    work = workload_class(name)(args)
    try:
        units, secs, sample = work.reference_steps(R, steps, warmup)
    except NotImplementedError:
        return {"unavailable": "the reference has no path for this workload"}
    val = units / secs
    return {"metric": work.metric, "value": val, "unit": work.unit,
            "steps": steps, "warmup": warmup, "ms_per_step": 1e3 * secs / steps,
            "higher_is_better": True, "dtype": work.dtype,
            "config": dict(workload=work.workload, threads=ncores, **work.config()),
            "cpu_baseline": {"value": val, "unit": work.unit, "cores": ncores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": val, "unit": work.unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_reference(args):
    """The reference's own CPU path (oracle/_ref) on this host's cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # the reference arm builds its inputs with the generators compiled into
    # the reference runner, so it loads no library of graphblas_b200
    os.environ["GRB_B200_GEN_LIB"] = os.path.join(ROOT, "oracle", "_ref", "libref_runner.so")
    from oracle import Reference, reference_available
    if not reference_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference library oracle/_ref not built"}))
        return 0
    ncores = os.cpu_count()
    R = Reference(nthreads=ncores)
    head = "tc" if args.config == "all" else args.config
    line = reference_line(args, head, args.steps, args.warmup, R, ncores)
    line.update({"impl": "reference", "n_gpus": args.gpus, "scaling": "weak",
                 "vs_baseline": None, "data": "synthetic"})
    if args.config == "all":
        # the other workloads, each a bounded sample: a few steps
        subs = {}
        for name in SUB_CONFIGS:
            k = 1 if name in ("batch", "serve") else min(args.steps, 5)
            subs[name] = reference_line(args, name, k, 1, R, ncores)
        line["configs"] = subs
    print(json.dumps(line))
    return 0


def pin_rank_gpu():
    """One GPU per rank: under torchrun (WORLD_SIZE > 1) each process sees
    only its own GPU, chosen before CUDA starts, so torch and the library
    (which carries its own CUDA runtime) agree on device 0.  Returns the CUDA
    device index to use and the GPU's index for nvidia-smi."""
    local = int(os.environ.get("LOCAL_RANK", "0"))
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    ids = [v.strip() for v in vis.split(",") if v.strip()] if vis else None
    physical = ids[local] if ids and local < len(ids) else str(local)
    if int(os.environ.get("WORLD_SIZE", "1")) <= 1:
        return local, physical
    os.environ["CUDA_VISIBLE_DEVICES"] = physical
    return 0, physical


class Harness:
    """Timing shared by every workload: warm-up, K timed steps between CUDA
    events on the library's stream with an L2 flush before each, clocks
    sampled meanwhile, max over ranks; then the same through the public API
    from pinned host buffers (e2e); then the reference on the host."""

    def __init__(self, args, gb, torch, dist, smi_index):
        self.args, self.gb, self.torch, self.dist = args, gb, torch, dist
        self.smi_index = smi_index
        self.L = gb.lib()
        self.stream = torch.cuda.Stream()
        self.L.grb_b200_set_stream(ctypes.c_void_p(self.stream.cuda_stream))
        # the stream lives as long as the process: it keeps a scratch buffer,
        # as the library's own streams do
        self.L.grb_b200_stream_keep_scratch(ctypes.c_void_p(self.stream.cuda_stream), True)
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))

    def barrier(self):
        self.torch.cuda.synchronize()
        if self.dist is not None:
            self.dist.barrier()

    def timed(self, fn, k_steps, profile_kernel=None):
        torch, stream, L_ = self.torch, self.stream, self.L
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k_steps)]
        units = 0.0
        if profile_kernel:
            # events around one in PROF_EVERY launches of the timed kernel
            # only: a timed range costs the stream several microseconds
            L_.grb_b200_profile_reset()
            L_.grb_b200_profile_select(profile_kernel.encode(), PROF_EVERY)
            L_.grb_b200_profile_enable(True)
        with torch.cuda.stream(stream):
            for k in range(k_steps):
                self.flush.fill_(k & 0xff)
                ev[k][0].record(stream)
                units += fn()
                ev[k][1].record(stream)
        torch.cuda.synchronize()
        if profile_kernel:
            L_.grb_b200_profile_enable(False)
            L_.grb_b200_profile_select(None, 1)
        return units, sum(a.elapsed_time(b) for a, b in ev)

    def measure(self, work, steps, warmup, cpu=True):
        torch, gb = self.torch, self.gb
        work.dev_setup(gb)
        with torch.cuda.stream(self.stream):
            for _ in range(warmup):
                work.step_dev()
        self.barrier()
        sampler = ClockSampler(self.smi_index)
        sampler.start()
        units, dev_ms = self.timed(work.step_dev, steps, profile_kernel=work.kernel)
        clocks = sampler.stop()
        kms, kcount = profile(self.L, work.kernel)
        self.barrier()
        t_max = allreduce_max(self.dist, dev_ms)
        units_all = allreduce_sum(self.dist, units)
        h2d, d2h = work.e2e_setup(torch)
        with torch.cuda.stream(self.stream):
            for _ in range(warmup):
                work.step_e2e()
        self.barrier()
        units2, e2e_ms = self.timed(work.step_e2e, steps)
        e2e_max = allreduce_max(self.dist, e2e_ms)
        units2_all = allreduce_sum(self.dist, units2)
        if hasattr(work, "finish"):
            work.finish(t_max / steps)
        hbm_peak, peak_kind = peaks()
        kernel_ms = kms / max(kcount, 1)
        launches_per_step = max(kcount // max(steps, 1), 1)
        if getattr(work, "kernel_ms_override", None):
            # numeric phase replayed as a CUDA graph: timed in a separate eager run
            kernel_ms, launches_per_step = work.kernel_ms_override, 1
        alg_per_launch = work.alg_bytes / launches_per_step
        achieved = alg_per_launch / (kernel_ms * 1e-3) / 1e9 if kernel_ms > 0 else None
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": (achieved / hbm_peak) if achieved else None,
                "peak_kind": peak_kind, "basis": getattr(work, "basis", None),
                "traffic": getattr(work, "traffic_per_launch", None),
                "kernel": work.kernel, "kernel_ms_per_launch": kernel_ms,
                "algorithmic_bytes_per_launch": alg_per_launch}
        if getattr(work, "merge_equiv_bytes", None):
            roof["merge_equiv_bytes"] = work.merge_equiv_bytes / launches_per_step
        line = {
            "metric": work.metric, "value": units_all / (t_max * 1e-3), "unit": work.unit,
            "ms_per_step": t_max / steps, "steps": steps, "warmup": warmup,
            "higher_is_better": True, "dtype": work.dtype,
            "config": dict(workload=work.workload,
                           parallelism="replicas" if self.world > 1 else "single",
                           l2="flushed (256 MB write) between steps", **work.config()),
            "e2e": {"value": units2_all / (e2e_max * 1e-3), "unit": work.unit,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_max / steps},
            "gpu_launches": work.launches_per_step() * steps,
            "roofline": roof, "clocks": clocks,
        }
        if self.rank == 0 and cpu:
            line["cpu_baseline"] = cpu_baseline(work)
            line["parity"] = line["cpu_baseline"].pop("parity", None)
        work.free()
        return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="all")
    ap.add_argument("--scale", type=int, default=0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.config != "all" and workload_class(args.config) is None:
        raise SystemExit("unknown --config %s" % args.config)
    if args.impl == "reference":
        return run_reference(args)

    device, smi_index = pin_rank_gpu()
    import torch
    import graphblas_b200 as gb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    gb.init()
    H = Harness(args, gb, torch, dist, smi_index)
    cpu = not args.no_cpu_baseline
    head = "tc" if args.config == "all" else args.config
    line = H.measure(workload_class(head)(args), args.steps, args.warmup, cpu)
    line.update({"n_gpus": world, "scaling": "weak", "vs_baseline": None,
                 "data": "synthetic"})
    mismatch = line.get("parity") and "MISMATCH" in line["parity"]
    if args.config == "all":
        subs = {}
        for name in SUB_CONFIGS:
            # the serving replay is seconds long: two timed replays
            k = 2 if name == "serve" else args.steps
            w = 1 if name == "serve" else args.warmup
            subs[name] = H.measure(workload_class(name)(args), k, w, cpu)
            p = subs[name].get("parity")
            mismatch = mismatch or bool(p and "MISMATCH" in p)
        line["configs"] = subs
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if mismatch:
        print("bench: a device result differs from the reference's (see parity)",
              file=sys.stderr)
    return 0


def cpu_baseline(work):
    """The reference library on this host's cores, and the parity of the
    device's result against the reference's."""
    try:
        from oracle import Reference, reference_available
        if not reference_available():
            return {"value": None, "unit": work.unit, "cores": 0, "kind": "reference",
                    "sample": "unavailable: oracle/_ref not built"}
        ncores = os.cpu_count()
        R = Reference(nthreads=ncores)
        out = work.cpu_baseline(R, ncores)
        val, sample = out[0], out[1]
        parity = out[2] if len(out) > 2 else None
        return {"value": val, "unit": work.unit, "cores": ncores, "kind": "reference",
                "sample": sample, "parity": parity}
    except Exception as e:   # the baseline is reported, never required
        return {"value": None, "unit": work.unit, "cores": 0, "kind": "reference",
                "sample": "failed: %s" % e}


def profile(L_, name):
    ms = ctypes.c_double()
    cnt = ctypes.c_int64()
    L_.grb_b200_profile(name.encode(), ctypes.byref(ms), ctypes.byref(cnt))
    return ms.value, cnt.value


def _reduce(dist, v, op):
    if dist is None:
        return v
    import torch
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def allreduce_max(dist, v):
    """The slowest rank's time (replicas: the job ends when the last ends)."""
    return _reduce(dist, v, None if dist is None else dist.ReduceOp.MAX)


def allreduce_sum(dist, v):
    """All ranks' units of work."""
    return _reduce(dist, v, None if dist is None else dist.ReduceOp.SUM)


def replica_value(dist, units, ms):
    """Whole-job throughput of N independent replicas: the units every rank
    processed over the slowest rank's time."""
    return allreduce_sum(dist, units) / (allreduce_max(dist, ms) * 1e-3)


if __name__ == "__main__":
    sys.exit(main())
