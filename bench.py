#!/usr/bin/env python
"""Benchmark of the B200 semiring SpGEMM path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config tc|saxpy|bfs|batch|serve]

Default workload (the headline): masked dot3 triangle counting,
C<L> = L*U' with plus_pair int64 followed by a sum reduction, on a
symmetrised R-MAT graph of scale 20, edge factor 16, (a,b,c,d) =
(0.57,0.19,0.19,0.05), self-loops and duplicates removed (seeded synthetic
input of the graph500 shape; no dataset).  One step = one GrB_mxm + reduce
over the whole graph.  Metric: triangles/s.

* value: device time with L and U resident in HBM, CUDA events on the
  launching stream, L2 flushed (256 MB write) between steps, max over ranks.
* e2e: the same step through the public C-ABI from pinned host buffers
  (upload L and U, multiply, reduce, read the count back), timed the same way.
* roofline: the dot3 kernel's algorithmic bytes per launch
  (4*(sum_i nnz(L(i,:))^2 + sum_j nnz(U(j,:))^2) merge reads + 16*nnz(L)
  mask read and C write) over its event-timed duration, against the measured
  HBM copy bandwidth.
* cpu_baseline: the reference library (oracle/_ref, SuiteSparse:GraphBLAS
  built from its own sources) on this host's cores, same graph.

--impl reference times that reference CPU path alone and prints its line.
Multi-GPU (torchrun): every rank runs an independent replica (the path has no
exchange step); value = all ranks' triangles / max step time.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
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
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def tc_inputs(scale, ef, seed):
    S = W.rmat(scale, ef, seed=seed)
    L, U = W.tril_triu(S)
    dL = np.diff(L.p).astype(np.float64)
    dU = np.diff(U.p).astype(np.float64)
    alg_bytes = 4.0 * (np.sum(dL * dL) + np.sum(dU * dU)) + 16.0 * L.nnz
    return S, L, U, alg_bytes


def run_reference(args):
    """The reference's own CPU path (oracle/_ref) on this host's cores."""
    from oracle import Reference, reference_available
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not reference_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference library oracle/_ref not built"}))
        return 0
    ncores = os.cpu_count()
    R = Reference(nthreads=ncores)
    S, L, U, _ = tc_inputs(args.scale, 16, args.seed)
    for _ in range(args.warmup):
        R.tricount(S.nrows, L.p, L.i, U.p, U.i, reps=1)
    ntri, times = R.tricount(S.nrows, L.p, L.i, U.p, U.i, reps=args.steps)
    t = float(np.sum(times))
    val = ntri * args.steps / t
    line = {"metric": "triangles/s", "value": val, "unit": "triangles/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64", "data": "synthetic",
            "config": {"workload": "tricount_rmat%d_ef16_dot3_plus_pair" % args.scale,
                       "nnz_L": int(L.nnz), "triangles": int(ntri),
                       "threads": ncores},
            "cpu_baseline": {"value": val, "unit": "triangles/s", "cores": ncores,
                             "kind": "reference",
                             "sample": "whole graph per step (GrB_mxm + GrB_reduce)"},
            "e2e": {"value": val, "unit": "triangles/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="tc")
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import graphblas_b200 as gb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    gb.init()
    L_ = gb.lib()
    stream = torch.cuda.Stream()
    L_.grb_b200_set_stream(ctypes_ptr(stream.cuda_stream))

    S, L, U, alg_bytes = tc_inputs(args.scale, 16, args.seed + 0)
    sr = gb.semiring("PLUS", "PAIR", "int64")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # ---- device-resident step ----
    dL = gb.DMatrix.upload(L, "bool")
    dU = gb.DMatrix.upload(U, "bool")

    def step_dev():
        C = gb.dot3(dL, dL, dU, sr)
        n = gb.reduce(C, "PLUS", np.int64)
        C.free()
        return int(n)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            ntri = step_dev()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    L_.grb_b200_profile_reset()
    L_.grb_b200_profile_enable(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            ev[k][0].record(stream)
            ntri = step_dev()
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    L_.grb_b200_profile_enable(False)
    clocks = sampler.stop()
    dev_ms = sum(a.elapsed_time(b) for a, b in ev)
    kms, kcount = profile(L_, "dot3")
    barrier()
    t_max = allreduce_max(dist, dev_ms)
    ntri_all = allreduce_sum(dist, float(ntri) * args.steps)

    # ---- end-to-end step through the C-ABI from pinned host buffers ----
    pin = {}
    for name, arr in (("Lp", L.p), ("Li", L.i), ("Up", U.p), ("Ui", U.i)):
        t = torch.from_numpy(arr).pin_memory()
        pin[name] = t
    h2d = sum(int(t.numel() * t.element_size()) for t in pin.values())

    def step_e2e():
        hL = ctypes_void()
        hU = ctypes_void()
        gb.check(L_.grb_b200_dmatrix_upload(byref(hL), L.nrows, L.ncols,
                                            pin["Lp"].data_ptr(), pin["Li"].data_ptr(),
                                            None, 1, True))
        gb.check(L_.grb_b200_dmatrix_upload(byref(hU), U.nrows, U.ncols,
                                            pin["Up"].data_ptr(), pin["Ui"].data_ptr(),
                                            None, 1, True))
        dl, du = gb.DMatrix(hL.value), gb.DMatrix(hU.value)
        C = gb.dot3(dl, dl, du, sr)
        n = gb.reduce(C, "PLUS", np.int64)
        for d in (C, dl, du):
            d.free()
        return int(n)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step_e2e()
    barrier()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            ev2[k][0].record(stream)
            n2 = step_e2e()
            ev2[k][1].record(stream)
    torch.cuda.synchronize()
    assert n2 == ntri
    e2e_ms = allreduce_max(dist, sum(a.elapsed_time(b) for a, b in ev2))

    hbm_peak, peak_kind = peaks()
    kernel_ms = kms / max(kcount, 1)
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(S, L, U, ntri)
        val = ntri_all / (t_max * 1e-3)
        line = {
            "metric": "triangles/s", "value": val, "unit": "triangles/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": {"workload": "tricount_rmat%d_ef16_dot3_plus_pair" % args.scale,
                       "n": int(S.nrows), "nnz_L": int(L.nnz), "triangles": int(ntri),
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "flushed (256 MB write) between steps",
                       "edges_per_s": int(L.nnz) * args.steps * world / (t_max * 1e-3)},
            "e2e": {"value": ntri_all / (e2e_ms * 1e-3), "unit": "triangles/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8,
                    "ms_per_step": e2e_ms / args.steps},
            "gpu_launches": 4 * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                         "unit": "GB/s", "frac": achieved / hbm_peak,
                         "peak_kind": peak_kind, "traffic": None,
                         "kernel": "k_dot3", "kernel_ms": kernel_ms,
                         "algorithmic_bytes": alg_bytes},
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    for d in (dL, dU):
        d.free()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baseline(S, L, U, ntri_gpu):
    """The reference library on this host's cores, one whole-graph run
    (GrB_mxm + GrB_reduce), checked against the GPU count."""
    try:
        from oracle import Reference, reference_available
        if not reference_available():
            return {"value": None, "unit": "triangles/s", "cores": 0,
                    "kind": "reference", "sample": "unavailable: oracle/_ref not built"}
        ncores = os.cpu_count()
        R = Reference(nthreads=ncores)
        ntri, times = R.tricount(S.nrows, L.p, L.i, U.p, U.i, reps=1)
        assert ntri == ntri_gpu, "CPU and GPU triangle counts differ"
        return {"value": ntri / float(times[0]), "unit": "triangles/s",
                "cores": ncores, "kind": "reference",
                "sample": "whole graph, one GrB_mxm + GrB_reduce (%.2f s)" % times[0]}
    except Exception as e:   # the baseline is reported, never required
        return {"value": None, "unit": "triangles/s", "cores": 0,
                "kind": "reference", "sample": "failed: %s" % e}


def profile(L_, name):
    import ctypes
    ms = ctypes.c_double()
    cnt = ctypes.c_int64()
    L_.grb_b200_profile(name.encode(), ctypes.byref(ms), ctypes.byref(cnt))
    return ms.value, cnt.value


def allreduce_max(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def ctypes_ptr(v):
    import ctypes
    return ctypes.c_void_p(v)


def ctypes_void():
    import ctypes
    return ctypes.c_void_p()


def byref(x):
    import ctypes
    return ctypes.byref(x)


if __name__ == "__main__":
    sys.exit(main())
