"""Build the native libraries of graphblas_b200 in-tree (no JIT cache).

    python -m graphblas_b200.build            # build what is out of date
    python -m graphblas_b200.build --force    # rebuild everything

Products (under graphblas_b200/lib/):
  libgrb_b200.so      CUDA kernels for sm_100a + the C-ABI (include/*.h)
  libgrb_b200_gen.so  seeded workload generators (plain C, OpenMP)

Every .cu file is compiled separately (in parallel) with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3``, then linked
with the static CUDA runtime.
"""

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "lib", "obj")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
CC_FLAGS = ["-O3", "-fPIC", "-std=gnu11", "-fopenmp",
            "-I" + os.path.join(ROOT, "include")]

CU_SOURCES = ["grb_runtime.cu", "grb_dot3.cu", "grb_saxpy3.cu", "grb_reduce.cu",
              "grb_ewise.cu", "grb_mxv.cu", "grb_batch.cu", "grb_serve.cu", "grb_abi.cu"]
C_SOURCES = ["grb_api.c", "grb_serialize.c", "grb_zstd.c"]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
          if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed:\n%s\n%s" % (" ".join(cmd), r.stdout))
    return r.stdout


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    jobs = []
    objs = []
    for f in CU_SOURCES:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(OBJ, f.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([nvcc] + NVCC_FLAGS + ["-c", src, "-o", obj])
    for f in C_SOURCES:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(OBJ, f.replace(".c", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append(["gcc"] + CC_FLAGS + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    so = os.path.join(LIB, "libgrb_b200.so")
    if force or jobs or _stale(so, objs):
        _run([nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", so] + objs +
             ["-Xcompiler", "-fopenmp", "-Xlinker", "-Bsymbolic"])
    gen_src = os.path.join(CSRC, "gen.c")
    gen_so = os.path.join(LIB, "libgrb_b200_gen.so")
    if force or _stale(gen_so, [gen_src]):
        _run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", gen_so,
              gen_src, "-lm"])
    return so


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    so = build(force=a.force, verbose=a.verbose)
    print(so)


if __name__ == "__main__":
    sys.exit(main())
