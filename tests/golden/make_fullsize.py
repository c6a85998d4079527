"""Regenerate tests/golden/fullsize.npz: the reference's own results at the
full sizes of the five benchmark configurations, as digests.

    python tests/golden/make_fullsize.py

Runs SuiteSparse:GraphBLAS itself (oracle/_ref, built from the reference's
own sources by oracle/ref.mk) through its public API on the seeded inputs the
benchmark uses, and stores what the full-size parity tests compare against:

* er16384: C = A*B, plus_times fp64, A and B 16384x16384 Erdos-Renyi with 8
  columns per row (seeds 2 and 3): csr_digest of C (1 thread: the ascending-k
  summation order of a coarse task);
* tc20: the triangle count of R-MAT scale 20, edge factor 16 (seed 1),
  C<L> = L*U' plus_pair int64 then a sum;
* bfs22: BFS parents on R-MAT scale 22, edge factor 16 (seed 1) from the
  first vertex with an edge (1 thread: the max-parent rule of the ANY
  monoid's last-wins update), as a digest, the number of levels and the
  number of reached vertices;
* batch4096: csr_digest of every C_i = A_i*A_i of the 4096 min_plus fp32
  instances (seed 12), one GrB_mxm each.

The digests are oracle.csr_digest (the runner computes the same in C).
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import Reference, csr_digest   # noqa: E402
from graphblas_b200 import workloads as W  # noqa: E402

BENCH_SEED = 1      # bench.py's default --seed


def vector_digest(parent):
    """Digest of a dense int64 vector (as a 1-row CSR over every position)."""
    n = len(parent)
    return csr_digest(np.array([0, n], np.int64), np.arange(n, dtype=np.int64),
                      np.asarray(parent, np.int64))


def main():
    R = Reference(nthreads=os.cpu_count())
    out = {}
    t0 = time.time()
    # cfg1: ER saxpy3 (bench.py Saxpy: seeds seed+1, seed+2)
    n = 16384
    A = W.er_fixed(n, n, 8, seed=BENCH_SEED + 1)
    B = W.er_fixed(n, n, 8, seed=BENCH_SEED + 2)
    R.set_nthreads(1)
    p, i, x = R.mxm(n, n, n, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS", "TIMES", 11)
    out["er16384_digest"] = np.uint64(csr_digest(p, i, x))
    out["er16384_nnz"] = np.int64(len(i))
    print("er16384", len(i), time.time() - t0, flush=True)
    # cfg2: triangle count
    R.set_nthreads(os.cpu_count())
    S = W.rmat(20, 16, seed=BENCH_SEED)
    L, U = W.tril_triu(S)
    ntri, _ = R.tricount(S.nrows, L.p, L.i, U.p, U.i)
    out["tc20_triangles"] = np.int64(ntri)
    out["tc20_nnz_L"] = np.int64(L.nnz)
    print("tc20", ntri, time.time() - t0, flush=True)
    del S, L, U
    # cfg3: BFS parents, single-threaded reference
    R.set_nthreads(1)
    S = W.rmat(22, 16, seed=BENCH_SEED)
    src = int(np.argmax(np.diff(S.p) > 0))
    parent, _, nlev = R.bfs(S.nrows, S.p, S.i, src)
    out["bfs22_source"] = np.int64(src)
    out["bfs22_parent_digest"] = np.uint64(vector_digest(parent))
    out["bfs22_levels"] = np.int64(nlev)
    out["bfs22_reached"] = np.int64(int(np.sum(parent >= 0)))
    print("bfs22", nlev, int(np.sum(parent >= 0)), time.time() - t0, flush=True)
    del S, parent
    # cfg4: the batch (graphblas_b200/batch.py BenchBatch: seed 11 + seed)
    from graphblas_b200.batch import concat
    R.set_nthreads(os.cpu_count())
    mats = W.batch_min_plus(count=4096, seed=11 + BENCH_SEED)
    rows, cols, P, J, X = concat(mats, np.float32)
    poff = np.concatenate([[0], np.cumsum(rows + 1)[:-1]]).astype(np.int64)
    ioff = P[poff]
    nnz, _, dig = R.batch_square(rows, poff, ioff, P, J, X, digests=True)
    out["batch4096_digests"] = dig
    out["batch4096_nnz"] = nnz
    print("batch4096", int(nnz.sum()), time.time() - t0, flush=True)
    np.savez_compressed(os.path.join(HERE, "fullsize.npz"), **out)


if __name__ == "__main__":
    main()
