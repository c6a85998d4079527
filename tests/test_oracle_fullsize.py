"""The oracle (oracle/oracle.c) pinned to the reference at the full sizes of
the benchmark configurations: its results on the benchmark's seeded inputs
have the digests the reference's own results have (tests/golden/fullsize.npz,
made by tests/golden/make_fullsize.py from SuiteSparse:GraphBLAS).  These pins
make the full-size GPU parity tests (tests/test_gpu_fullsize.py), which
compare the device with the oracle, comparisons with the reference."""

import os

import numpy as np

from graphblas_b200 import workloads as W
from oracle import csr_digest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "fullsize.npz"))
SEED = 1


def test_oracle_er16384_matches_reference(oracle):
    n = 16384
    A = W.er_fixed(n, n, 8, seed=SEED + 1)
    B = W.er_fixed(n, n, 8, seed=SEED + 2)
    C = oracle.saxpy(n, n, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS", "TIMES", 11)
    assert csr_digest(*C) == int(GOLD["er16384_digest"])


def test_oracle_tricount_rmat20_matches_reference(oracle):
    S = W.rmat(20, 16, seed=SEED)
    L, U = W.tril_triu(S)
    assert L.nnz == int(GOLD["tc20_nnz_L"])
    assert oracle.tricount(S.nrows, L.p, L.i, U.p, U.i) == int(GOLD["tc20_triangles"])


def test_oracle_bfs_rmat22_matches_reference(oracle):
    S = W.rmat(22, 16, seed=SEED)
    n = S.nrows
    src = int(np.argmax(np.diff(S.p) > 0))
    assert src == int(GOLD["bfs22_source"])
    parent, level = oracle.bfs(n, S.p, S.i, src)
    dig = csr_digest(np.array([0, n], np.int64), np.arange(n, dtype=np.int64), parent)
    assert dig == int(GOLD["bfs22_parent_digest"])
    assert int(np.sum(parent >= 0)) == int(GOLD["bfs22_reached"])


def test_oracle_batch4096_matches_reference(oracle):
    mats = W.batch_min_plus(count=4096, seed=11 + SEED)
    ref = GOLD["batch4096_digests"]
    for k, a in enumerate(mats):
        C = oracle.saxpy(a.nrows, a.ncols, (a.p, a.i, a.x, 10), (a.p, a.i, a.x, 10),
                         "MIN", "PLUS", 10)
        assert csr_digest(*C) == int(ref[k]), "instance %d" % k
