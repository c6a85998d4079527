"""Parity at the stated sizes of the benchmark configurations.

Each test runs one configuration at its full size on the GPU, through the
same public entry points the benchmark times, and compares the result with
the oracle (oracle/oracle.c) bit for bit, and with the reference's own result
at that size (tests/golden/fullsize.npz, made by tests/golden/make_fullsize.py
from SuiteSparse:GraphBLAS built from its sources) through csr_digest:

* cfg1  C = A*B, plus_times fp64, Erdos-Renyi 16384 x 16384, 8 per row: the
        whole of C (pattern and values; the device folds every entry's terms
        in the reference's ascending-k order, so the values are bit-identical,
        inside the reference's own 64*eps 1-norm rule a fortiori);
* cfg2  triangle counting, R-MAT scale 20: C<L> = L*U' entry by entry against
        the oracle's dot3, and the count against the reference's;
* cfg3  BFS parents, R-MAT scale 22, from the first vertex with an edge:
        every parent (the max-parent rule) and the level count;
* cfg4  all 4096 min_plus fp32 instances of the batch, each bit-identical.
"""

import os

import numpy as np
import pytest

from graphblas_b200 import workloads as W
from oracle import csr_digest
from tests.helpers import assert_exact, assert_roundoff

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "fullsize.npz"))
SEED = 1        # the benchmark's default seed


@pytest.fixture(scope="module")
def api(gpu):
    from graphblas_b200.grb import API
    return API()


def test_cfg1_er16384_plus_times_fp64(api, oracle):
    n = 16384
    A = W.er_fixed(n, n, 8, seed=SEED + 1)
    B = W.er_fixed(n, n, 8, seed=SEED + 2)
    Ag, Bg = api.matrix_from_csr(A), api.matrix_from_csr(B)
    Cg = api.matrix_new(11, n, n)
    api.mxm(Cg, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", Ag, Bg)
    got = api.matrix_to_csr(Cg, 11, n)
    want = oracle.saxpy(n, n, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS", "TIMES", 11)
    assert_roundoff(got, want, n, "ER 16384 plus_times fp64")
    assert_exact(got, want, "ER 16384 plus_times fp64")
    assert len(got[1]) == int(GOLD["er16384_nnz"])
    assert csr_digest(*got) == int(GOLD["er16384_digest"]), "differs from the reference"
    for X in (Ag, Bg, Cg):
        api.free(X)


def test_cfg2_tricount_rmat20(api, oracle):
    S = W.rmat(20, 16, seed=SEED)
    Lc, Uc = W.tril_triu(S)
    assert Lc.nnz == int(GOLD["tc20_nnz_L"])
    L = api.matrix_from_csr(Lc, 1)
    U = api.matrix_from_csr(Uc, 1)
    C = api.matrix_new(8, S.nrows, S.ncols)
    api.mxm(C, L, None, "GxB_PLUS_PAIR_INT64", L, U, "GrB_DESC_ST1")
    ntri = api.reduce(C, "GrB_PLUS_MONOID_INT64", 8)
    assert ntri == int(GOLD["tc20_triangles"])
    got = api.matrix_to_csr(C, 8, S.nrows)
    want = oracle.dot3(S.nrows, S.ncols, (Lc.p, Lc.i, None, 1), (Uc.p, Uc.i, None, 1),
                       (Lc.p, Lc.i, None, 1), "PLUS", "PAIR", 8)
    assert_exact(got, want, "C<L>=L*U' at scale 20")
    for X in (L, U, C):
        api.free(X)


def test_cfg3_bfs_rmat22_parents(api, oracle):
    S = W.rmat(22, 16, seed=SEED)
    n = S.nrows
    src = int(np.argmax(np.diff(S.p) > 0))
    assert src == int(GOLD["bfs22_source"])
    A = api.matrix_from_csr(S, 1)
    q = api.vector_from([src], [src], 8, n)
    p = api.vector_from([src], [src], 8, n)
    levels = 0
    while True:
        levels += 1
        api.vxm(q, p, None, "GxB_ANY_SECONDI_INT64", q, A, "GrB_DESC_RSC")
        if api.vnvals(q) == 0:
            break
        api.assign_all(p, q, None, q, n, "GrB_DESC_S")
    idx, par = api.vector_to(p, 8)
    parent = np.full(n, -1, np.int64)
    parent[idx] = par
    want, _ = oracle.bfs(n, S.p, S.i, src)
    assert np.array_equal(parent, want)
    assert levels == int(GOLD["bfs22_levels"])
    assert int(np.sum(parent >= 0)) == int(GOLD["bfs22_reached"])
    dig = csr_digest(np.array([0, n], np.int64), np.arange(n, dtype=np.int64), parent)
    assert dig == int(GOLD["bfs22_parent_digest"]), "differs from the reference"
    for v in (q, p):
        api.vfree(v)
    api.free(A)


def test_cfg4_batch4096_min_plus(gpu, oracle, tmp_path, monkeypatch):
    from graphblas_b200.batch import Batch
    monkeypatch.setenv("GRB_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    mats = W.batch_min_plus(count=4096, seed=11 + SEED)
    B = Batch(mats, gpu.semiring("MIN", "PLUS", "fp32"))
    B.tune(use_cache=False)
    B.run(use_graph=True)
    got = B.result()
    B.free()
    ref = GOLD["batch4096_digests"]
    for k, a in enumerate(mats):
        assert csr_digest(*got[k]) == int(ref[k]), "instance %d differs from the reference" % k
    # the oracle on every instance as well
    for k, a in enumerate(mats):
        want = oracle.saxpy(a.nrows, a.ncols, (a.p, a.i, a.x, 10), (a.p, a.i, a.x, 10),
                            "MIN", "PLUS", 10)
        assert_exact(got[k], want, "instance %d" % k)
