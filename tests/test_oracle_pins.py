"""Pin the oracle restatement (oracle/oracle.c) to the reference itself.

* Against the committed golden fixtures (tests/golden/*.npz, produced by
  SuiteSparse:GraphBLAS through its public API by tests/golden/make_golden.py):
  always runs.
* Against the live reference library (oracle/_ref) on fresh seeded inputs,
  including larger ones: runs where that library was built.

Integer / boolean / pair / min-plus results must be bit-identical; floating
PLUS_TIMES must match bit for bit as well when the reference ran its
sequential (coarse, k ascending) tasks, which is the case single-threaded.
"""

import glob
import os

import numpy as np
import pytest

from oracle import Oracle, Reference, reference_available
from graphblas_b200 import workloads as W
from tests.helpers import assert_exact, random_csr

HERE = os.path.dirname(os.path.abspath(__file__))
# blobs.npz: test_serialize.py; fullsize.npz: test_oracle_fullsize.py
GOLD = sorted(g for g in glob.glob(os.path.join(HERE, "golden", "*.npz"))
              if not g.endswith(("blobs.npz", "fullsize.npz")))


@pytest.fixture(scope="module")
def O():
    return Oracle()


@pytest.fixture(scope="module")
def R():
    if not reference_available():
        pytest.skip("reference library not built here")
    return Reference(nthreads=1)


@pytest.mark.parametrize("path", [g for g in GOLD if "rmat9" not in g],
                         ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_golden(O, path):
    d = np.load(path, allow_pickle=False)
    tc = int(d["type"])
    A = (d["Ap"], d["Ai"], d["Ax"], tc)
    B = (d["Bp"], d["Bi"], d["Bx"], tc)
    m, n = int(d["m"]), int(d["n"])
    add, mult = str(d["add"]), str(d["mult"])
    if bool(d["dot3"]):
        got = O.dot3(m, n, A, B, (d["Mp"], d["Mi"], None, 1), add, mult, tc)
    else:
        M = (d["Mp"], d["Mi"], None, 1) if bool(d["masked"]) else None
        got = O.saxpy(m, n, A, B, add, mult, tc, M=M, mask_comp=bool(d["comp"]))
    assert_exact(got, (d["Cp"], d["Ci"], d["Cx"]), os.path.basename(path))


def test_oracle_tc_bfs_golden(O):
    d = np.load(os.path.join(HERE, "golden", "rmat9_tc_bfs.npz"))
    n = int(d["n"])
    S = W.Csr(n, n, d["Sp"], d["Si"])
    L, U = W.tril_triu(S)
    assert O.tricount(n, L.p, L.i, U.p, U.i) == int(d["ntri"])
    parent, level = O.bfs(n, S.p, S.i, int(d["src"]))
    assert np.array_equal(parent, d["parent"])


def test_generators_reproduce_golden_graph():
    """The workload generator is deterministic: it rebuilds the fixture graph."""
    d = np.load(os.path.join(HERE, "golden", "rmat9_tc_bfs.npz"))
    S = W.rmat(9, 16, seed=77)
    assert np.array_equal(S.p, d["Sp"]) and np.array_equal(S.i, d["Si"])


LIVE = [("PLUS", "TIMES", "fp64"), ("PLUS", "TIMES", "fp32"),
        ("PLUS", "TIMES", "int64"), ("MIN", "PLUS", "fp32"),
        ("MIN", "PLUS", "fp64"), ("MAX", "PLUS", "fp32"),
        ("PLUS", "PAIR", "int64"), ("ANY", "SECONDI", "int64"),
        ("ANY", "FIRSTJ", "int64"), ("MIN", "SECONDI", "int64"),
        ("LOR", "LAND", "bool"), ("PLUS", "FIRST", "fp64"),
        ("MIN", "SECOND", "fp32")]


@pytest.mark.parametrize("add,mult,tname", LIVE)
@pytest.mark.parametrize("mask", ["none", "mask", "comp"])
def test_oracle_vs_reference_saxpy(O, R, add, mult, tname, mask):
    from oracle import TYPE_CODES, NP_TYPES
    tc = TYPE_CODES[tname]
    np_t = NP_TYPES[tc]
    m, k, n = 90, 70, 80
    A = random_csr(m, k, 0.1, 5, np_t, lo=0.5, hi=3.0)
    B = random_csr(k, n, 0.1, 6, np_t, lo=0.5, hi=3.0)
    M = random_csr(m, n, 0.3, 7, np.bool_)
    Mt = None if mask == "none" else (M.p, M.i, None, 1)
    comp = mask == "comp"
    got = O.saxpy(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc,
                  M=Mt, mask_comp=comp)
    # method 2 (Gustavson) runs the coarse tasks the oracle restates
    want = R.mxm(m, k, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc,
                 M=Mt, mask_comp=comp, method=2)
    assert_exact(got, want, "saxpy %s %s %s" % (add, mult, tname))


@pytest.mark.parametrize("add,mult,tname", LIVE)
def test_oracle_vs_reference_dot3(O, R, add, mult, tname):
    from oracle import TYPE_CODES, NP_TYPES
    tc = TYPE_CODES[tname]
    np_t = NP_TYPES[tc]
    m, k, n = 70, 90, 60
    A = random_csr(m, k, 0.15, 8, np_t, lo=0.5, hi=3.0)
    B = random_csr(n, k, 0.15, 9, np_t, lo=0.5, hi=3.0)
    M = random_csr(m, n, 0.3, 10, np.bool_)
    got = O.dot3(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc),
                 (M.p, M.i, None, 1), add, mult, tc)
    want = R.mxm(m, k, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc,
                 M=(M.p, M.i, None, 1), transpose_b=True, method=1)
    assert_exact(got, want, "dot3 %s %s %s" % (add, mult, tname))


def test_oracle_vs_reference_valued_mask_and_accum(O, R):
    A = random_csr(50, 40, 0.2, 1)
    B = random_csr(40, 45, 0.2, 2)
    M = random_csr(50, 45, 0.4, 3)
    M.x = (np.arange(M.nnz) % 3).astype(np.float64)
    C0 = random_csr(50, 45, 0.2, 4)
    for replace in (False, True):
        for comp in (False, True):
            T = O.saxpy(50, 45, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS",
                        "TIMES", 11)
            got = O.accum_mask(50, 45, (C0.p, C0.i, C0.x), T, 11,
                               M=(M.p, M.i, M.x, 11), mask_struct=False,
                               mask_comp=comp, replace=replace, accum="PLUS")
            want = R.mxm(50, 40, 45, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11),
                         "PLUS", "TIMES", 11, M=(M.p, M.i, M.x, 11),
                         mask_struct=False, mask_comp=comp, replace=replace,
                         accum="PLUS", C=(C0.p, C0.i, C0.x), method=2)
            assert_exact(got, want, "accum replace=%s comp=%s" % (replace, comp))


@pytest.mark.parametrize("scale", [10, 13])
def test_oracle_vs_reference_tc_bfs(O, R, scale):
    S = W.rmat(scale, 16, seed=scale + 100)
    L, U = W.tril_triu(S)
    ntri, _ = R.tricount(S.nrows, L.p, L.i, U.p, U.i)
    assert O.tricount(S.nrows, L.p, L.i, U.p, U.i) == ntri
    p1, _ = O.bfs(S.nrows, S.p, S.i, 0)
    p2, _, _ = R.bfs(S.nrows, S.p, S.i, 0)
    assert np.array_equal(p1, p2)


def test_oracle_vs_reference_er_fp64(O, R):
    """The saxpy3 configuration's shape (ER, 8/row, U[-1,1]) at n = 2048."""
    A = W.er_fixed(2048, 2048, 8, seed=1)
    B = W.er_fixed(2048, 2048, 8, seed=2)
    got = O.saxpy(2048, 2048, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS",
                  "TIMES", 11)
    want = R.mxm(2048, 2048, 2048, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11),
                 "PLUS", "TIMES", 11)
    assert_exact(got, want, "ER fp64 (auto method, 1 thread)")


def test_oracle_vs_reference_batch(O, R):
    mats = W.batch_min_plus(count=12, nmin=64, nmax=600, seed=3)
    nsz = np.array([a.nrows for a in mats], np.int64)
    poff = np.concatenate([[0], np.cumsum(nsz + 1)[:-1]]).astype(np.int64)
    ioff = np.concatenate([[0], np.cumsum([a.nnz for a in mats])[:-1]]).astype(np.int64)
    Ap = np.concatenate([a.p for a in mats])
    Ai = np.concatenate([a.i for a in mats])
    Ax = np.concatenate([a.x for a in mats])
    nnz_ref, _ = R.batch_square(nsz, poff, ioff, Ap, Ai, Ax)
    for k, a in enumerate(mats):
        C = O.saxpy(a.nrows, a.ncols, (a.p, a.i, a.x, 10), (a.p, a.i, a.x, 10),
                    "MIN", "PLUS", 10)
        assert C[0][-1] == nnz_ref[k]


def test_reference_serve_replay_matches_oracle(O, R):
    """The reference arm of the serving workload: the request trace replayed
    through a thread pool on the reference library gives, request by request,
    the triangle counts and result sizes the oracle computes."""
    from graphblas_b200.serve import make_graphs, make_trace, K_TRICOUNT, K_SSSP
    graphs = make_graphs(seed=3, tc_scales=range(6, 9), n_sssp=1, n_mxm=2, mxm_nmax=2000)
    trace = make_trace(graphs, nreq=40, rate=4000.0, seed=5)
    status, count, checksum, latency, makespan = R.serve(graphs, trace, 4, 1)
    assert (status == 0).all()
    assert makespan > 0 and (latency > 0).all()
    for k in range(40):
        kind = int(trace["kind"][k])
        g = graphs[int(trace["graph"][k])][1]
        if kind == K_TRICOUNT:
            L, U = W.tril_triu(g)
            assert count[k] == O.tricount(g.nrows, L.p, L.i, U.p, U.i)
        elif kind == K_SSSP:
            lo, hi = trace["fp"][k], trace["fp"][k + 1]
            u = (np.array([0, hi - lo], np.int64), trace["fi"][lo:hi], trace["fx"][lo:hi], 10)
            want = O.saxpy(1, g.ncols, u, (g.p, g.i, g.x, 10), "MIN", "PLUS", 10)
            assert count[k] == len(want[1])
        else:
            want = O.saxpy(g.nrows, g.ncols, (g.p, g.i, g.x, 11), (g.p, g.i, g.x, 11),
                           "PLUS", "TIMES", 11)
            assert count[k] == len(want[1])
