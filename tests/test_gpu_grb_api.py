"""The GraphBLAS C API of the path (include/GraphBLAS_b200.h) end to end on
the GPU, written the way the reference's own demos and tests call it:
triangle counting (LAGraph's C<L> = L*U' plus_pair + reduce), BFS parents
(vxm any_secondi with a complemented structural mask and replace, then
assign), mxm with accumulators, masks, replace and transposes, mxv, and the
error codes of the API.  Checked against the oracle (oracle/oracle.c).
"""

import numpy as np
import pytest

from graphblas_b200 import workloads as W
from tests.helpers import assert_exact, random_csr, transpose_csr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(gpu):
    from graphblas_b200.grb import API
    return API()


def test_tricount_through_grb_mxm(api, oracle):
    S = W.rmat(13, 16, seed=4)
    Lc, Uc = W.tril_triu(S)
    L = api.matrix_from_csr(Lc, 1)
    U = api.matrix_from_csr(Uc, 1)
    C = api.matrix_new(8, S.nrows, S.ncols)
    api.mxm(C, L, None, "GxB_PLUS_PAIR_INT64", L, U, "GrB_DESC_ST1")
    ntri = api.reduce(C, "GrB_PLUS_MONOID_INT64", 8)
    assert ntri == oracle.tricount(S.nrows, Lc.p, Lc.i, Uc.p, Uc.i)
    want = oracle.dot3(S.nrows, S.ncols, (Lc.p, Lc.i, None, 1), (Uc.p, Uc.i, None, 1),
                       (Lc.p, Lc.i, None, 1), "PLUS", "PAIR", 8)
    assert api.nvals(C) == len(want[1])          # zombies are not counted
    got = api.matrix_to_csr(C, 8, S.nrows)
    assert_exact(got, want, "C<L>=L*U'")
    for A in (L, U, C):
        api.free(A)


def test_bfs_parents_through_grb_vxm(api, oracle):
    S = W.rmat(14, 16, seed=8)
    n = S.nrows
    A = api.matrix_from_csr(S, 1)
    src = 3
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
    for v in (q, p):
        api.vfree(v)
    api.free(A)


# (replace, complement, structural) of each predefined descriptor
DESC_FLAGS = {None: (False, False, False), "GrB_DESC_R": (True, False, False),
              "GrB_DESC_S": (False, False, True), "GrB_DESC_RS": (True, False, True),
              "GrB_DESC_SC": (False, True, True), "GrB_DESC_RSC": (True, True, True),
              "GrB_DESC_C": (False, True, False), "GrB_DESC_RC": (True, True, False)}


@pytest.mark.parametrize("accum", [None, "GrB_PLUS_FP64", "GrB_MIN_FP64",
                                   "GrB_SECOND_FP64"])
@pytest.mark.parametrize("desc", [None, "GrB_DESC_R", "GrB_DESC_S", "GrB_DESC_RS",
                                  "GrB_DESC_SC", "GrB_DESC_RSC", "GrB_DESC_C",
                                  "GrB_DESC_RC"])
def test_mxm_accum_mask_replace(api, oracle, accum, desc):
    m, k, n = 70, 60, 80
    Ac = random_csr(m, k, 0.1, 1)
    Bc = random_csr(k, n, 0.1, 2)
    Mc = random_csr(m, n, 0.3, 3)
    Mc.x = (np.arange(Mc.nnz) % 3).astype(np.float64)      # a third are false
    Cc = random_csr(m, n, 0.2, 4)
    A, B = api.matrix_from_csr(Ac), api.matrix_from_csr(Bc)
    use_mask = desc is not None and desc != "GrB_DESC_R"
    M = api.matrix_from_csr(Mc) if use_mask else None
    C = api.matrix_from_csr(Cc)
    api.mxm(C, M, accum, "GrB_PLUS_TIMES_SEMIRING_FP64", A, B, desc)
    got = api.matrix_to_csr(C, 11, m)
    T = oracle.saxpy(m, n, (Ac.p, Ac.i, Ac.x, 11), (Bc.p, Bc.i, Bc.x, 11), "PLUS",
                     "TIMES", 11)
    replace, comp, strct = DESC_FLAGS[desc]
    acc = {None: None, "GrB_PLUS_FP64": "PLUS", "GrB_MIN_FP64": "MIN",
           "GrB_SECOND_FP64": "SECOND"}[accum]
    want = oracle.accum_mask(m, n, (Cc.p, Cc.i, Cc.x), T, 11,
                             M=(Mc.p, Mc.i, Mc.x, 11) if use_mask else None,
                             mask_struct=strct, mask_comp=comp, replace=replace,
                             accum=acc)
    assert_exact(got, want, "accum=%s desc=%s" % (accum, desc))
    for X in (A, B, M, C):
        if X is not None:
            api.free(X)


@pytest.mark.parametrize("desc", ["GrB_DESC_T0", "GrB_DESC_T1", "GrB_DESC_T0T1"])
def test_mxm_transposes(api, oracle, desc):
    m, k, n = 50, 65, 45
    Ac = random_csr(m, k, 0.1, 5)
    Bc = random_csr(k, n, 0.1, 6)
    At, Bt = transpose_csr(Ac), transpose_csr(Bc)
    A = api.matrix_from_csr(At if "T0" in desc else Ac)
    B = api.matrix_from_csr(Bt if "T1" in desc else Bc)
    C = api.matrix_new(11, m, n)
    api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, B, desc)
    got = api.matrix_to_csr(C, 11, m)
    want = oracle.saxpy(m, n, (Ac.p, Ac.i, Ac.x, 11), (Bc.p, Bc.i, Bc.x, 11), "PLUS",
                        "TIMES", 11)
    assert_exact(got, want, desc)
    for X in (A, B, C):
        api.free(X)


def test_mxv_and_vxm_transposed(api, oracle):
    m, n = 90, 70
    Ac = random_csr(m, n, 0.1, 7)
    rng = np.random.default_rng(8)
    ui = np.sort(rng.choice(n, 30, replace=False)).astype(np.int64)
    ux = rng.random(30)
    A = api.matrix_from_csr(Ac)
    u = api.vector_from(ui, ux, 11, n)
    w = api.vector_new(11, m)
    api.mxv(w, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, u, None)
    wi, wx = api.vector_to(w, 11)
    # oracle: dot of each row of A with u, ascending k (rows of M = all rows)
    U1 = (np.array([0, 30], np.int64), ui, ux, 11)
    Mall = (np.arange(m + 1, dtype=np.int64), np.zeros(m, np.int64), None, 1)
    want = oracle.dot3(m, 1, (Ac.p, Ac.i, Ac.x, 11), U1, Mall, "PLUS", "TIMES", 11)
    rows = np.repeat(np.arange(m), np.diff(want[0]))
    assert np.array_equal(wi, rows)
    assert np.array_equal(wx, want[2])
    # w' = u'*A' equals A*u
    w2 = api.vector_new(11, m)
    api.vxm(w2, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", u, A, "GrB_DESC_T1")
    wi2, wx2 = api.vector_to(w2, 11)
    assert np.array_equal(wi2, wi) and np.array_equal(wx2, wx)
    for v in (u, w, w2):
        api.vfree(v)
    api.free(A)


def test_api_error_codes(api):
    from graphblas_b200.grb import GrBError
    A = api.matrix_from_csr(random_csr(10, 12, 0.3, 1))
    B = api.matrix_from_csr(random_csr(10, 12, 0.3, 2))
    C = api.matrix_new(11, 10, 12)
    with pytest.raises(GrBError) as e:                 # 10x12 * 10x12
        api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, B, None)
    assert e.value.info == -6                          # GrB_DIMENSION_MISMATCH
    Ci = api.matrix_new(8, 10, 10)
    with pytest.raises(GrBError) as e:
        api.mxm(Ci, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, B, "GrB_DESC_T1")
    assert e.value.info == -5                          # GrB_DOMAIN_MISMATCH
    with pytest.raises(GrBError) as e:
        api.call("GrB_mxm", C, None, None, None, A, B, None)
    assert e.value.info == -2                          # GrB_NULL_POINTER
    for X in (A, B, C, Ci):
        api.free(X)


def test_api_out_of_memory_injection(api, gpu):
    """Host-side fault injection (the reference's malloc_debug idea): the next
    device allocation fails and the call returns GrB_OUT_OF_MEMORY cleanly;
    the following call succeeds."""
    from graphblas_b200.grb import GrBError
    Ac = random_csr(40, 40, 0.2, 9)
    A = api.matrix_from_csr(Ac)
    C = api.matrix_new(11, 40, 40)
    api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, A, None)   # warm
    gpu.lib().grb_b200_debug_fail_alloc(1)
    with pytest.raises(GrBError) as e:
        api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, A, None)
    assert e.value.info == -102
    gpu.lib().grb_b200_debug_fail_alloc(0)
    api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, A, None)
    assert api.nvals(C) > 0
    api.free(A)
    api.free(C)


def _addr(a):
    return a.ctypes.data


def test_import_export_round_trip_and_product(api, oracle):
    """GrB_Matrix_import copies the caller's CSR arrays straight to HBM (checked
    on the device), GrB_Matrix_export copies a result straight back."""
    Ac = random_csr(300, 280, 0.05, 11)
    Bc = random_csr(280, 260, 0.05, 12)
    A = api.matrix_import(11, 300, 280, _addr(Ac.p), _addr(Ac.i), _addr(Ac.x), Ac.nnz)
    B = api.matrix_import(11, 280, 260, _addr(Bc.p), _addr(Bc.i), _addr(Bc.x), Bc.nnz)
    assert api.export_size(A) == (301, Ac.nnz)
    p = np.zeros(301, np.int64)
    i = np.zeros(Ac.nnz, np.int64)
    x = np.zeros(Ac.nnz)
    assert api.matrix_export(A, 11, _addr(p), _addr(i), _addr(x), 301, Ac.nnz) == Ac.nnz
    assert_exact((p, i, x), (Ac.p, Ac.i, Ac.x), "import/export round trip")
    C = api.matrix_new(11, 300, 260)
    api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, B)
    plen, nv = api.export_size(C)
    cp = np.zeros(plen, np.int64)
    ci = np.zeros(nv, np.int64)
    cx = np.zeros(nv)
    api.matrix_export(C, 11, _addr(cp), _addr(ci), _addr(cx), plen, nv)
    want = oracle.saxpy(300, 260, (Ac.p, Ac.i, Ac.x, 11), (Bc.p, Bc.i, Bc.x, 11),
                        "PLUS", "TIMES", 11)
    assert_exact((cp, ci, cx), want, "mxm of imported matrices")
    for X in (A, B, C):
        api.free(X)


def test_import_sorts_jumbled_rows_and_rejects_bad_arrays(api):
    from graphblas_b200.grb import GrBError
    rng = np.random.default_rng(5)
    Ac = random_csr(200, 150, 0.1, 13)
    jp, ji, jx = Ac.p.copy(), Ac.i.copy(), Ac.x.copy()
    for r in range(200):                      # shuffle every row
        lo, hi = jp[r], jp[r + 1]
        perm = lo + rng.permutation(hi - lo)
        ji[lo:hi], jx[lo:hi] = ji[perm], jx[perm]
    A = api.matrix_import(11, 200, 150, _addr(jp), _addr(ji), _addr(jx), Ac.nnz)
    p = np.zeros(201, np.int64)
    i = np.zeros(Ac.nnz, np.int64)
    x = np.zeros(Ac.nnz)
    api.matrix_export(A, 11, _addr(p), _addr(i), _addr(x), 201, Ac.nnz)
    assert_exact((p, i, x), (Ac.p, Ac.i, Ac.x), "jumbled rows come back sorted")
    # export into arrays that are too small
    with pytest.raises(GrBError) as e:
        api.matrix_export(A, 11, _addr(p), _addr(i), _addr(x), 201, Ac.nnz - 1)
    assert e.value.info == -103                   # GrB_INSUFFICIENT_SPACE
    api.free(A)

    def bad(p_, i_, x_, what):
        with pytest.raises(GrBError) as e:
            api.matrix_import(11, 200, 150, _addr(p_), _addr(i_), _addr(x_), len(i_))
        assert e.value.info == -104, what         # GrB_INVALID_OBJECT
    i2 = Ac.i.copy()
    i2[7] = 150                                   # column out of range
    bad(Ac.p, i2, Ac.x, "index out of range")
    p2 = Ac.p.copy()
    p2[50] = p2[51] + 1                           # offsets decrease
    bad(p2, Ac.i, Ac.x, "decreasing offsets")
    r = int(np.argmax(np.diff(Ac.p) >= 2))        # a row with two entries
    i3 = Ac.i.copy()
    i3[Ac.p[r] + 1] = i3[Ac.p[r]]                 # duplicate index in a row
    bad(Ac.p, i3, Ac.x, "duplicate")
    import ctypes
    h = ctypes.c_void_p()
    with pytest.raises(GrBError) as e:            # only GrB_CSR_FORMAT is built
        api.call("GrB_Matrix_import_FP64", ctypes.byref(h), api.obj("GrB_FP64"), 200, 150,
                 _addr(Ac.p), _addr(Ac.i), _addr(Ac.x), 201, Ac.nnz, Ac.nnz, 1)
    assert e.value.info == -8                     # GrB_NOT_IMPLEMENTED
    with pytest.raises(GrBError) as e:            # Ap shorter than nrows+1
        api.call("GrB_Matrix_import_FP64", ctypes.byref(h), api.obj("GrB_FP64"), 200, 150,
                 _addr(Ac.p), _addr(Ac.i), _addr(Ac.x), 200, Ac.nnz, Ac.nnz, 0)
    assert e.value.info == -3                     # GrB_INVALID_VALUE


def test_vector_extract_from_device(api):
    """GrB_Vector_extractTuples of a vector computed on the device copies its
    indices and values straight from HBM."""
    S = W.rmat(10, 8, seed=2)
    A = api.matrix_from_csr(S, 1)
    n = S.nrows
    v0 = int(np.argmax(np.diff(S.p)))
    q = api.vector_from([v0], [v0], 8, n)
    w = api.vector_new(8, n)
    api.vxm(w, None, None, "GxB_ANY_SECONDI_INT64", q, A, None)
    nv = api.vnvals(w)
    i = np.zeros(nv, np.int64)
    x = np.zeros(nv, np.int64)
    assert api.vector_extract(w, 8, _addr(i), _addr(x), nv) == nv
    lo, hi = S.p[v0], S.p[v0 + 1]
    assert np.array_equal(i, S.i[lo:hi])
    assert np.array_equal(x, np.full(hi - lo, v0))  # any_secondi: row index of q's entry
    for v in (q, w):
        api.vfree(v)
    api.free(A)


@pytest.mark.parametrize("accum", [None, "GrB_PLUS_INT64", "GrB_MIN_INT64"])
@pytest.mark.parametrize("desc", [None, "GrB_DESC_S", "GrB_DESC_RS", "GrB_DESC_SC",
                                  "GrB_DESC_RSC"])
def test_assign_with_its_own_pattern_as_mask(api, oracle, accum, desc):
    """w<u> = accum(w, u) with u as both mask and source (the BFS parent
    update), against the oracle's accumulate / mask step.  Without GrB_STRUCTURE
    the mask is u's values (about 1% of them are zero)."""
    n = 5000
    rng = np.random.default_rng(11)
    wi = np.sort(rng.choice(n, 1200, replace=False)).astype(np.int64)
    ui = np.sort(rng.choice(n, 900, replace=False)).astype(np.int64)
    wx = rng.integers(-50, 50, len(wi)).astype(np.int64)
    ux = rng.integers(-50, 50, len(ui)).astype(np.int64)
    w = api.vector_from(wi, wx, 8, n)
    u = api.vector_from(ui, ux, 8, n)
    api.assign_all(w, u, accum, u, n, desc)
    gi, gx = api.vector_to(w, 8)
    replace, comp, strct = DESC_FLAGS[desc]
    acc = {None: None, "GrB_PLUS_INT64": "PLUS", "GrB_MIN_INT64": "MIN"}[accum]
    p1 = lambda k: np.array([0, k], np.int64)
    want = oracle.accum_mask(1, n, (p1(len(wi)), wi, wx), (p1(len(ui)), ui, ux), 8,
                             M=(p1(len(ui)), ui, ux, 8), mask_struct=strct,
                             mask_comp=comp, replace=replace, accum=acc)
    assert np.array_equal(gi, want[1]), "pattern, accum=%s desc=%s" % (accum, desc)
    assert np.array_equal(gx, want[2]), "values, accum=%s desc=%s" % (accum, desc)
    for v in (w, u):
        api.vfree(v)


@pytest.mark.parametrize("nw,nu", [(60000, 50000), (0, 3000), (3000, 0), (1, 1), (0, 0)])
def test_assign_union_many_tiles(api, oracle, nw, nu):
    """w<u> = u (structural, no accumulator, no replace) on row vectors is
    one merge-path union launch over tiles of 3072 merged positions: many
    tiles with ties across tile boundaries, and empty sides."""
    n = 200000
    rng = np.random.default_rng(nw + 7 * nu)
    wi = np.sort(rng.choice(n, nw, replace=False)).astype(np.int64)
    # u shares about a third of its indices with w
    share = wi[rng.random(nw) < (nu / max(nw, 1)) / 3] if nw else np.zeros(0, np.int64)
    rest = np.setdiff1d(rng.choice(n, nu, replace=False), share)[: max(nu - len(share), 0)]
    ui = np.sort(np.unique(np.concatenate([share, rest]))).astype(np.int64)
    wx = rng.integers(-50, 50, len(wi)).astype(np.int64)
    ux = rng.integers(-50, 50, len(ui)).astype(np.int64)
    w = api.vector_from(wi, wx, 8, n)
    u = api.vector_from(ui, ux, 8, n)
    api.assign_all(w, u, None, u, n, "GrB_DESC_S")
    gi, gx = api.vector_to(w, 8)
    p1 = lambda k: np.array([0, k], np.int64)
    want = oracle.accum_mask(1, n, (p1(len(wi)), wi, wx), (p1(len(ui)), ui, ux), 8,
                             M=(p1(len(ui)), ui, ux, 8), mask_struct=True)
    assert np.array_equal(gi, want[1])
    assert np.array_equal(gx, want[2])
    for v in (w, u):
        api.vfree(v)


def test_bfs_push_pull_parents_exact(api, oracle):
    """Direction-optimising BFS on R-MAT scale 18: levels with a large
    frontier pull (GrB_mxv with S as its own transpose, S symmetric: each
    unvisited vertex walks its row from the end to its largest frontier
    neighbour), the others push (GrB_vxm).  MAX_SECONDI makes both
    directions pick the largest frontier neighbour, the single-threaded
    reference's ANY rule, so every parent is bit-identical to the push-only
    traversal's."""
    S = W.rmat(18, 16, seed=2)
    n = S.nrows
    src = int(np.argmax(np.diff(S.p) > 0))
    A = api.matrix_from_csr(S, 1)
    q = api.vector_from([src], [src], 8, n)
    p = api.vector_from([src], [src], 8, n)
    pulls = 0
    while True:
        if api.vnvals(q) > n // 32:
            api.mxv(q, p, None, "GxB_MAX_SECONDI_INT64", A, q, "GrB_DESC_RSC")
            pulls += 1
        else:
            api.vxm(q, p, None, "GxB_MAX_SECONDI_INT64", q, A, "GrB_DESC_RSC")
        if api.vnvals(q) == 0:
            break
        api.assign_all(p, q, None, q, n, "GrB_DESC_S")
    idx, par = api.vector_to(p, 8)
    parent = np.full(n, -1, np.int64)
    parent[idx] = par
    want, _ = oracle.bfs(n, S.p, S.i, src)
    assert pulls >= 1
    assert np.array_equal(parent, want)
    for v in (q, p):
        api.vfree(v)
    api.free(A)


def test_pull_step_on_a_caller_stream(api, oracle):
    """One pull BFS step through GrB_mxv on a caller's stream (its scratch
    allocated for the call) and on the library's stream: the same parents."""
    import ctypes
    import torch
    S = W.rmat(12, 16, seed=4)
    n = S.nrows
    rng = np.random.default_rng(3)
    front = np.sort(rng.choice(n, 800, replace=False)).astype(np.int64)
    visited = np.sort(np.unique(np.concatenate([front, rng.choice(n, 1500, replace=False)])))
    A = api.matrix_from_csr(S, 1)
    outs = []
    for caller in (True, False):
        q = api.vector_from(front, front, 8, n)
        p = api.vector_from(visited, visited, 8, n)
        L_ = api.L
        st = torch.cuda.Stream()
        if caller:
            L_.grb_b200_set_stream(ctypes.c_void_p(st.cuda_stream))
        try:
            api.mxv(q, p, None, "GxB_MAX_SECONDI_INT64", A, q, "GrB_DESC_RSC")
        finally:
            if caller:
                L_.grb_b200_set_stream(None)
        outs.append(api.vector_to(q, 8))
        api.vfree(q)
        api.vfree(p)
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    # against the oracle: the largest frontier neighbour of every unvisited vertex
    fr = np.zeros(n, bool)
    fr[front] = True
    seen = np.zeros(n, bool)
    seen[visited] = True
    wi, wx = [], []
    for v in range(n):
        if seen[v]:
            continue
        nb = S.i[S.p[v]:S.p[v + 1]]
        nb = nb[fr[nb]]
        if len(nb):
            wi.append(v)
            wx.append(int(nb.max()))
    assert np.array_equal(outs[1][0], np.array(wi, np.int64))
    assert np.array_equal(outs[1][1], np.array(wx, np.int64))
    api.free(A)


@pytest.mark.parametrize("case", ["empty_frontier", "all_visited", "no_mask", "plain_mask"])
def test_pull_step_edge_cases(api, case):
    """The pull step (GrB_mxv with MAX_SECONDI) with an empty frontier, a
    visited set that covers every vertex, no mask, and a plain (not
    complemented) mask, against a dense evaluation."""
    S = W.rmat(10, 16, seed=8)
    n = S.nrows
    rng = np.random.default_rng(9)
    front = (np.zeros(0, np.int64) if case == "empty_frontier"
             else np.sort(rng.choice(n, 100, replace=False)).astype(np.int64))
    mask_idx = (np.arange(n, dtype=np.int64) if case == "all_visited"
                else np.sort(rng.choice(n, n // 2, replace=False)).astype(np.int64))
    A = api.matrix_from_csr(S, 1)
    q = api.vector_from(front, front, 8, n)
    w = api.vector_new(8, n)
    m = api.vector_from(mask_idx, mask_idx, 8, n)
    desc = {"empty_frontier": "GrB_DESC_RSC", "all_visited": "GrB_DESC_RSC",
            "no_mask": None, "plain_mask": "GrB_DESC_RS"}[case]
    api.mxv(w, None if case == "no_mask" else m, None, "GxB_MAX_SECONDI_INT64", A, q, desc)
    gi, gx = api.vector_to(w, 8)
    fr = np.zeros(n, bool)
    fr[front] = True
    inm = np.zeros(n, bool)
    inm[mask_idx] = True
    wi, wx = [], []
    for v in range(n):
        if case in ("empty_frontier", "all_visited") and inm[v]:
            continue
        if case == "plain_mask" and not inm[v]:
            continue
        nb = S.i[S.p[v]:S.p[v + 1]]
        nb = nb[fr[nb]]
        if len(nb):
            wi.append(v)
            wx.append(int(nb.max()))
    assert np.array_equal(gi, np.array(wi, np.int64)), case
    assert np.array_equal(gx, np.array(wx, np.int64)), case
    for v in (q, w, m):
        api.vfree(v)
    api.free(A)
