"""GPU parity of row-wise saxpy3, C<M> = A*B, against the oracle
(oracle/oracle.c restating the coarse Gustavson/hash tasks of
Source/mxm/template/GB_AxB_saxpy3_template.c), called through the C-ABI.
Every bin is covered: shared-memory hash rows of each size class, heavy rows
in the dense accumulator (sequential-k and atomic variants), masks and
complemented masks.
"""

import numpy as np
import pytest

from graphblas_b200 import workloads as W
from tests.helpers import assert_exact, assert_roundoff, random_csr

pytestmark = pytest.mark.gpu


def _saxpy_dev(gb, A, B, sr, M=None, mask_comp=False, mask_struct=True,
               type_name=None):
    dA = gb.DMatrix.upload(A, type_name=type_name)
    dB = gb.DMatrix.upload(B, type_name=type_name)
    dM = None
    if M is not None:
        dM = gb.DMatrix.upload(M, type_name=None if M.x is not None else "bool")
    C = gb.saxpy3(dA, dB, sr, M=dM, mask_comp=mask_comp, mask_struct=mask_struct)
    out = C.download(prune=True)
    for d in (dA, dB, dM, C):
        if d is not None:
            d.free()
    return out


def test_er_plus_times_fp64_exact(gpu, oracle):
    """The saxpy3 configuration (Erdos-Renyi, 8 per row, U[-1,1]) at 4096."""
    gb = gpu
    A = W.er_fixed(4096, 4096, 8, seed=1)
    B = W.er_fixed(4096, 4096, 8, seed=2)
    got = _saxpy_dev(gb, A, B, gb.semiring("PLUS", "TIMES", "fp64"))
    want = oracle.saxpy(4096, 4096, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11),
                        "PLUS", "TIMES", 11)
    assert_roundoff(got, want, 4096, "er fp64")
    assert_exact(got, want, "er fp64 (k-ordered accumulation)")


SEMIRINGS = [
    ("PLUS", "TIMES", "fp64", np.float64),
    ("PLUS", "TIMES", "fp32", np.float32),
    ("PLUS", "TIMES", "int64", np.int64),
    ("PLUS", "TIMES", "int32", np.int32),
    ("MIN", "PLUS", "fp32", np.float32),
    ("MIN", "PLUS", "fp64", np.float64),
    ("MIN", "PLUS", "int32", np.int32),
    ("MAX", "PLUS", "fp32", np.float32),
    ("PLUS", "PAIR", "int64", np.int64),
    ("ANY", "SECONDI", "int64", np.int64),
    ("ANY", "FIRSTJ", "int64", np.int64),
    ("ANY", "SECONDJ", "int64", np.int64),
    ("MIN", "SECONDI", "int64", np.int64),
    ("MAX", "SECONDI", "int64", np.int64),
    ("LOR", "LAND", "bool", np.bool_),
    ("PLUS", "SECOND", "fp64", np.float64),
    ("ANY", "TIMES", "fp64", np.float64),
]


@pytest.mark.parametrize("add,mult,tname,np_t", SEMIRINGS)
@pytest.mark.parametrize("density", [0.01, 0.05, 0.3])
def test_saxpy_semirings_nomask(gpu, oracle, add, mult, tname, np_t, density):
    gb = gpu
    tc = gb.TYPES[tname]
    m, k, n = 150, 180, 160
    A = random_csr(m, k, density, 21, np_t, empty_rows=0.1)
    B = random_csr(k, n, density, 22, np_t, empty_rows=0.1)
    got = _saxpy_dev(gb, A, B, gb.semiring(add, mult, tname))
    want = oracle.saxpy(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc)
    assert_exact(got, want, "%s_%s_%s" % (add, mult, tname))


@pytest.mark.parametrize("add,mult,tname,np_t", SEMIRINGS[:10])
@pytest.mark.parametrize("comp", [False, True])
def test_saxpy_masked(gpu, oracle, add, mult, tname, np_t, comp):
    gb = gpu
    tc = gb.TYPES[tname]
    m, k, n = 130, 140, 150
    A = random_csr(m, k, 0.08, 31, np_t)
    B = random_csr(k, n, 0.08, 32, np_t)
    M = random_csr(m, n, 0.15, 33, np.bool_)
    M.x = None
    got = _saxpy_dev(gb, A, B, gb.semiring(add, mult, tname), M=M, mask_comp=comp)
    want = oracle.saxpy(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult,
                        tc, M=(M.p, M.i, None, 1), mask_comp=comp)
    assert_exact(got, want, "masked comp=%s" % comp)


def test_saxpy_valued_mask(gpu, oracle):
    gb = gpu
    A = random_csr(80, 90, 0.1, 41)
    B = random_csr(90, 70, 0.1, 42)
    M = random_csr(80, 70, 0.3, 43)
    M.x = (np.arange(M.nnz) % 2).astype(np.float64)
    got = _saxpy_dev(gb, A, B, gb.semiring("PLUS", "TIMES", "fp64"), M=M,
                     mask_struct=False)
    want = oracle.saxpy(80, 70, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS",
                        "TIMES", 11, M=(M.p, M.i, M.x, 11), mask_struct=False)
    assert_exact(got, want, "valued mask")


@pytest.mark.parametrize("add,mult,tname", [("PLUS", "PAIR", "int64"),
                                            ("PLUS", "TIMES", "fp64"),
                                            ("MIN", "PLUS", "fp32")])
def test_saxpy_rmat_square_heavy_rows(gpu, oracle, add, mult, tname):
    """R-MAT A*A: hub rows exceed every shared-memory bin (dense accumulator),
    both the atomic (order-free) and the sequential-k (floating PLUS) kinds."""
    gb = gpu
    S = W.rmat(11, 16, seed=3)
    rng = np.random.default_rng(1)
    np_t = {"int64": np.int64, "fp64": np.float64, "fp32": np.float32}[tname]
    tc = gb.TYPES[tname]
    x = (0.1 + 9.9 * rng.random(S.nnz)).astype(np_t)
    A = W.Csr(S.nrows, S.ncols, S.p, S.i, x)
    got = _saxpy_dev(gb, A, A, gb.semiring(add, mult, tname))
    want = oracle.saxpy(S.nrows, S.ncols, (A.p, A.i, A.x, tc), (A.p, A.i, A.x, tc),
                        add, mult, tc)
    assert_exact(got, want, "rmat A*A %s_%s" % (add, mult))


def test_vxm_bfs_step_complemented(gpu, oracle):
    """One BFS push step: q<!p> = q any_secondi S on R-MAT (a single heavy row)."""
    gb = gpu
    S = W.rmat(12, 16, seed=9)
    n = S.nrows
    rng = np.random.default_rng(2)
    front = np.sort(rng.choice(n, 300, replace=False)).astype(np.int64)
    visited = np.sort(np.unique(np.concatenate([front, rng.choice(n, 900, replace=False)])))
    q = W.Csr(1, n, np.array([0, len(front)], np.int64), front, front.copy())
    p = W.Csr(1, n, np.array([0, len(visited)], np.int64), visited.astype(np.int64))
    Sx = W.Csr(n, n, S.p, S.i)
    got = _saxpy_dev(gb, q, Sx, gb.semiring("ANY", "SECONDI", "int64"), M=p,
                     mask_comp=True, type_name="int64")
    want = oracle.saxpy(1, n, (q.p, q.i, q.x, 8), (S.p, S.i, None, 1), "ANY",
                        "SECONDI", 8, M=(p.p, p.i, None, 1), mask_comp=True)
    assert_exact(got, want, "bfs step")


def test_saxpy_edge_cases(gpu, oracle):
    gb = gpu
    sr = gb.semiring("PLUS", "TIMES", "fp64")
    # A with no entries
    A0 = W.Csr(20, 30, np.zeros(21, np.int64), np.zeros(0, np.int64), np.zeros(0))
    B = random_csr(30, 25, 0.3, 1)
    got = _saxpy_dev(gb, A0, B, sr)
    assert got[0][-1] == 0 and len(got[0]) == 21
    # B with empty rows hit by A (zero-flop rows)
    A = random_csr(20, 30, 0.3, 2)
    B0 = W.Csr(30, 25, np.zeros(31, np.int64), np.zeros(0, np.int64), np.zeros(0))
    got = _saxpy_dev(gb, A, B0, sr)
    assert got[0][-1] == 0
    # a mask with no entries: nothing allowed
    M0 = W.Csr(20, 25, np.zeros(21, np.int64), np.zeros(0, np.int64))
    got = _saxpy_dev(gb, A, B, sr, M=M0)
    assert got[0][-1] == 0
    # its complement allows everything
    got = _saxpy_dev(gb, A, B, sr, M=M0, mask_comp=True)
    want = oracle.saxpy(20, 25, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS",
                        "TIMES", 11)
    assert_exact(got, want, "complement of empty mask")


@pytest.mark.parametrize("add,mult,tname,np_t", [("PLUS", "TIMES", "fp64", np.float64),
                                                 ("MIN", "PLUS", "fp32", np.float32)])
def test_saxpy_short_rows_wide_columns(gpu, oracle, add, mult, tname, np_t):
    """Short rows (expand-sort-compress bin) over 2^24 + 5 columns: the sort
    keys (column, position) no longer fit 32 bits and take the 64-bit form;
    columns repeat inside a row so the runs are folded in ascending k."""
    gb = gpu
    tc = gb.TYPES[tname]
    rng = np.random.default_rng(17)
    m, k, n = 64, 300, (1 << 24) + 5
    A = random_csr(m, k, 0.05, 18, np_t, lo=0.5, hi=2.0)
    hot = rng.integers(0, n, 40)                 # columns shared by many rows of B
    bp, bi = [0], []
    for _ in range(k):
        c = np.unique(np.concatenate([rng.integers(0, n, 5), rng.choice(hot, 3)]))
        bi.append(c)
        bp.append(bp[-1] + len(c))
    bi = np.concatenate(bi).astype(np.int64)
    B = W.Csr(k, n, np.array(bp, np.int64), bi,
              (0.5 + 1.5 * rng.random(len(bi))).astype(np_t))
    got = _saxpy_dev(gb, A, B, gb.semiring(add, mult, tname))
    want = oracle.saxpy(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc)
    assert_exact(got, want, "wide columns %s_%s" % (add, mult))


def _frontier_case(seed, n_front=2000, scale=12):
    """A one-row product with a large frontier over R-MAT (the direct dense
    row), its B, and masks: the frontier's visited set and a random plain
    mask."""
    S = W.rmat(scale, 16, seed=seed)
    n = S.nrows
    rng = np.random.default_rng(seed)
    front = np.sort(rng.choice(n, n_front, replace=False)).astype(np.int64)
    visited = np.sort(np.unique(np.concatenate([front, rng.choice(n, n // 3, replace=False)])))
    plain = np.sort(rng.choice(n, n // 2, replace=False)).astype(np.int64)
    return S, n, front, visited.astype(np.int64), plain


@pytest.mark.parametrize("add,mult,tname,mask", [
    ("ANY", "SECONDI", "int64", "comp"), ("ANY", "SECONDI", "int64", None),
    ("ANY", "SECONDI", "int32", "plain"), ("ANY", "FIRSTJ", "int64", "comp"),
    ("MIN", "PLUS", "fp32", "comp"), ("PLUS", "TIMES", "int64", "plain"),
    ("ANY", "PAIR", "bool", "comp"), ("MAX", "SECONDI", "int64", None)])
def test_vxm_large_frontier_dense_row(gpu, oracle, add, mult, tname, mask):
    """u' (x) S with a large frontier goes straight to the dense row (no
    symbolic phase); packed state|k words for the max-k ANY semirings, byte
    flags and values for the others; plain and complemented masks."""
    gb = gpu
    S, n, front, visited, plain = _frontier_case(21)
    tc = gb.TYPES[tname]
    np_t = {"int64": np.int64, "int32": np.int32, "fp32": np.float32, "bool": np.bool_}[tname]
    rng = np.random.default_rng(5)
    ux = (1 + rng.integers(0, 50, len(front))).astype(np_t)
    sx = (1 + rng.integers(0, 9, S.nnz)).astype(np_t)
    u = W.Csr(1, n, np.array([0, len(front)], np.int64), front, ux)
    B = W.Csr(n, n, S.p, S.i, sx)
    M = None
    if mask == "comp":
        M = W.Csr(1, n, np.array([0, len(visited)], np.int64), visited)
    elif mask == "plain":
        M = W.Csr(1, n, np.array([0, len(plain)], np.int64), plain)
    got = _saxpy_dev(gb, u, B, gb.semiring(add, mult, tname), M=M,
                     mask_comp=(mask == "comp"), type_name=tname)
    want = oracle.saxpy(1, n, (u.p, u.i, u.x, tc), (B.p, B.i, B.x, tc), add, mult, tc,
                        M=None if M is None else (M.p, M.i, None, 1),
                        mask_comp=(mask == "comp"))
    assert_exact(got, want, "dense row %s_%s_%s mask=%s" % (add, mult, tname, mask))


def test_saxpy_slots_overflow_on_caller_stream(gpu, oracle):
    """On a caller's stream the slots are the call's own buffer, first sized
    from B's mean row length: rows that all hit one long row of B need far
    more, so the bins run again with the buffer grown, and the result is
    unchanged."""
    import torch
    gb = gpu
    L = gb.lib()
    n = 20001
    rng = np.random.default_rng(4)
    bp = np.zeros(n + 1, np.int64)
    bp[1:] = 20000                         # row 0 holds columns 1..20000
    bi = np.arange(1, 20001, dtype=np.int64)
    B = W.Csr(n, n, bp, bi, rng.random(20000))
    m = 200
    A = W.Csr(m, n, np.arange(m + 1, dtype=np.int64), np.zeros(m, np.int64),
              1.0 + rng.random(m))
    st = torch.cuda.Stream()
    L.grb_b200_set_stream(ctypes_void(st.cuda_stream))
    try:
        got = _saxpy_dev(gb, A, B, gb.semiring("PLUS", "TIMES", "fp64"))
    finally:
        L.grb_b200_set_stream(None)
    want = oracle.saxpy(m, n, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS", "TIMES", 11)
    assert_exact(got, want, "slots grown on a caller stream")
    # the same on the library's own stream, then a small product after it
    got = _saxpy_dev(gb, A, B, gb.semiring("PLUS", "TIMES", "fp64"))
    assert_exact(got, want, "slots on the library stream")
    A2 = random_csr(30, n, 0.001, 9)
    got = _saxpy_dev(gb, A2, B, gb.semiring("PLUS", "TIMES", "fp64"))
    want = oracle.saxpy(30, n, (A2.p, A2.i, A2.x, 11), (B.p, B.i, B.x, 11), "PLUS",
                        "TIMES", 11)
    assert_exact(got, want, "small product after a large one")


def ctypes_void(ptr):
    import ctypes
    return ctypes.c_void_p(ptr)


@pytest.mark.parametrize("add,mult,tname", [("PLUS", "TIMES", "int64"),
                                            ("ANY", "SECONDI", "int64")])
def test_saxpy_many_heavy_rows(gpu, oracle, add, mult, tname):
    """More than 1024 heavy rows in one product: their offsets into the flat
    product index take the multi-launch path, and the rows share the
    grid-wide compaction."""
    gb = gpu
    tc = gb.TYPES[tname]
    m, k, n = 1500, 200, 5000
    rng = np.random.default_rng(8)
    A = W.Csr(m, k, np.arange(0, (m + 1) * k, k, dtype=np.int64),
              np.tile(np.arange(k, dtype=np.int64), m),
              rng.integers(1, 5, m * k).astype(np.int64))
    bp, bi = [0], []
    for _ in range(k):
        c = np.sort(rng.choice(n, 100, replace=False))
        bi.append(c)
        bp.append(bp[-1] + 100)
    B = W.Csr(k, n, np.array(bp, np.int64), np.concatenate(bi).astype(np.int64),
              rng.integers(1, 5, 100 * k).astype(np.int64))
    got = _saxpy_dev(gb, A, B, gb.semiring(add, mult, tname))
    want = oracle.saxpy(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc)
    assert_exact(got, want, "many heavy rows %s_%s" % (add, mult))


def test_caller_stream_keeping_a_scratch_buffer(gpu, oracle):
    """A caller's stream that keeps a scratch buffer (grb_b200_stream_keep_
    scratch): products before and after the buffer grows, and a masked dot
    product, give the results of the library's own streams; the buffer is
    released before the stream goes."""
    import ctypes
    import torch
    gb = gpu
    L = gb.lib()
    st = torch.cuda.Stream()
    h = ctypes.c_void_p(st.cuda_stream)
    assert L.grb_b200_stream_keep_scratch(h, True) == 0
    L.grb_b200_set_stream(h)
    try:
        A = random_csr(300, 400, 0.02, 31)
        B = random_csr(400, 500, 0.02, 32)
        small = _saxpy_dev(gb, A, B, gb.semiring("PLUS", "TIMES", "fp64"))
        A2 = random_csr(3000, 4000, 0.01, 33)
        B2 = random_csr(4000, 5000, 0.01, 34)
        big = _saxpy_dev(gb, A2, B2, gb.semiring("PLUS", "TIMES", "fp64"))
        S = W.rmat(11, 16, seed=5)
        Lc, Uc = W.tril_triu(S)
        dL = gb.DMatrix.upload(Lc, "bool")
        dU = gb.DMatrix.upload(Uc, "bool")
        C = gb.dot3(dL, dL, dU, gb.semiring("PLUS", "PAIR", "int64"))
        tri = C.download(prune=True)
        for d in (dL, dU, C):
            d.free()
    finally:
        L.grb_b200_set_stream(None)
        assert L.grb_b200_stream_keep_scratch(h, False) == 0
        st.synchronize()
    assert_exact(small, oracle.saxpy(300, 500, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11),
                                     "PLUS", "TIMES", 11), "small product")
    assert_exact(big, oracle.saxpy(3000, 5000, (A2.p, A2.i, A2.x, 11), (B2.p, B2.i, B2.x, 11),
                                   "PLUS", "TIMES", 11), "larger product")
    want = oracle.dot3(S.nrows, S.ncols, (Lc.p, Lc.i, None, 1), (Uc.p, Uc.i, None, 1),
                       (Lc.p, Lc.i, None, 1), "PLUS", "PAIR", 8)
    assert_exact(tri, want, "C<L>=L*U'")


# ---- the one-launch path for small products (k_saxpy_small) ----------------

@pytest.mark.parametrize("add,mult,tname,np_t", SEMIRINGS)
def test_one_launch_small_products(gpu, oracle, add, mult, tname, np_t):
    """256+ rows whose products fit the expand-sort-compress bin: the product
    runs in one launch (products per row, slots, expand-sort-compress, C's
    offsets and entries, with two grid barriers between them)."""
    gb = gpu
    tc = gb.TYPES[tname]
    m, k, n = 700, 500, 800
    A = random_csr(m, k, 0.012, 51, np_t, empty_rows=0.1)
    B = random_csr(k, n, 0.012, 52, np_t, empty_rows=0.1)
    got = _saxpy_dev(gb, A, B, gb.semiring(add, mult, tname))
    want = oracle.saxpy(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc)
    assert_exact(got, want, "one launch %s_%s_%s" % (add, mult, tname))


@pytest.mark.parametrize("add,mult,tname,np_t", SEMIRINGS[:10])
@pytest.mark.parametrize("comp", [False, True])
def test_one_launch_small_products_masked(gpu, oracle, add, mult, tname, np_t, comp):
    gb = gpu
    tc = gb.TYPES[tname]
    m, k, n = 520, 400, 450
    A = random_csr(m, k, 0.015, 61, np_t)
    B = random_csr(k, n, 0.015, 62, np_t)
    M = random_csr(m, n, 0.05, 63, np.bool_)
    M.x = None
    got = _saxpy_dev(gb, A, B, gb.semiring(add, mult, tname), M=M, mask_comp=comp)
    want = oracle.saxpy(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult,
                        tc, M=(M.p, M.i, None, 1), mask_comp=comp)
    assert_exact(got, want, "one launch masked comp=%s" % comp)


def _csr_from_rows(nrows, ncols, rows, seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(nrows + 1, np.int64)
    for r, c in rows.items():
        p[r + 1] = len(c)
    p = np.cumsum(p)
    i = np.concatenate([np.sort(np.asarray(rows[r], np.int64)) for r in sorted(rows)]) \
        if rows else np.zeros(0, np.int64)
    return W.Csr(nrows, ncols, p, i, rng.random(len(i)) - 0.5)


@pytest.mark.parametrize("case", ["row_past_bin", "c_past_estimate", "b_mean_under_one"])
def test_one_launch_fallbacks(gpu, oracle, case):
    """Products the one-launch path starts but cannot finish go to the general
    path with the same result: a row of more than 256 products, and more
    entries than C's arrays sized from B's mean row length (rows reading
    only B's long rows; B's mean row length under one)."""
    gb = gpu
    rng = np.random.default_rng(7)
    m, k, n = 600, 400, 3000
    if case == "row_past_bin":
        B = random_csr(k, n, 0.004, 71)                      # about 12 per row
        arows = {r: rng.choice(k, 4, replace=False) for r in range(m)}
        arows[17] = rng.choice(k, 120, replace=False)        # about 1400 products
    elif case == "c_past_estimate":
        # half of B's rows hold 200 columns, the other half none; A reads only
        # the long ones, so every row has about twice B's mean row length
        brows = {r: (rng.choice(n, 200, replace=False) if r % 2 == 0 else [])
                 for r in range(k)}
        B = _csr_from_rows(k, n, brows, 72)
        arows = {r: [2 * int(rng.integers(0, k // 2))] for r in range(m)}
    else:
        # one row of B holds 250 columns (mean row length under 1): every
        # row of C has 250 entries against an estimate of one
        brows = {r: (rng.choice(n, 250, replace=False) if r == 5 else []) for r in range(k)}
        B = _csr_from_rows(k, n, brows, 73)
        arows = {r: [5] for r in range(m)}
    A = _csr_from_rows(m, k, arows, 74)
    got = _saxpy_dev(gb, A, B, gb.semiring("PLUS", "TIMES", "fp64"))
    want = oracle.saxpy(m, n, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS", "TIMES", 11)
    assert_exact(got, want, case)


def test_one_launch_route(gpu):
    """The saxpy configuration's product (Erdos-Renyi, 8 per row) at 4096 rows
    launches the one-launch kernel and none of the general path's."""
    import torch
    from torch.profiler import profile, ProfilerActivity
    gb = gpu
    A = W.er_fixed(4096, 4096, 8, seed=1)
    B = W.er_fixed(4096, 4096, 8, seed=2)
    dA, dB = gb.DMatrix.upload(A), gb.DMatrix.upload(B)
    sr = gb.semiring("PLUS", "TIMES", "fp64")
    gb.saxpy3(dA, dB, sr).free()
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        C = gb.saxpy3(dA, dB, sr)
        torch.cuda.synchronize()
    names = [e.name for e in prof.events() if e.device_type.name == "CUDA"]
    C.free(); dA.free(); dB.free()
    assert any("k_saxpy_small" in s for s in names), names
    assert not any("k_saxpy_esc" in s or "k_flops_flat" in s or "k_pack" in s
                   for s in names), names
