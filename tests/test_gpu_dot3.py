"""GPU parity of masked dot3, C<M> = A*B' (row i of A . row j of B for (i,j)
in M), against the oracle (oracle/oracle.c restating
Source/mxm/template/GB_AxB_dot_cij.c), called through the C-ABI.
"""

import numpy as np
import pytest

from graphblas_b200 import workloads as W
from tests.helpers import assert_exact, assert_roundoff, random_csr

pytestmark = pytest.mark.gpu


def _dot3_dev(gb, M, A, B, sr, mask_struct=True, type_name=None):
    dM = gb.DMatrix.upload(M, type_name=None if M.x is not None else "bool")
    dA = gb.DMatrix.upload(A, type_name=type_name)
    dB = gb.DMatrix.upload(B, type_name=type_name)
    C = gb.dot3(dM, dA, dB, sr, mask_struct=mask_struct)
    out = C.download(prune=True)
    info = C.info()
    for d in (dM, dA, dB, C):
        d.free()
    return out, info


@pytest.mark.parametrize("scale", [6, 8, 10, 12, 14, 16])
def test_tricount_rmat(gpu, oracle, scale):
    S = W.rmat(scale, 16, seed=scale)
    L, U = W.tril_triu(S)
    ref = oracle.tricount(S.nrows, L.p, L.i, U.p, U.i)
    gb = gpu
    sr = gb.semiring("PLUS", "PAIR", "int64")
    dL = gb.DMatrix.upload(L, "bool")
    dU = gb.DMatrix.upload(U, "bool")
    C = gb.dot3(dL, dL, dU, sr)
    got = gb.reduce(C, "PLUS", np.int64)
    assert int(got) == ref
    # the full C matches too (pattern after zombie removal, counts exact)
    want = oracle.dot3(S.nrows, S.ncols, (L.p, L.i, None, 1), (U.p, U.i, None, 1),
                       (L.p, L.i, None, 1), "PLUS", "PAIR", 8)
    assert_exact(C.download(prune=True), want, "C<L>=L*U'")
    for d in (dL, dU, C):
        d.free()


@pytest.mark.parametrize("add,mult,tname,np_t", [
    ("PLUS", "TIMES", "fp64", np.float64),
    ("PLUS", "TIMES", "fp32", np.float32),
    ("PLUS", "TIMES", "int64", np.int64),
    ("PLUS", "TIMES", "int32", np.int32),
    ("MIN", "PLUS", "fp32", np.float32),
    ("MIN", "PLUS", "int64", np.int64),
    ("MAX", "PLUS", "fp64", np.float64),
    ("PLUS", "PAIR", "int64", np.int64),
    ("ANY", "SECONDI", "int64", np.int64),
    ("ANY", "FIRSTJ", "int64", np.int64),
    ("MIN", "SECONDI", "int64", np.int64),
    ("LOR", "LAND", "bool", np.bool_),
    ("PLUS", "FIRST", "fp64", np.float64),
    ("MIN", "SECOND", "fp64", np.float64),
])
@pytest.mark.parametrize("density", [0.02, 0.3])
def test_dot3_semirings(gpu, oracle, add, mult, tname, np_t, density):
    gb = gpu
    tc = gb.TYPES[tname]
    m, n, k = 120, 90, 200
    A = random_csr(m, k, density, 1, np_t, empty_rows=0.1)
    B = random_csr(n, k, density, 2, np_t, empty_rows=0.1)
    M = random_csr(m, n, 0.2, 3, np.bool_)
    M.x = None
    sr = gb.semiring(add, mult, tname)
    got, info = _dot3_dev(gb, M, A, B, sr)
    want = oracle.dot3(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc),
                       (M.p, M.i, None, 1), add, mult, tc)
    if np.dtype(np_t).kind == "f" and add in ("PLUS", "TIMES"):
        # the device folds matches in ascending k like the reference: exact
        assert_exact(got, want, "dot3 fp")
        assert_roundoff(got, want, n, "dot3 fp")
    else:
        assert_exact(got, want, "dot3")


def test_dot3_long_rows(gpu, oracle):
    """Rows longer than the shared-memory stage, heavy imbalance (hub rows)."""
    gb = gpu
    S = W.rmat(13, 32, seed=5)
    L, U = W.tril_triu(S)
    rng = np.random.default_rng(0)
    L.x = rng.random(L.nnz)
    U.x = rng.random(U.nnz)
    sr = gb.semiring("PLUS", "TIMES", "fp64")
    got, _ = _dot3_dev(gb, W.Csr(L.nrows, L.ncols, L.p, L.i), L, U, sr)
    want = oracle.dot3(S.nrows, S.ncols, (L.p, L.i, L.x, 11), (U.p, U.i, U.x, 11),
                       (L.p, L.i, None, 1), "PLUS", "TIMES", 11)
    assert_exact(got, want, "dot3 long rows")


@pytest.mark.parametrize("tname,np_t,alen,blen", [
    ("int64", np.int64, 400, 400), ("int32", np.int32, 400, 400),
    ("int64", np.int64, 3000, 80),        # A's rows the longer list: kept whole as keys
    ("int64", np.int64, 80, 3000)])       # B's rows the longer list
def test_dot3_count_bitmap_and_merge_mix(gpu, oracle, tname, np_t, alen, blen):
    """PLUS_PAIR on a mask large enough for the bitmap path, with rows whose
    column span fits the shared-memory bitmap (grouped) and rows spanning
    4M columns (left on the merge path), long and short lists, empty rows;
    list lengths up to alen (A) and blen (B)."""
    gb = gpu
    m, n, k = 3000, 2500, 4_000_000

    def rows(nr, seed, maxlen):
        r = np.random.default_rng(seed)
        p = [0]
        idx = []
        for q in range(nr):
            ln = int(r.integers(0, maxlen)) if q % 11 else 0
            hi = k if q % 2 else 60_000          # wide or narrow column span
            c = np.unique(r.integers(0, hi, ln))
            idx.append(c)
            p.append(p[-1] + len(c))
        return W.Csr(nr, k, np.array(p, np.int64), np.concatenate(idx).astype(np.int64),
                     np.ones(p[-1], np_t))
    A, B = rows(m, 1, alen), rows(n, 2, blen)
    M = random_csr(m, n, 0.03, 3, np.bool_)
    M.x = None
    assert M.nnz >= 1 << 16
    sr = gb.semiring("PLUS", "PAIR", tname)
    got, _ = _dot3_dev(gb, M, A, B, sr)
    tc = gb.TYPES[tname]
    want = oracle.dot3(m, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc),
                       (M.p, M.i, None, 1), "PLUS", "PAIR", tc)
    assert_exact(got, want, "plus_pair bitmap/merge mix")


def test_dot3_valued_mask(gpu, oracle):
    gb = gpu
    A = random_csr(60, 50, 0.2, 11)
    B = random_csr(70, 50, 0.2, 12)
    M = random_csr(60, 70, 0.3, 13)
    M.x = (np.arange(M.nnz) % 3).astype(np.float64)      # a third are false
    sr = gb.semiring("PLUS", "TIMES", "fp64")
    got, _ = _dot3_dev(gb, M, A, B, sr, mask_struct=False)
    want = oracle.dot3(60, 70, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11),
                       (M.p, M.i, M.x, 11), "PLUS", "TIMES", 11, mask_struct=False)
    assert_exact(got, want, "valued mask")


def test_dot3_edge_cases(gpu, oracle):
    gb = gpu
    sr = gb.semiring("PLUS", "PAIR", "int64")
    # empty A: every mask entry is a zombie
    A = W.Csr(10, 10, np.zeros(11, np.int64), np.zeros(0, np.int64))
    B = random_csr(12, 10, 0.5, 1, np.bool_)
    M = random_csr(10, 12, 0.5, 2, np.bool_)
    M.x = None
    got, info = _dot3_dev(gb, M, A, W.Csr(12, 10, B.p, B.i), sr, type_name="bool")
    assert got[0][-1] == 0 and info["nzombies"] == M.nnz
    # empty mask
    M0 = W.Csr(10, 12, np.zeros(11, np.int64), np.zeros(0, np.int64))
    A2 = random_csr(10, 10, 0.5, 3, np.bool_)
    got, info = _dot3_dev(gb, M0, W.Csr(10, 10, A2.p, A2.i), W.Csr(12, 10, B.p, B.i),
                          sr, type_name="bool")
    assert got[0][-1] == 0
    # single row / single column shapes
    A1 = random_csr(1, 40, 0.5, 4, np.int64)
    B1 = random_csr(1, 40, 0.5, 5, np.int64)
    M1 = W.Csr(1, 1, np.array([0, 1], np.int64), np.array([0], np.int64))
    sr2 = gb.semiring("PLUS", "TIMES", "int64")
    got, _ = _dot3_dev(gb, M1, A1, B1, sr2)
    want = oracle.dot3(1, 1, (A1.p, A1.i, A1.x, 8), (B1.p, B1.i, B1.x, 8),
                       (M1.p, M1.i, None, 1), "PLUS", "TIMES", 8)
    assert_exact(got, want, "1x1")


@pytest.mark.parametrize("tname,np_t", [("int64", np.int64), ("int32", np.int32)])
@pytest.mark.parametrize("mask_struct", [True, False])
def test_dot3_count_groups_valued_mask_and_sum(gpu, oracle, tname, np_t, mask_struct):
    """The counting path (PLUS_PAIR on integers) on skewed operands: key rows
    of every size (warp hash tables up to 1024 entries, block bitmaps above),
    groups keyed by A's rows and by B's rows, lists long enough for every
    lane class, empty rows, and a valued mask a third of whose entries are
    false.  C must equal the oracle's, and the sum that comes back with C
    (used by the following reduction) must equal the sum of its values."""
    gb = gpu
    S = W.rmat(12, 24, seed=17)
    n = S.nrows
    A = W.Csr(n, n, S.p, S.i, np.ones(S.nnz, np_t))
    T = W.rmat(12, 24, seed=18)
    B = W.Csr(n, n, T.p, T.i, np.ones(T.nnz, np_t))
    M = random_csr(n, n, 0.004, 19, np.float64, empty_rows=0.2)
    M.x = (np.arange(M.nnz) % 3).astype(np.float64)
    tc = gb.TYPES[tname]
    sr = gb.semiring("PLUS", "PAIR", tname)
    dM = gb.DMatrix.upload(M)
    dA = gb.DMatrix.upload(A)
    dB = gb.DMatrix.upload(B)
    C = gb.dot3(dM, dA, dB, sr, mask_struct=mask_struct)
    total = int(gb.reduce(C, "PLUS", np_t))
    got = C.download(prune=True)
    want = oracle.dot3(n, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc),
                       (M.p, M.i, None if mask_struct else M.x, 1 if mask_struct else 11),
                       "PLUS", "PAIR", tc, mask_struct=mask_struct)
    assert_exact(got, want, "plus_pair groups")
    assert total == int(np.sum(want[2].astype(np.int64)).astype(np_t))
    for d in (dM, dA, dB, C):
        d.free()


def test_dot3_on_a_caller_stream(gpu, oracle):
    """On a caller's stream (grb_b200_set_stream) the counting path's scratch
    is allocated for the call instead of taken from the library stream's
    buffer; the results are the same."""
    import ctypes
    import torch
    gb = gpu
    L_ = gb.lib()
    S = W.rmat(13, 16, seed=6)
    Lc, Uc = W.tril_triu(S)
    want = oracle.dot3(S.nrows, S.ncols, (Lc.p, Lc.i, None, 1), (Uc.p, Uc.i, None, 1),
                       (Lc.p, Lc.i, None, 1), "PLUS", "PAIR", 8)
    st = torch.cuda.Stream()
    L_.grb_b200_set_stream(ctypes.c_void_p(st.cuda_stream))
    try:
        got, _ = _dot3_dev(gb, Lc, Lc, Uc, gb.semiring("PLUS", "PAIR", "int64"),
                           type_name="bool")
    finally:
        L_.grb_b200_set_stream(None)
    assert_exact(got, want, "C<L>=L*U' on a caller stream")
    got2, _ = _dot3_dev(gb, Lc, Lc, Uc, gb.semiring("PLUS", "PAIR", "int64"),
                        type_name="bool")
    assert_exact(got2, want, "C<L>=L*U' on the library stream")
