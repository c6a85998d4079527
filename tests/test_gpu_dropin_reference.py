"""The drop-in, demonstrated on the reference library itself.

oracle/ref.mk links SuiteSparse:GraphBLAS (built from its own sources) with
the maintainer's shim graphblas_b200/integration/gb_b200_gateway.c and
-Wl,--wrap=GB_AxB_dot3,--wrap=GB_AxB_saxpy3, so the library's own GrB_mxm /
GrB_vxm run their dot3 and saxpy3 kernels on the B200 when GB_B200=1.  Every
result must equal the unmodified library's (bit for bit here: both follow the
same ascending-k order), and the shim's counters must show that the GPU
took every call that reached it (none declined to the CPU) and at least
one.  Skipped where the wrapped library was not built.
"""

import ctypes
import os

import numpy as np
import pytest

from graphblas_b200 import workloads as W
from tests.helpers import assert_exact, random_csr

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
WRAP_RUNNER = os.path.join(REF, "libref_runner_wrap.so")
WRAP_LIB = os.path.join(REF, "libgraphblas_b200wrap.so")


class Counters:
    """The shim's counters: calls the GPU took and calls it declined (a
    declined call runs the reference's own CPU kernel)."""

    def __init__(self, lib):
        self.taken = ctypes.c_int64.in_dll(lib, "gb_b200_gateway_taken")
        self.declined = ctypes.c_int64.in_dll(lib, "gb_b200_gateway_declined")

    def snap(self):
        return self.taken.value, self.declined.value

    def check(self, before, expect_calls=True):
        """Every call that reached the shim since `before` ran on the GPU,
        and (with expect_calls) at least one did."""
        t0, d0 = before
        assert self.declined.value == d0, "the shim declined a call (CPU fallback)"
        if expect_calls:
            assert self.taken.value > t0, "no call reached the GPU"


@pytest.fixture(scope="module")
def refs(gpu):
    if not (os.path.exists(WRAP_RUNNER) and os.path.exists(WRAP_LIB)):
        pytest.skip("wrapped reference library not built")
    from oracle import Reference
    os.environ["GB_B200"] = "1"
    wrapped = Reference(nthreads=1, path=WRAP_RUNNER)
    plain = Reference(nthreads=1)
    return wrapped, plain, Counters(ctypes.CDLL(WRAP_LIB))


def test_tricount_through_reference_grb_mxm(refs):
    wrapped, plain, cnt = refs
    S = W.rmat(12, 16, seed=31)
    L, U = W.tril_triu(S)
    before = cnt.snap()
    n1, _ = wrapped.tricount(S.nrows, L.p, L.i, U.p, U.i)
    cnt.check(before)                                # dot3 ran on the GPU
    n2, _ = plain.tricount(S.nrows, L.p, L.i, U.p, U.i)
    assert n1 == n2


@pytest.mark.parametrize("add,mult,tname,method", [
    ("PLUS", "TIMES", "fp64", 2), ("PLUS", "TIMES", "fp64", 0),
    ("MIN", "PLUS", "fp32", 0), ("PLUS", "PAIR", "int64", 0),
    ("ANY", "SECONDI", "int64", 2), ("PLUS", "TIMES", "int32", 0),
    ("ANY", "PAIR", "bool", 2),             # an iso result (GB_AxB_iso.c:79)
])
@pytest.mark.parametrize("mask", ["none", "mask", "comp"])
def test_mxm_through_reference(refs, add, mult, tname, method, mask):
    from oracle import TYPE_CODES, NP_TYPES
    wrapped, plain, cnt = refs
    tc = TYPE_CODES[tname]
    np_t = NP_TYPES[tc]
    m, k, n = 300, 250, 280
    A = random_csr(m, k, 0.03, 1, np_t, lo=0.5, hi=3.0)
    B = random_csr(k, n, 0.03, 2, np_t, lo=0.5, hi=3.0)
    M = random_csr(m, n, 0.2, 3, np.bool_)
    Mt = None if mask == "none" else (M.p, M.i, None, 1)
    before = cnt.snap()
    got = wrapped.mxm(m, k, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc,
                      M=Mt, mask_comp=(mask == "comp"), method=method)
    # the product reaches saxpy3 or dot3 (the reference picks between them and
    # its bitmap methods by sizes; these inputs are sparse enough for the
    # sparse methods), and the GPU takes it
    cnt.check(before)
    want = plain.mxm(m, k, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc), add, mult, tc,
                     M=Mt, mask_comp=(mask == "comp"), method=method)
    assert_exact(got, want, "%s_%s_%s %s" % (add, mult, tname, mask))


def test_masked_dot3_through_reference(refs):
    wrapped, plain, cnt = refs
    m, k, n = 200, 300, 220
    A = random_csr(m, k, 0.05, 4)
    B = random_csr(n, k, 0.05, 5)
    M = random_csr(m, n, 0.3, 6, np.bool_)
    before = cnt.snap()
    got = wrapped.mxm(m, k, n, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS", "TIMES",
                      11, M=(M.p, M.i, None, 1), transpose_b=True, method=1)
    cnt.check(before)
    want = plain.mxm(m, k, n, (A.p, A.i, A.x, 11), (B.p, B.i, B.x, 11), "PLUS", "TIMES",
                     11, M=(M.p, M.i, None, 1), transpose_b=True, method=1)
    assert_exact(got, want, "dot3 via reference")


def test_bfs_through_reference_vxm(refs):
    wrapped, plain, cnt = refs
    S = W.rmat(12, 16, seed=41)
    before = cnt.snap()
    p1, _, _ = wrapped.bfs(S.nrows, S.p, S.i, 2)
    cnt.check(before)                                # the vxm levels ran on the GPU
    p2, _, _ = plain.bfs(S.nrows, S.p, S.i, 2)
    assert np.array_equal(p1, p2)
