"""GrB/GxB serialize and deserialize through the GraphBLAS C API
(include/GraphBLAS_b200.h) with the matrices on the GPU: a blob written by
the reference (ZSTD, its default compression) becomes an operand of GrB_mxm,
and a product computed in HBM is written as a blob that decodes to the
oracle's product and that the reference's own GxB_Matrix_deserialize reads.
"""

import os

import numpy as np
import pytest

from graphblas_b200 import grb
from oracle import Reference, reference_available
from tests.helpers import assert_exact, random_csr

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "blobs.npz")


@pytest.fixture(scope="module")
def api(gpu):
    return grb.API()


def test_reference_blob_as_mxm_operand(api, oracle):
    d = np.load(GOLDEN)
    name = "fp32_sparse_col_zstd19"                 # ZSTD level 19, by column
    m, n, t, _ = d[name + "__shape"]
    A = api.matrix_deserialize(d[name + "__blob"].tobytes())
    assert api.nvals(A) == len(d[name + "__i"])
    Bc = random_csr(int(n), 37, 0.2, 5, dtype=np.float32)
    B = api.matrix_from_csr(Bc, 10)
    C = api.matrix_new(10, int(m), 37)
    api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP32", A, B)
    want = oracle.saxpy(int(m), 37, (d[name + "__p"], d[name + "__i"], d[name + "__x"], 10),
                        (Bc.p, Bc.i, Bc.x, 10), "PLUS", "TIMES", 10)
    assert_exact(api.matrix_to_csr(C, 10, int(m)), want, "deserialized A * B")
    for M in (A, B, C):
        api.free(M)


def test_golden_blobs_through_api(api):
    d = np.load(GOLDEN)
    for name in sorted({k.split("__")[0] for k in d.files}):
        m, n, t, iso = (int(v) for v in d[name + "__shape"])
        A = api.matrix_deserialize(d[name + "__blob"].tobytes(), type_code=t,
                                   gxb=name.endswith("none"))
        p, i, x = api.matrix_to_csr(A, t, m)
        assert np.array_equal(p, d[name + "__p"]) and np.array_equal(i, d[name + "__i"])
        assert np.array_equal(x, d[name + "__x"])
        api.free(A)
        with pytest.raises(grb.GrBError) as e:
            api.matrix_deserialize(d[name + "__blob"].tobytes(), type_code=8 if t != 8 else 11)
        assert e.value.info == -5                  # GrB_DOMAIN_MISMATCH


def test_device_product_serialized(api, oracle):
    Ac = random_csr(120, 90, 0.08, 1)
    Bc = random_csr(90, 110, 0.08, 2)
    A = api.matrix_from_csr(Ac, 11)
    B = api.matrix_from_csr(Bc, 11)
    C = api.matrix_new(11, 120, 110)
    api.mxm(C, None, None, "GrB_PLUS_TIMES_SEMIRING_FP64", A, B)   # C lives in HBM
    want = oracle.saxpy(120, 110, (Ac.p, Ac.i, Ac.x, 11), (Bc.p, Bc.i, Bc.x, 11),
                        "PLUS", "TIMES", 11)
    blob = api.matrix_serialize(C)
    blob2 = api.matrix_serialize(C, preallocated=True)
    assert blob == blob2
    nr, nc, t, p, i, x, iso = grb.blob_decode(blob)
    assert (nr, nc, t, iso) == (120, 110, 11, False)
    assert_exact((p, i, x), want, "serialized C")
    if reference_available():
        R = Reference(nthreads=1)
        nr, nc, t, p, i, x = R.deserialize(blob)
        assert (nr, nc, t) == (120, 110, 11)
        assert_exact((p, i, x), want, "reference-deserialized C")
    # the round trip gives the same product back
    C2 = api.matrix_deserialize(blob)
    assert_exact(api.matrix_to_csr(C2, 11, 120), want, "round trip")
    for M in (A, B, C, C2):
        api.free(M)


def test_serialize_short_buffer(api):
    import ctypes
    Ac = random_csr(30, 30, 0.2, 3)
    A = api.matrix_from_csr(Ac, 11)
    n = grb.U64()
    api.call("GrB_Matrix_serializeSize", ctypes.byref(n), A)
    buf = ctypes.create_string_buffer(n.value)
    short = grb.U64(n.value - 8)
    assert api.L.GrB_Matrix_serialize(buf, ctypes.byref(short), A) == -103
    api.free(A)


def test_vector_round_trip(api):
    n = 1000
    idx = np.array([0, 5, 17, 999], np.int64)
    vals = np.array([3, -1, 7, 42], np.int64)
    v = api.vector_from(idx, vals, 8, n)
    blob = api.vector_serialize(v)
    nr, nc, t, p, i, x, iso = grb.blob_decode(blob)       # an n-by-1 matrix
    assert (nr, nc, t) == (n, 1, 8)
    assert np.array_equal(np.repeat(np.arange(n), np.diff(p)), idx)
    w = api.vector_deserialize(blob)
    gi, gx = api.vector_to(w, 8)
    assert np.array_equal(gi, idx) and np.array_equal(gx, vals)
    d = np.load(GOLDEN)
    with pytest.raises(grb.GrBError) as e:                 # a matrix blob is no vector
        api.vector_deserialize(d["fp64_sparse_row_none__blob"].tobytes())
    assert e.value.info == -104
    for x_ in (v, w):
        api.vfree(x_)
