"""Serialized-matrix blobs (GxB_Matrix_serialize / GxB_Matrix_deserialize,
Source/serialize/GB_serialize.c:43, GB_deserialize.c:22) read and written by
the library's host code (graphblas_b200/csrc/grb_serialize.c, grb_zstd.c).

* The committed blobs in tests/golden/blobs.npz, written by the reference
  itself (tests/golden/make_blobs.py), decode to the matrices they hold: no
  reference build needed.
* Where the reference library is built here (oracle/_ref), fresh blobs of
  every type, compression method (none, LZ4, LZ4HC, ZSTD levels), storage
  form (hypersparse, sparse, bitmap, full; by row or column; iso) and a
  multi-block array decode bit-exactly, and blobs written by the library are
  read back by the reference's own GxB_Matrix_deserialize.
* Malformed blobs give the reference's error codes and never crash.

Host code only: nothing here needs a GPU.
"""

import os
import struct

import numpy as np
import pytest

from graphblas_b200 import grb, NP_OF
from oracle import Reference, reference_available

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "blobs.npz")

INVALID_OBJECT, DOMAIN_MISMATCH, NOT_IMPLEMENTED = -104, -5, -8
INSUFFICIENT_SPACE = -103
TYPES = [1, 6, 7, 8, 9, 10, 11]


@pytest.fixture(scope="module")
def R():
    if not reference_available():
        pytest.skip("reference library not built here")
    ref = Reference(nthreads=1)
    yield ref
    ref.set_nthreads(1)


def values(t, k, seed):
    rng = np.random.default_rng(seed)
    if t == 1:
        return rng.integers(0, 2, k).astype(np.bool_)
    if t in (10, 11):
        return rng.standard_normal(k).astype(NP_OF[t])
    if t == 9:
        return rng.integers(0, 2**63, k, dtype=np.uint64)
    if t == 7:
        return (np.arange(k) % 9).astype(np.uint32)
    return rng.integers(-50, 50, k).astype(NP_OF[t])


def pattern(m, n, density, seed):
    rng = np.random.default_rng(seed)
    mask = rng.random((m, n)) < density
    p = np.concatenate([[0], np.cumsum(mask.sum(1))]).astype(np.int64)
    i = np.nonzero(mask)[1].astype(np.int64)
    return p, i


def decoded(blob, **kw):
    nr, nc, t, p, i, x, iso = grb.blob_decode(blob, **kw)
    if iso:
        x = np.full(len(i), x[0], x.dtype)
    return nr, nc, t, p, i, x


def assert_same(got, want):
    nr, nc, t, p, i, x = got
    assert (nr, nc, t) == tuple(want[:3])
    assert np.array_equal(p, want[3])
    assert np.array_equal(i, want[4])
    assert x.dtype == np.dtype(NP_OF[t])
    assert np.array_equal(x.view(np.uint8), np.asarray(want[5], NP_OF[t]).view(np.uint8))


def test_golden_blobs_decode():
    d = np.load(GOLDEN)
    names = sorted({k.split("__")[0] for k in d.files})
    assert len(names) >= 10
    for name in names:
        m, n, t, iso = d[name + "__shape"]
        got = decoded(d[name + "__blob"].tobytes())
        assert_same(got, (m, n, t, d[name + "__p"], d[name + "__i"], d[name + "__x"]))
        # the blob's own type is accepted as the expected type; others are not
        decoded(d[name + "__blob"].tobytes(), expected_type=int(t))
        other = 8 if t != 8 else 11
        with pytest.raises(grb.GrBError) as e:
            grb.blob_decode(d[name + "__blob"].tobytes(), expected_type=other)
        assert e.value.info == DOMAIN_MISMATCH


@pytest.mark.parametrize("t", TYPES)
@pytest.mark.parametrize("iso", [False, True])
def test_own_round_trip(t, iso):
    for (m, n, dens) in [(0, 0, 0), (5, 0, 0), (0, 7, 0), (6, 9, 0.0), (40, 33, 0.25),
                         (3, 200, 0.9)]:
        p, i = pattern(m, n, dens, 3)
        x = values(t, 1 if iso else len(i), 5)
        blob = grb.blob_encode(m, n, t, p, i, x, iso=iso)
        nr, nc, tt, pp, ii, xx, isoo = grb.blob_decode(blob)
        assert (nr, nc, tt, isoo) == (m, n, t, iso)
        assert np.array_equal(pp, p) and np.array_equal(ii, i)
        assert np.array_equal(xx, x)


def test_own_blob_by_column_reads_back_by_row():
    m, n = 30, 20
    p, i = pattern(m, n, 0.3, 8)
    x = values(11, len(i), 9)
    rows = np.repeat(np.arange(m), np.diff(p))
    order = np.lexsort((rows, i))                  # by column, rows ascending
    cp = np.concatenate([[0], np.cumsum(np.bincount(i, minlength=n))]).astype(np.int64)
    blob = grb.blob_encode(m, n, 11, cp, rows[order], x[order], by_col=True)
    assert_same(decoded(blob), (m, n, 11, p, i, x))


FORMS = [(1, False), (2, True), (4, False), (8, True), (2, False), (4, True)]
METHODS = [-1, 1000, 2000, 2009, 0, 3001, 3019]


@pytest.mark.parametrize("t", TYPES)
@pytest.mark.parametrize("method", METHODS)
def test_reference_blobs_decode(R, t, method):
    m, n = 70, 50
    p, i = pattern(m, n, 0.15, t)
    x = values(t, len(i), method + 7)
    dense_p = np.arange(0, m * n + 1, n, dtype=np.int64)
    dense_i = np.tile(np.arange(n, dtype=np.int64), m)
    dense_x = values(t, m * n, 11)
    for sparsity, by_col in FORMS:
        if sparsity == 8:
            P, I, X = dense_p, dense_i, dense_x
        else:
            P, I, X = p, i, x
        blob = R.serialize(t, m, n, P, I, X, sparsity, by_col, method)
        assert_same(decoded(blob), (m, n, t, P, I, X))
    # iso-valued (pattern) matrices
    blob = R.serialize(t, m, n, p, i, None, 2, False, method)
    nr, nc, tt, pp, ii, xx, iso = grb.blob_decode(blob)
    assert iso and len(xx) == 1 and np.array_equal(ii, i)


@pytest.mark.parametrize("method", [1000, 2009, 0, 3019])
def test_reference_multi_block_arrays(R, method):
    """Arrays of many 64 KiB blocks (the reference splits large arrays across
    threads, GB_serialize_array.c:124-147), highly repetitive values (long
    matches, RLE) and random ones."""
    R.set_nthreads(8)
    try:
        m, n = 3000, 2000
        p, i = pattern(m, n, 0.012, 21)
        for t, x in ((11, values(11, len(i), 2)), (7, np.full(len(i), 7, np.uint32)),
                     (6, (np.arange(len(i)) % 17).astype(np.int32))):
            for sparsity, by_col in ((2, False), (1, True)):
                blob = R.serialize(t, m, n, p, i, x, sparsity, by_col, method)
                nblocks = struct.unpack_from("<i", blob, 120 + 8 * 3)[0]   # Ai blocks
                assert nblocks > 1
                assert_same(decoded(blob), (m, n, t, p, i, x))
    finally:
        R.set_nthreads(1)


@pytest.mark.parametrize("t", TYPES)
def test_reference_reads_own_blobs(R, t):
    for (m, n, dens, iso) in [(40, 33, 0.25, False), (40, 33, 0.25, True), (0, 0, 0, False),
                              (8, 5, 0.0, False), (1, 300, 0.5, False)]:
        p, i = pattern(m, n, dens, 13)
        x = values(t, 1 if iso else len(i), 17)
        blob = grb.blob_encode(m, n, t, p, i, x, iso=iso)
        nr, nc, tt, pp, ii, xx = R.deserialize(blob)
        assert (nr, nc, tt) == (m, n, t)
        assert np.array_equal(pp, p) and np.array_equal(ii, i)
        assert np.array_equal(xx, np.full(len(i), x[0]) if iso else x)
    # a vector: n-by-1, by column
    vi = np.array([1, 4, 9], np.int64)
    blob = grb.blob_encode(12, 1, t, np.array([0, 3], np.int64), vi, values(t, 3, 1),
                           by_col=True)
    nr, nc, tt, pp, ii, xx = R.deserialize(blob)
    assert (nr, nc) == (12, 1)
    assert np.array_equal(np.repeat(np.arange(12), np.diff(pp)), vi)


def test_encode_size_query_and_short_buffer():
    import ctypes
    L = grb._blob_lib()
    p, i = pattern(10, 10, 0.3, 1)
    x = values(11, len(i), 2)
    size = ctypes.c_size_t()
    assert L.grb_b200_blob_encode(None, ctypes.byref(size), 10, 10, 11, p.ctypes.data,
                                  i.ctypes.data, x.ctypes.data, False, False) == 0
    assert size.value == len(grb.blob_encode(10, 10, 11, p, i, x))
    buf = ctypes.create_string_buffer(size.value)
    short = ctypes.c_size_t(size.value - 1)
    assert L.grb_b200_blob_encode(buf, ctypes.byref(short), 10, 10, 11, p.ctypes.data,
                                  i.ctypes.data, x.ctypes.data, False,
                                  False) == INSUFFICIENT_SPACE


def _golden_blob(name):
    d = np.load(GOLDEN)
    return bytearray(d[name + "__blob"].tobytes())


def _info(blob, **kw):
    with pytest.raises(grb.GrBError) as e:
        grb.blob_decode(bytes(blob), **kw)
    return e.value.info


def test_malformed_blobs():
    b = _golden_blob("fp64_sparse_row_none")
    assert _info(b[:-1]) == INVALID_OBJECT                 # size field != length
    assert _info(b[:100]) == INVALID_OBJECT                 # shorter than a header
    c = bytearray(b)
    struct.pack_into("<i", c, 8, 14)                        # user-defined type
    assert _info(c) == DOMAIN_MISMATCH
    c = bytearray(b)
    struct.pack_into("<i", c, 8, 2)                         # GrB_INT8: not built here
    assert _info(c) == NOT_IMPLEMENTED
    c = bytearray(b)
    struct.pack_into("<q", c, 16 + 5 * 8, 4)                # typesize != sizeof(double)
    assert _info(c) == DOMAIN_MISMATCH
    c = bytearray(b)
    struct.pack_into("<q", c, 16 + 6 * 8, 8 * 1000)         # Ap_len inconsistent with vdim
    assert _info(c) == INVALID_OBJECT
    c = bytearray(b)
    struct.pack_into("<i", c, 116, 4 * 16)                  # no such sparsity
    assert _info(c) == INVALID_OBJECT
    # indices out of order inside a row
    p = np.array([0, 3], np.int64)
    assert _info(grb.blob_encode(1, 5, 11, p, np.array([0, 3, 2]), np.ones(3))) == INVALID_OBJECT
    assert _info(grb.blob_encode(1, 5, 11, p, np.array([0, 2, 2]), np.ones(3))) == INVALID_OBJECT
    assert _info(grb.blob_encode(1, 5, 11, p, np.array([0, 2, 5]), np.ones(3))) == INVALID_OBJECT


@pytest.mark.parametrize("name", ["fp64_hyper_col_lz4", "bool_sparse_row_zstd",
                                  "fp32_sparse_col_zstd19", "uint32_bitmap_col_zstd"])
def test_corrupted_payloads_are_rejected_or_valid(name):
    """Single-byte corruptions of compressed blobs: each either decodes to a
    well-formed matrix or is rejected with GrB_INVALID_OBJECT (the reader
    bounds-checks every step of LZ4 and ZSTD decoding)."""
    b = _golden_blob(name)
    rng = np.random.default_rng(99)
    rejected = 0
    for _ in range(300):
        c = bytearray(b)
        pos = int(rng.integers(160, len(c)))
        c[pos] ^= 1 << int(rng.integers(0, 8))
        try:
            nr, nc, t, p, i, x, iso = grb.blob_decode(bytes(c))
        except grb.GrBError as e:
            assert e.info in (INVALID_OBJECT, DOMAIN_MISMATCH, NOT_IMPLEMENTED)
            rejected += 1
            continue
        assert p[0] == 0 and np.all(np.diff(p) >= 0) and p[-1] == len(i)
        assert len(i) == 0 or (i.min() >= 0 and i.max() < nc)
    assert rejected > 0
