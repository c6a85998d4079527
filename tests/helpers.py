"""Shared checks for the parity tests.

Parity rules (the reference's own test rules, Test/GB_spec_compare.m:20-31 and
Test/isequal_roundoff.m):
  * integer, boolean, pair and min/max semirings: identical sorted pattern and
    bit-identical values;
  * floating PLUS/TIMES: identical sorted pattern and
    norm(C1-C2,1) <= 64*eps*max(norm(C1,1),1), matrix 1-norms (largest
    column sum of |.|), NaN/Inf positions equal.
"""

import numpy as np

FP_TOL_ULPS = 64


def csr_to_dense_cols_abs(p, i, x, ncols):
    """Column sums of |x| (for the matrix 1-norm)."""
    s = np.zeros(ncols, np.float64)
    np.add.at(s, i, np.abs(x.astype(np.float64)))
    return s


def assert_same_pattern(a, b, what=""):
    ap, ai = a[0], a[1]
    bp, bi = b[0], b[1]
    assert np.array_equal(np.asarray(ap), np.asarray(bp)), what + ": row pointers differ"
    assert np.array_equal(np.asarray(ai), np.asarray(bi)), what + ": column indices differ"


def assert_exact(a, b, what=""):
    assert_same_pattern(a, b, what)
    xa, xb = np.asarray(a[2]), np.asarray(b[2])
    if xa.dtype.kind == "f":
        # bit-identical, NaN included
        assert np.array_equal(xa.view(np.uint8), xb.astype(xa.dtype).view(np.uint8)), \
            what + ": values differ"
    else:
        assert np.array_equal(xa, xb.astype(xa.dtype)), what + ": values differ"


def assert_roundoff(a, b, ncols, what=""):
    assert_same_pattern(a, b, what)
    xa = np.asarray(a[2], np.float64)
    xb = np.asarray(b[2], np.float64)
    assert np.array_equal(np.isnan(xa), np.isnan(xb)), what + ": NaN pattern"
    assert np.array_equal(np.isinf(xa), np.isinf(xb)), what + ": Inf pattern"
    ok = np.isfinite(xa) & np.isfinite(xb)
    i = np.asarray(a[1])
    d = csr_to_dense_cols_abs(a[0], i[ok], (xa - xb)[ok], ncols).max(initial=0.0)
    n = csr_to_dense_cols_abs(a[0], i[ok], xa[ok], ncols).max(initial=0.0)
    eps = np.finfo(np.asarray(a[2]).dtype).eps if np.asarray(a[2]).dtype.kind == "f" else 0
    assert d <= FP_TOL_ULPS * eps * max(n, 1.0), \
        "%s: 1-norm error %g > %g" % (what, d, FP_TOL_ULPS * eps * max(n, 1.0))


def random_csr(nrows, ncols, density, seed, dtype=np.float64, lo=-1.0, hi=1.0,
               empty_rows=0.0):
    """Small seeded random CSR (sorted, no duplicates) for parity cases."""
    from graphblas_b200.workloads import Csr
    rng = np.random.default_rng(seed)
    rows_p = [0]
    cols = []
    for r in range(nrows):
        if empty_rows and rng.random() < empty_rows:
            rows_p.append(rows_p[-1])
            continue
        k = rng.binomial(ncols, density)
        c = np.sort(rng.choice(ncols, size=k, replace=False)) if k else np.zeros(0, np.int64)
        cols.append(c)
        rows_p.append(rows_p[-1] + k)
    i = np.concatenate(cols).astype(np.int64) if cols else np.zeros(0, np.int64)
    p = np.array(rows_p, np.int64)
    if dtype == np.bool_:
        x = rng.random(len(i)) < 0.7
    elif np.dtype(dtype).kind == "f":
        x = (lo + (hi - lo) * rng.random(len(i))).astype(dtype)
    else:
        x = rng.integers(-5, 6, len(i)).astype(dtype)
    return Csr(nrows, ncols, p, i, x)


def transpose_csr(A):
    """Host transpose (sorted) of a Csr, used to build reference-orientation
    inputs in tests."""
    from graphblas_b200.workloads import Csr
    rows = np.repeat(np.arange(A.nrows), np.diff(A.p))
    order = np.lexsort((rows, A.i))
    ti = rows[order].astype(np.int64)
    counts = np.bincount(A.i, minlength=A.ncols)
    tp = np.zeros(A.ncols + 1, np.int64)
    np.cumsum(counts, out=tp[1:])
    tx = None if A.x is None else A.x[order]
    return Csr(A.ncols, A.nrows, tp, ti, tx)
