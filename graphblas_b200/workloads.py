"""Seeded synthetic workloads for the semiring SpGEMM path.

Thin numpy front end of ``lib/libgrb_b200_gen.so`` (``csrc/gen.c``).  Every
generator is counter-based, so results do not depend on the thread count or
the host.  Matrices are returned as ``Csr`` objects holding sorted,
duplicate-free CSR arrays with int64 row pointers and column indices, the
layout of a by-row GrB_Matrix in SuiteSparse:GraphBLAS
(Source/builtin/include/GB_matrix.h:213-235).

The reference measures on graph500-style R-MAT and Erdos-Renyi inputs; no
public dataset is used here.
"""

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_P = np.ctypeslib.ndpointer
_lib = None


def _gen():
    """The generator library: lib/libgrb_b200_gen.so, or the library named by
    $GRB_B200_GEN_LIB holding the same gen.c (bench.py's reference arm uses
    the reference runner's copy so that it loads nothing of this package)."""
    global _lib
    if _lib is None:
        path = os.environ.get("GRB_B200_GEN_LIB") or os.path.join(_HERE, "lib",
                                                                  "libgrb_b200_gen.so")
        L = ctypes.CDLL(path)
        i32, i64, f64, f32 = (_P(np.int32), _P(np.int64), _P(np.float64),
                              _P(np.float32))
        L.grbgen_rmat_edges.argtypes = [ctypes.c_int, ctypes.c_int64,
                                        ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_uint64,
                                        i32, i32]
        L.grbgen_csr_from_edges.argtypes = [ctypes.c_int64, ctypes.c_int64,
                                            i32, i32, ctypes.c_int,
                                            ctypes.c_int, i64, i64]
        L.grbgen_csr_from_edges.restype = ctypes.c_int64
        L.grbgen_split_tril_triu.argtypes = [ctypes.c_int64, i64, i64, i64,
                                             i64, i64, i64]
        L.grbgen_er_fixed.argtypes = [ctypes.c_int64, ctypes.c_int64,
                                      ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_uint64, i64,
                                      i64, ctypes.c_void_p, ctypes.c_void_p]
        L.grbgen_er_range.argtypes = [ctypes.c_int64, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_uint64, i64,
                                      ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
        L.grbgen_er_range.restype = ctypes.c_int64
        L.grbgen_poisson_minw.argtypes = [ctypes.c_int64, ctypes.c_double,
                                          ctypes.c_float, ctypes.c_float,
                                          ctypes.c_uint64, i64,
                                          ctypes.c_void_p, ctypes.c_void_p]
        L.grbgen_poisson_minw.restype = ctypes.c_int64
        L.grbgen_unif01.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.grbgen_unif01.restype = ctypes.c_double
        _lib = L
    return _lib


@dataclass
class Csr:
    """A sorted CSR matrix; ``x`` is None for a pattern (iso true) matrix."""
    nrows: int
    ncols: int
    p: np.ndarray
    i: np.ndarray
    x: np.ndarray = None

    @property
    def nnz(self):
        return int(self.p[self.nrows])

    def row_degrees(self):
        return np.diff(self.p)


def rmat(scale, edge_factor=16, abcd=(0.57, 0.19, 0.19, 0.05), seed=1):
    """Symmetrised R-MAT graph: 2^scale vertices, edge_factor*2^scale draws,
    self-loops and duplicates removed, boolean pattern."""
    L = _gen()
    n = 1 << scale
    m = edge_factor * n
    u = np.empty(m, np.int32)
    v = np.empty(m, np.int32)
    a, b, c, _ = abcd
    L.grbgen_rmat_edges(scale, m, a, b, c, seed, u, v)
    p = np.empty(n + 1, np.int64)
    i = np.empty(2 * m, np.int64)
    nnz = L.grbgen_csr_from_edges(n, m, u, v, 1, 1, p, i)
    if nnz < 0:
        raise MemoryError("rmat generator out of memory")
    return Csr(n, n, p, i[:nnz].copy())


def tril_triu(S):
    """Strict lower and upper triangles (L, U) of a square pattern matrix."""
    L = _gen()
    n = S.nrows
    Lp = np.empty(n + 1, np.int64)
    Up = np.empty(n + 1, np.int64)
    Li = np.empty(max(S.nnz, 1), np.int64)
    Ui = np.empty(max(S.nnz, 1), np.int64)
    L.grbgen_split_tril_triu(n, S.p, S.i, Lp, Li, Up, Ui)
    return (Csr(n, n, Lp, Li[:Lp[n]].copy()), Csr(n, n, Up, Ui[:Up[n]].copy()))


def er_fixed(nrows, ncols, d, seed=1, lo=-1.0, hi=1.0, dtype=np.float64):
    """Exactly d distinct uniform columns per row, values uniform [lo, hi]."""
    L = _gen()
    p = np.empty(nrows + 1, np.int64)
    i = np.empty(nrows * d, np.int64)
    x = np.empty(nrows * d, dtype)
    x64 = x.ctypes.data_as(ctypes.c_void_p) if dtype == np.float64 else None
    x32 = x.ctypes.data_as(ctypes.c_void_p) if dtype == np.float32 else None
    L.grbgen_er_fixed(nrows, ncols, d, lo, hi, seed, p, i, x64, x32)
    return Csr(nrows, ncols, p, i, x)


def er_range(n, dmin, dmax, seed=1, lo=-1.0, hi=1.0, dtype=np.float64):
    """Square Erdos-Renyi matrix with a uniform [dmin, dmax] count per row."""
    L = _gen()
    p = np.empty(n + 1, np.int64)
    nnz = L.grbgen_er_range(n, dmin, dmax, lo, hi, seed, p, None, None, None)
    i = np.empty(max(nnz, 1), np.int64)
    x = np.empty(max(nnz, 1), dtype)
    xp = x.ctypes.data_as(ctypes.c_void_p)
    L.grbgen_er_range(n, dmin, dmax, lo, hi, seed, p,
                      i.ctypes.data_as(ctypes.c_void_p),
                      xp if dtype == np.float64 else None,
                      xp if dtype == np.float32 else None)
    return Csr(n, n, p, i[:nnz], x[:nnz])


def poisson_minw(n, mean=6.0, wlo=0.1, whi=10.0, seed=1):
    """Poisson(mean) uniform columns per row, duplicates merged by min,
    weights uniform [wlo, whi] fp32 (square n-by-n)."""
    L = _gen()
    p = np.empty(n + 1, np.int64)
    raw = L.grbgen_poisson_minw(n, mean, wlo, whi, seed, p, None, None)
    i = np.empty(max(raw, 1), np.int64)
    x = np.empty(max(raw, 1), np.float32)
    nnz = L.grbgen_poisson_minw(n, mean, wlo, whi, seed, p,
                                i.ctypes.data_as(ctypes.c_void_p),
                                x.ctypes.data_as(ctypes.c_void_p))
    return Csr(n, n, p, i[:nnz].copy(), x[:nnz].copy())


def unif01(seed, ctr):
    return _gen().grbgen_unif01(seed, ctr)


def batch_sizes(count, nmin=64, nmax=8192, seed=7):
    """Log-uniform instance sizes in [nmin, nmax]."""
    lo, hi = math.log(nmin), math.log(nmax)
    return [int(round(math.exp(lo + (hi - lo) * unif01(seed, k))))
            for k in range(count)]


def batch_min_plus(count=4096, nmin=64, nmax=8192, mean=6.0, seed=11):
    """The batched workload: `count` independent square matrices A_k with
    log-uniform sizes, Poisson(mean) entries per row (duplicates merged by
    min) and fp32 weights uniform [0.1, 10]."""
    sizes = batch_sizes(count, nmin, nmax, seed)
    return [poisson_minw(n, mean, 0.1, 10.0, seed * 100003 + k)
            for k, n in enumerate(sizes)]
