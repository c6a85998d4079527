"""The oracle: test infrastructure for the semiring SpGEMM path.

Two checkers live here, both CPU-only:

* ``Oracle`` wraps ``liboracle.so``, a plain-C restatement of the
  reference's algorithm (``oracle/oracle.c``; every function there cites the
  SuiteSparse:GraphBLAS file:line it follows).
* ``Reference`` wraps ``_ref/libref_runner.so``, which drives the reference
  library itself (built from its own sources by ``oracle/ref.mk``) through its
  public C API.  It pins the restatement and serves as the CPU baseline.

Only the tests, the smoke check and the CPU-baseline leg of ``bench.py`` use
this package, and only as the checker: the product (``graphblas_b200``) never
imports it.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_P = np.ctypeslib.ndpointer

TYPE_CODES = {"bool": 1, "int32": 6, "uint32": 7, "int64": 8, "uint64": 9,
              "fp32": 10, "fp64": 11}
NP_TYPES = {1: np.bool_, 6: np.int32, 7: np.uint32, 8: np.int64, 9: np.uint64,
            10: np.float32, 11: np.float64}
OPS = {"FIRST": 72, "SECOND": 73, "ANY": 74, "PAIR": 75, "MIN": 76, "MAX": 77,
       "PLUS": 78, "MINUS": 79, "RMINUS": 80, "TIMES": 81, "DIV": 82, "LOR": 91,
       "LAND": 92, "LXOR": 93, "EQ": 102, "FIRSTI": 115, "FIRSTJ": 117,
       "SECONDI": 119, "SECONDJ": 121}


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.c_void_p)


def _i64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int64)


class Oracle:
    """ctypes front end of the C restatement (liboracle.so)."""

    def __init__(self, path=None):
        path = path or os.path.join(HERE, "liboracle.so")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        vp = ctypes.c_void_p
        L.oracle_saxpy.restype = vp
        L.oracle_saxpy.argtypes = [ctypes.c_int64, ctypes.c_int64,
                                   vp, vp, vp, ctypes.c_int, vp, vp, vp,
                                   ctypes.c_int, vp, vp, vp, ctypes.c_int,
                                   ctypes.c_bool, ctypes.c_bool, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int]
        L.oracle_dot3.restype = vp
        L.oracle_dot3.argtypes = [ctypes.c_int64, ctypes.c_int64,
                                  vp, vp, vp, ctypes.c_int, vp, vp, vp,
                                  ctypes.c_int, vp, vp, vp, ctypes.c_int,
                                  ctypes.c_bool, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int]
        L.oracle_accum_mask.restype = vp
        L.oracle_accum_mask.argtypes = [ctypes.c_int64, ctypes.c_int64,
                                        vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                        ctypes.c_int, ctypes.c_bool,
                                        ctypes.c_bool, ctypes.c_bool,
                                        ctypes.c_int, ctypes.c_int]
        L.oracle_nnz.restype = ctypes.c_int64
        L.oracle_nnz.argtypes = [vp]
        L.oracle_export.argtypes = [vp, vp, vp, vp]
        L.oracle_free.argtypes = [vp]
        L.oracle_tricount.restype = ctypes.c_int64
        L.oracle_tricount.argtypes = [ctypes.c_int64, vp, vp, vp, vp]
        L.oracle_bfs.restype = ctypes.c_int
        L.oracle_bfs.argtypes = [ctypes.c_int64, vp, vp, ctypes.c_int64, vp, vp]

    def _take(self, h, m, ctype):
        L = self.lib
        nnz = L.oracle_nnz(h)
        p = np.empty(m + 1, np.int64)
        i = np.empty(max(nnz, 1), np.int64)
        x = np.empty(max(nnz, 1), NP_TYPES[ctype])
        L.oracle_export(h, _ptr(p), _ptr(i), _ptr(x))
        L.oracle_free(h)
        return p, i[:nnz], x[:nnz]

    def saxpy(self, m, ncols, A, B, add, mult, ctype, M=None,
              mask_struct=True, mask_comp=False):
        """C<M> = A*B row by row.  A, B, M are (p, i, x, type) tuples."""
        Ap, Ai, Ax, at = A
        Bp, Bi, Bx, bt = B
        Mp = Mi = Mx = None
        mt = 1
        if M is not None:
            Mp, Mi, Mx, mt = M
        keep = [_i64(Ap), _i64(Ai), _i64(Bp), _i64(Bi), _i64(Mp), _i64(Mi)]
        h = self.lib.oracle_saxpy(m, ncols, _ptr(keep[0]), _ptr(keep[1]),
                                  _ptr(Ax), at, _ptr(keep[2]), _ptr(keep[3]),
                                  _ptr(Bx), bt, _ptr(keep[4]), _ptr(keep[5]),
                                  _ptr(Mx), mt, mask_struct, mask_comp,
                                  OPS[add], OPS[mult], ctype)
        return self._take(h, m, ctype)

    def dot3(self, m, ncols, A, B, M, add, mult, ctype, mask_struct=True):
        """C<M> = A*B' (row i of A dot row j of B), zombies removed."""
        Ap, Ai, Ax, at = A
        Bp, Bi, Bx, bt = B
        Mp, Mi, Mx, mt = M
        keep = [_i64(Ap), _i64(Ai), _i64(Bp), _i64(Bi), _i64(Mp), _i64(Mi)]
        h = self.lib.oracle_dot3(m, ncols, _ptr(keep[0]), _ptr(keep[1]),
                                 _ptr(Ax), at, _ptr(keep[2]), _ptr(keep[3]),
                                 _ptr(Bx), bt, _ptr(keep[4]), _ptr(keep[5]),
                                 _ptr(Mx), mt, mask_struct, OPS[add],
                                 OPS[mult], ctype)
        return self._take(h, m, ctype)

    def accum_mask(self, m, ncols, C, T, ctype, M=None, mask_struct=True,
                   mask_comp=False, replace=False, accum=None):
        Cp, Ci, Cx = C
        Tp, Ti, Tx = T
        Mp = Mi = Mx = None
        mt = 1
        if M is not None:
            Mp, Mi, Mx, mt = M
        keep = [_i64(Cp), _i64(Ci), _i64(Tp), _i64(Ti), _i64(Mp), _i64(Mi)]
        h = self.lib.oracle_accum_mask(
            m, ncols, _ptr(keep[0]), _ptr(keep[1]), _ptr(Cx), _ptr(keep[2]),
            _ptr(keep[3]), _ptr(Tx), _ptr(keep[4]), _ptr(keep[5]), _ptr(Mx),
            mt, mask_struct, mask_comp, replace, OPS[accum] if accum else 0,
            ctype)
        return self._take(h, m, ctype)

    def tricount(self, n, Lp, Li, Up, Ui):
        keep = [_i64(Lp), _i64(Li), _i64(Up), _i64(Ui)]
        return int(self.lib.oracle_tricount(n, *[_ptr(k) for k in keep]))

    def bfs(self, n, Sp, Si, src):
        parent = np.empty(n, np.int64)
        level = np.empty(n, np.int64)
        keep = [_i64(Sp), _i64(Si)]
        self.lib.oracle_bfs(n, _ptr(keep[0]), _ptr(keep[1]), src,
                            _ptr(parent), _ptr(level))
        return parent, level


class Reference:
    """ctypes front end of the reference library itself (oracle/_ref)."""

    def __init__(self, nthreads=None, path=None):
        path = path or os.path.join(HERE, "_ref", "libref_runner.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        vp = ctypes.c_void_p
        L.ref_init.argtypes = [ctypes.c_int]
        L.ref_set_nthreads.argtypes = [ctypes.c_int]
        L.ref_mxm.restype = vp
        L.ref_mxm.argtypes = ([ctypes.c_int64] * 3 + [vp, vp, vp, ctypes.c_int]
                              + [ctypes.c_int64, vp, vp, vp, ctypes.c_int]
                              + [vp, vp, vp, ctypes.c_int] + [vp, vp, vp]
                              + [ctypes.c_bool] * 4 + [ctypes.c_int] * 5
                              + [ctypes.POINTER(ctypes.c_int)])
        L.ref_nnz.restype = ctypes.c_int64
        L.ref_nnz.argtypes = [vp]
        L.ref_seconds.restype = ctypes.c_double
        L.ref_seconds.argtypes = [vp]
        L.ref_export.argtypes = [vp, vp, vp, vp]
        L.ref_free.argtypes = [vp]
        L.ref_tricount.argtypes = [ctypes.c_int64, vp, vp, vp, vp, ctypes.c_int,
                                   vp, vp]
        L.ref_bfs.argtypes = [ctypes.c_int64, vp, vp, ctypes.c_int64, vp, vp, vp]
        L.ref_serve_add_graph.argtypes = [ctypes.c_int, ctypes.c_int64, vp, vp, vp]
        L.ref_serve_clear.restype = None
        L.ref_serve_replay.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64] + [vp] * 10 \
            + [vp]
        L.ref_batch_square.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp,
                                       ctypes.c_int, ctypes.c_int, vp, vp, vp]
        L.ref_serialize.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, vp, vp,
                                    vp, ctypes.c_int, ctypes.c_bool, ctypes.c_int,
                                    ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_uint64)]
        L.ref_blob_free.argtypes = [vp]
        L.ref_blob_free.restype = None
        L.ref_deserialize.restype = vp
        L.ref_deserialize.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int)]
        self.nthreads = nthreads or os.cpu_count()
        info = L.ref_init(self.nthreads)
        if info != 0:
            raise RuntimeError("GrB_init failed: %d" % info)

    def set_nthreads(self, n):
        self.nthreads = n
        self.lib.ref_set_nthreads(n)

    def mxm(self, m, n, ncols, A, B, add, mult, ctype, M=None,
            mask_struct=True, mask_comp=False, replace=False,
            transpose_b=False, accum=None, C=None, method=0):
        """C<M> = accum(C, A*B or A*B') with the reference GrB_mxm; returns
        the sorted CSR (p, i, x) after GrB_Matrix_wait."""
        Ap, Ai, Ax, at = A
        Bp, Bi, Bx, bt = B
        Mp = Mi = Mx = None
        mt = 1
        if M is not None:
            Mp, Mi, Mx, mt = M
        Cp = Ci = Cx = None
        if C is not None:
            Cp, Ci, Cx = C
        bn = len(Bp) - 1
        keep = [_i64(a) for a in (Ap, Ai, Bp, Bi, Mp, Mi, Cp, Ci)]
        info = ctypes.c_int(0)
        h = self.lib.ref_mxm(m, n, ncols, _ptr(keep[0]), _ptr(keep[1]),
                             _ptr(Ax), at, bn, _ptr(keep[2]), _ptr(keep[3]),
                             _ptr(Bx), bt, _ptr(keep[4]), _ptr(keep[5]),
                             _ptr(Mx), mt, _ptr(keep[6]), _ptr(keep[7]),
                             _ptr(Cx), mask_struct, mask_comp, replace,
                             transpose_b, OPS[accum] if accum else 0,
                             OPS[add], OPS[mult], ctype, method,
                             ctypes.byref(info))
        if not h:
            raise RuntimeError("reference GrB_mxm failed: %d" % info.value)
        L = self.lib
        nnz = L.ref_nnz(h)
        p = np.empty(m + 1, np.int64)
        i = np.empty(max(nnz, 1), np.int64)
        x = np.empty(max(nnz, 1), NP_TYPES[ctype])
        L.ref_export(h, _ptr(p), _ptr(i), _ptr(x))
        L.ref_free(h)
        return p, i[:nnz], x[:nnz]

    def serialize(self, t, nrows, ncols, p, i, x, sparsity=2, by_col=False,
                  method=-1):
        """The reference's GxB_Matrix_serialize blob (bytes) of a CSR matrix
        (x None: iso-true pattern) stored with GxB_SPARSITY_CONTROL
        `sparsity`, by column when by_col, compressed with GxB_COMPRESSION
        `method`."""
        keep = [_i64(p), _i64(i)]
        xx = None if x is None else np.ascontiguousarray(x, NP_TYPES[t])
        bp, n = ctypes.c_void_p(), ctypes.c_uint64()
        info = self.lib.ref_serialize(t, nrows, ncols, _ptr(keep[0]), _ptr(keep[1]),
                                      _ptr(xx), sparsity, by_col, method,
                                      ctypes.byref(bp), ctypes.byref(n))
        if info != 0:
            raise RuntimeError("reference GxB_Matrix_serialize failed: %d" % info)
        out = ctypes.string_at(bp.value, n.value)
        self.lib.ref_blob_free(bp)
        return out

    def deserialize(self, blob):
        """The reference's GxB_Matrix_deserialize of a blob, as
        (nrows, ncols, type, p, i, x) CSR by row; raises with the GrB_Info
        of a rejected blob (attribute .info)."""
        buf = ctypes.create_string_buffer(bytes(blob), max(len(blob), 1))
        nr, nc, t, info = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int(), ctypes.c_int()
        h = self.lib.ref_deserialize(buf, len(blob), ctypes.byref(nr), ctypes.byref(nc),
                                     ctypes.byref(t), ctypes.byref(info))
        if not h:
            e = RuntimeError("reference GxB_Matrix_deserialize failed: %d" % info.value)
            e.info = info.value
            raise e
        L = self.lib
        nnz = L.ref_nnz(h)
        p = np.empty(nr.value + 1, np.int64)
        i = np.empty(max(nnz, 1), np.int64)
        x = np.empty(max(nnz, 1), NP_TYPES[t.value])
        L.ref_export(h, _ptr(p), _ptr(i), _ptr(x))
        L.ref_free(h)
        return nr.value, nc.value, t.value, p, i[:nnz], x[:nnz]

    def tricount(self, n, Lp, Li, Up, Ui, reps=1):
        keep = [_i64(a) for a in (Lp, Li, Up, Ui)]
        times = np.zeros(reps, np.float64)
        ntri = np.zeros(1, np.int64)
        info = self.lib.ref_tricount(n, *[_ptr(k) for k in keep], reps,
                                     _ptr(times), _ptr(ntri))
        if info != 0:
            raise RuntimeError("reference tricount failed: %d" % info)
        return int(ntri[0]), times

    def bfs(self, n, Sp, Si, src):
        keep = [_i64(Sp), _i64(Si)]
        parent = np.empty(n, np.int64)
        secs = np.zeros(1, np.float64)
        nlev = np.zeros(1, np.int32)
        info = self.lib.ref_bfs(n, _ptr(keep[0]), _ptr(keep[1]), src,
                                _ptr(parent), _ptr(secs), _ptr(nlev))
        if info != 0:
            raise RuntimeError("reference bfs failed: %d" % info)
        return parent, float(secs[0]), int(nlev[0])

    def batch_square(self, nsz, poff, ioff, Ap, Ai, Ax, add="MIN", mult="PLUS",
                     digests=False):
        """A loop of GrB_mxm calls C_i = A_i*A_i (fp32); returns nnz(C_i), the
        loop's seconds and, with `digests`, csr_digest of every C_i."""
        count = len(nsz)
        keep = [_i64(nsz), _i64(poff), _i64(ioff), _i64(Ap), _i64(Ai)]
        Ax = np.ascontiguousarray(Ax, dtype=np.float32)
        nnz_out = np.zeros(count, np.int64)
        secs = np.zeros(1, np.float64)
        dig = np.zeros(count, np.uint64) if digests else None
        info = self.lib.ref_batch_square(count, *[_ptr(k) for k in keep],
                                         _ptr(Ax), OPS[add], OPS[mult],
                                         _ptr(nnz_out), _ptr(secs), _ptr(dig))
        if info != 0:
            raise RuntimeError("reference batch failed: %d" % info)
        if digests:
            return nnz_out, float(secs[0]), dig
        return nnz_out, float(secs[0])


    def serve(self, graphs, trace, nworkers, nthreads_per_call):
        """Replay a request trace (graphblas_b200.serve.make_trace) through a
        pool of host threads running the reference library; graphs are the
        (kind, Csr) list of graphblas_b200.serve.make_graphs.  Returns
        (status, count, checksum, latency, makespan)."""
        L = self.lib
        L.ref_serve_clear()
        keep = []
        for kind, g in graphs:
            x = None
            if kind == 2:
                x = np.ascontiguousarray(g.x, np.float32)
            elif kind == 3:
                x = np.ascontiguousarray(g.x, np.float64)
            p, i = _i64(g.p), _i64(g.i)
            keep += [p, i, x]
            info = L.ref_serve_add_graph(kind, g.nrows, _ptr(p), _ptr(i), _ptr(x))
            if info != 0:
                raise RuntimeError("reference serve graph failed: %d" % info)
        kind = np.ascontiguousarray(trace["kind"], np.int32)
        graph = np.ascontiguousarray(trace["graph"], np.int32)
        t = np.ascontiguousarray(trace["t"], np.float64)
        fp, fi = _i64(trace["fp"]), _i64(trace["fi"])
        fx = np.ascontiguousarray(trace["fx"], np.float32)
        n = len(kind)
        status = np.zeros(n, np.int32)
        count = np.zeros(n, np.int64)
        checksum = np.zeros(n, np.float64)
        latency = np.zeros(n, np.float64)
        makespan = np.zeros(1, np.float64)
        L.ref_serve_replay(nworkers, nthreads_per_call, n, _ptr(kind), _ptr(graph),
                           _ptr(t), _ptr(fp), _ptr(fi), _ptr(fx), _ptr(status),
                           _ptr(count), _ptr(checksum), _ptr(latency), _ptr(makespan))
        L.ref_serve_clear()
        return status, count, checksum, latency, float(makespan[0])


_DK1, _DK2 = np.uint64(0x9E3779B97F4A7C15), np.uint64(0xC2B2AE3D27D4EB4F)
_DK3, _DK4 = np.uint64(0x165667B19E3779F9), np.uint64(0x27D4EB2F165667C5)


def csr_digest(p, i, x):
    """Position-weighted 64-bit digest of a CSR matrix: every entry's row,
    column and value bits, weighted by its position, summed mod 2^64 (the
    reference runner's csr_digest computes the same).  Equal digests mean the
    same sorted pattern and bit-identical values, short of a collision."""
    p = np.asarray(p, np.int64)
    n = len(p) - 1
    nnz = int(p[-1]) if n >= 0 else 0
    i = np.asarray(i[:nnz], np.int64).view(np.uint64)
    x = np.ascontiguousarray(x[:nnz])
    if x.dtype.itemsize == 4:
        bits = x.view(np.uint32).astype(np.uint64)
    elif x.dtype.itemsize == 8:
        bits = x.view(np.uint64)
    else:
        bits = x.view(np.uint8).astype(np.uint64)
    rows = np.repeat(np.arange(n, dtype=np.uint64), np.diff(p))
    t = np.arange(nnz, dtype=np.uint64)
    with np.errstate(over="ignore"):
        h = np.uint64(n) * _DK1 + np.uint64(nnz)
        terms = ((rows * _DK1 + i) * _DK2 + bits + np.uint64(1)) * (t * _DK3 + _DK4)
        return int(h + np.sum(terms, dtype=np.uint64))


def reference_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libref_runner.so"))
