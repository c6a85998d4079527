"""ctypes front end of the GraphBLAS C API in include/GraphBLAS_b200.h.

Lets Python tests and the benchmark drive GrB_mxm / GrB_vxm / GrB_mxv the way
a C caller of SuiteSparse:GraphBLAS does (GrB_Matrix_new,
GxB_Matrix_pack_CSR, GrB_mxm(C, M, accum, semiring, A, B, desc), ...).  All
arithmetic happens in libgrb_b200.so.
"""

import ctypes

import numpy as np

from . import lib as _lib_loader, NP_OF, TYPES

_libc = ctypes.CDLL(None)
_libc.malloc.restype = ctypes.c_void_p
_libc.malloc.argtypes = [ctypes.c_size_t]
_libc.free.argtypes = [ctypes.c_void_p]

vp = ctypes.c_void_p
U64 = ctypes.c_uint64

TYPE_NAMES = {1: "GrB_BOOL", 6: "GrB_INT32", 7: "GrB_UINT32", 8: "GrB_INT64",
              9: "GrB_UINT64", 10: "GrB_FP32", 11: "GrB_FP64"}
SUFFIX = {1: "BOOL", 6: "INT32", 8: "INT64", 10: "FP32", 11: "FP64"}
SUFFIX_ALL = {**SUFFIX, 7: "UINT32", 9: "UINT64"}
CTYPE = {1: ctypes.c_bool, 6: ctypes.c_int32, 8: ctypes.c_int64,
         10: ctypes.c_float, 11: ctypes.c_double}


class GrBError(RuntimeError):
    def __init__(self, info, what):
        super().__init__("%s returned GrB_Info %d" % (what, info))
        self.info = info


class API:
    """The C API of the library, one instance per process."""

    _inited = False

    def __init__(self):
        self.L = _lib_loader()
        L = self.L
        for name in ("GrB_init", "GrB_finalize", "GrB_Matrix_new", "GrB_Matrix_free",
                     "GrB_Matrix_nvals", "GrB_Matrix_wait", "GxB_Matrix_pack_CSR",
                     "GxB_Matrix_unpack_CSR", "GrB_Vector_new", "GrB_Vector_free",
                     "GrB_Vector_nvals", "GxB_Vector_pack_CSC", "GxB_Vector_unpack_CSC",
                     "GrB_mxm", "GrB_vxm", "GrB_mxv", "GrB_Vector_assign",
                     "GrB_Semiring_new", "GrB_Descriptor_new", "GrB_Descriptor_set",
                     "GrB_Vector_setElement_INT64", "GrB_Matrix_dup", "GrB_Matrix_clear"):
            getattr(L, name).restype = ctypes.c_int
        L.GrB_Matrix_new.argtypes = [ctypes.POINTER(vp), vp, U64, U64]
        L.GrB_Matrix_free.argtypes = [ctypes.POINTER(vp)]
        L.GrB_Matrix_nvals.argtypes = [ctypes.POINTER(U64), vp]
        L.GrB_Matrix_wait.argtypes = [vp, ctypes.c_int]
        L.GxB_Matrix_pack_CSR.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                          ctypes.POINTER(vp), U64, U64, U64,
                                          ctypes.c_bool, ctypes.c_bool, vp]
        L.GxB_Matrix_unpack_CSR.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                            ctypes.POINTER(vp), ctypes.POINTER(U64),
                                            ctypes.POINTER(U64), ctypes.POINTER(U64),
                                            ctypes.POINTER(ctypes.c_bool),
                                            ctypes.POINTER(ctypes.c_bool), vp]
        L.GrB_Vector_new.argtypes = [ctypes.POINTER(vp), vp, U64]
        L.GrB_Vector_free.argtypes = [ctypes.POINTER(vp)]
        L.GrB_Vector_nvals.argtypes = [ctypes.POINTER(U64), vp]
        L.GxB_Vector_pack_CSC.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                          U64, U64, ctypes.c_bool, U64, ctypes.c_bool, vp]
        L.GxB_Vector_unpack_CSC.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                            ctypes.POINTER(U64), ctypes.POINTER(U64),
                                            ctypes.POINTER(ctypes.c_bool),
                                            ctypes.POINTER(U64),
                                            ctypes.POINTER(ctypes.c_bool), vp]
        L.GrB_mxm.argtypes = [vp] * 7
        L.GrB_vxm.argtypes = [vp] * 7
        L.GrB_mxv.argtypes = [vp] * 7
        L.GrB_Vector_assign.argtypes = [vp, vp, vp, vp, vp, U64, vp]
        L.GrB_Semiring_new.argtypes = [ctypes.POINTER(vp), vp, vp]
        L.GrB_Descriptor_new.argtypes = [ctypes.POINTER(vp)]
        L.GrB_Descriptor_set.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.GrB_Vector_setElement_INT64.argtypes = [vp, ctypes.c_int64, U64]
        L.GrB_Matrix_dup.argtypes = [ctypes.POINTER(vp), vp]
        L.GrB_Matrix_clear.argtypes = [vp]
        for suf in set(SUFFIX.values()) | {"UINT32", "UINT64"}:
            f = getattr(L, "GrB_Matrix_import_" + suf)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.POINTER(vp), vp, U64, U64, vp, vp, vp, U64, U64, U64,
                          ctypes.c_int]
            f = getattr(L, "GrB_Matrix_export_" + suf)
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, vp, ctypes.POINTER(U64), ctypes.POINTER(U64),
                          ctypes.POINTER(U64), ctypes.c_int, vp]
        for name in ("GrB_Matrix_serializeSize", "GrB_Matrix_serialize",
                     "GxB_Matrix_serialize", "GrB_Matrix_deserialize",
                     "GxB_Matrix_deserialize", "GxB_Vector_serialize",
                     "GxB_Vector_deserialize"):
            getattr(L, name).restype = ctypes.c_int
        L.GrB_Matrix_serializeSize.argtypes = [ctypes.POINTER(U64), vp]
        L.GrB_Matrix_serialize.argtypes = [vp, ctypes.POINTER(U64), vp]
        L.GxB_Matrix_serialize.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(U64), vp, vp]
        L.GxB_Vector_serialize.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(U64), vp, vp]
        L.GrB_Matrix_deserialize.argtypes = [ctypes.POINTER(vp), vp, vp, U64]
        L.GxB_Matrix_deserialize.argtypes = [ctypes.POINTER(vp), vp, vp, U64, vp]
        L.GxB_Vector_deserialize.argtypes = [ctypes.POINTER(vp), vp, vp, U64, vp]
        L.GrB_Matrix_exportSize.restype = ctypes.c_int
        L.GrB_Matrix_exportSize.argtypes = [ctypes.POINTER(U64), ctypes.POINTER(U64),
                                            ctypes.POINTER(U64), ctypes.c_int, vp]
        for suf in SUFFIX.values():
            f = getattr(L, "GrB_Vector_extractTuples_" + suf)
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, ctypes.POINTER(U64), vp]
        for t, suf in SUFFIX.items():
            f = getattr(L, "GrB_Matrix_reduce_" + suf)
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, vp, vp, vp]
            f = getattr(L, "GrB_Vector_reduce_" + suf)
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, vp, vp, vp]
        if not API._inited:
            info = L.GrB_init(0)
            if info not in (0, -3):       # -3: already initialised
                raise GrBError(info, "GrB_init")
            API._inited = True

    def obj(self, name):
        """A predefined object (type, operator, monoid, semiring, descriptor)."""
        if name is None:
            return None
        return vp.in_dll(self.L, name).value

    def call(self, name, *args):
        info = getattr(self.L, name)(*args)
        if info != 0:
            raise GrBError(info, name)
        return info

    # ---- matrices ----
    def matrix_new(self, type_code, nrows, ncols):
        A = vp()
        self.call("GrB_Matrix_new", ctypes.byref(A), self.obj(TYPE_NAMES[type_code]),
                  nrows, ncols)
        return A

    def matrix_from_csr(self, csr, type_code=None, iso=False):
        """GrB_Matrix_new + GxB_Matrix_pack_CSR from a Csr (copied into
        malloc'd arrays that the matrix then owns)."""
        if type_code is None:
            type_code = 1 if csr.x is None else {v: k for k, v in NP_OF.items()}[csr.x.dtype.type]
        A = self.matrix_new(type_code, csr.nrows, csr.ncols)
        ts = np.dtype(NP_OF[type_code]).itemsize
        nnz = int(csr.p[csr.nrows])
        p = _copy_to_malloc(np.ascontiguousarray(csr.p, np.int64))
        j = _copy_to_malloc(np.ascontiguousarray(csr.i, np.int64))
        if csr.x is None:
            one = np.ones(1, NP_OF[type_code])
            x = _copy_to_malloc(one)
            iso = True
            xs = ts
        else:
            x = _copy_to_malloc(np.ascontiguousarray(csr.x, NP_OF[type_code]))
            xs = max(nnz, 1) * ts
        pp, jp, xp = vp(p), vp(j), vp(x)
        self.call("GxB_Matrix_pack_CSR", A, ctypes.byref(pp), ctypes.byref(jp),
                  ctypes.byref(xp), (csr.nrows + 1) * 8, max(nnz, 1) * 8, xs, iso,
                  False, None)
        return A

    def matrix_import(self, type_code, nrows, ncols, p, i, x, nvals):
        """GrB_Matrix_import (CSR) from raw host addresses (numpy or pinned
        buffers): int64 offsets p, int64 indices i, nvals values x."""
        A = vp()
        self.call("GrB_Matrix_import_" + SUFFIX_ALL[type_code], ctypes.byref(A),
                  self.obj(TYPE_NAMES[type_code]), nrows, ncols, p, i, x, nrows + 1,
                  nvals, nvals, 0)
        return A

    def matrix_export(self, A, type_code, p, i, x, plen, nvals):
        """GrB_Matrix_export (CSR) into raw host addresses; returns nvals."""
        a, b, c = U64(plen), U64(nvals), U64(nvals)
        self.call("GrB_Matrix_export_" + SUFFIX_ALL[type_code], p, i, x, ctypes.byref(a),
                  ctypes.byref(b), ctypes.byref(c), 0, A)
        return b.value

    def export_size(self, A):
        a, b, c = U64(), U64(), U64()
        self.call("GrB_Matrix_exportSize", ctypes.byref(a), ctypes.byref(b),
                  ctypes.byref(c), 0, A)
        return a.value, b.value

    def vector_extract(self, v, type_code, i, x, cap):
        """GrB_Vector_extractTuples into raw host addresses; returns nvals."""
        n = U64(cap)
        self.call("GrB_Vector_extractTuples_" + SUFFIX[type_code], i, x, ctypes.byref(n), v)
        return n.value

    # ---- serialize / deserialize ----
    def matrix_serialize(self, A, preallocated=False):
        """The blob of A as bytes: GxB_Matrix_serialize, or with preallocated
        GrB_Matrix_serializeSize + GrB_Matrix_serialize into a caller buffer."""
        if preallocated:
            n = U64()
            self.call("GrB_Matrix_serializeSize", ctypes.byref(n), A)
            buf = ctypes.create_string_buffer(max(n.value, 1))
            used = U64(n.value)
            self.call("GrB_Matrix_serialize", buf, ctypes.byref(used), A)
            return buf.raw[:used.value]
        return self._take_blob("GxB_Matrix_serialize", A)

    def vector_serialize(self, v):
        return self._take_blob("GxB_Vector_serialize", v)

    def _take_blob(self, name, obj):
        bp, n = vp(), U64()
        self.call(name, ctypes.byref(bp), ctypes.byref(n), obj, None)
        out = ctypes.string_at(bp.value, n.value)
        _libc.free(bp.value)
        return out

    def matrix_deserialize(self, blob, type_code=None, gxb=True):
        """GxB_Matrix_deserialize (or GrB_Matrix_deserialize) of a bytes blob."""
        A = vp()
        t = None if type_code is None else self.obj(TYPE_NAMES[type_code])
        buf = ctypes.create_string_buffer(blob, max(len(blob), 1))
        if gxb:
            self.call("GxB_Matrix_deserialize", ctypes.byref(A), t, buf, len(blob), None)
        else:
            self.call("GrB_Matrix_deserialize", ctypes.byref(A), t, buf, len(blob))
        return A

    def vector_deserialize(self, blob, type_code=None):
        v = vp()
        t = None if type_code is None else self.obj(TYPE_NAMES[type_code])
        buf = ctypes.create_string_buffer(blob, max(len(blob), 1))
        self.call("GxB_Vector_deserialize", ctypes.byref(v), t, buf, len(blob), None)
        return v

    def matrix_to_csr(self, A, type_code, nrows):
        """GxB_Matrix_unpack_CSR into numpy (the matrix becomes empty)."""
        pp, jp, xp = vp(), vp(), vp()
        ps, js, xs = U64(), U64(), U64()
        iso = ctypes.c_bool()
        jumbled = ctypes.c_bool()
        self.call("GxB_Matrix_unpack_CSR", A, ctypes.byref(pp), ctypes.byref(jp),
                  ctypes.byref(xp), ctypes.byref(ps), ctypes.byref(js), ctypes.byref(xs),
                  ctypes.byref(iso), ctypes.byref(jumbled), None)
        p = _take(pp.value, nrows + 1, np.int64)
        nnz = int(p[-1])
        j = _take(jp.value, nnz, np.int64)
        dt = NP_OF[type_code]
        if iso.value:
            x1 = _take(xp.value, 1, dt)
            x = np.full(nnz, x1[0], dt)
        else:
            x = _take(xp.value, nnz, dt)
        return p, j, x

    def nvals(self, A):
        n = U64()
        self.call("GrB_Matrix_nvals", ctypes.byref(n), A)
        return n.value

    def free(self, A):
        if A is not None and A.value:
            self.L.GrB_Matrix_free(ctypes.byref(A))

    # ---- vectors ----
    def vector_new(self, type_code, n):
        v = vp()
        self.call("GrB_Vector_new", ctypes.byref(v), self.obj(TYPE_NAMES[type_code]), n)
        return v

    def vector_from(self, idx, vals, type_code, n):
        v = self.vector_new(type_code, n)
        idx = np.ascontiguousarray(idx, np.int64)
        dt = NP_OF[type_code]
        ip = vp(_copy_to_malloc(idx))
        xp = vp(_copy_to_malloc(np.ascontiguousarray(vals, dt)))
        self.call("GxB_Vector_pack_CSC", v, ctypes.byref(ip), ctypes.byref(xp),
                  max(len(idx), 1) * 8, max(len(idx), 1) * np.dtype(dt).itemsize,
                  False, len(idx), False, None)
        return v

    def vector_to(self, v, type_code):
        ip, xp = vp(), vp()
        isz, xsz, nv = U64(), U64(), U64()
        iso, jumbled = ctypes.c_bool(), ctypes.c_bool()
        self.call("GxB_Vector_unpack_CSC", v, ctypes.byref(ip), ctypes.byref(xp),
                  ctypes.byref(isz), ctypes.byref(xsz), ctypes.byref(iso),
                  ctypes.byref(nv), ctypes.byref(jumbled), None)
        n = nv.value
        idx = _take(ip.value, n, np.int64)
        dt = NP_OF[type_code]
        if iso.value:
            x1 = _take(xp.value, 1, dt)
            x = np.full(n, x1[0] if n else 0, dt)
        else:
            x = _take(xp.value, n, dt)
        return idx, x

    def vnvals(self, v):
        n = U64()
        self.call("GrB_Vector_nvals", ctypes.byref(n), v)
        return n.value

    def vfree(self, v):
        if v is not None and v.value:
            self.L.GrB_Vector_free(ctypes.byref(v))

    # ---- operations ----
    def mxm(self, C, M, accum, semiring, A, B, desc=None):
        return self.call("GrB_mxm", C, M, self.obj(accum), self.obj(semiring), A, B,
                         self.obj(desc))

    def vxm(self, w, mask, accum, semiring, u, A, desc=None):
        return self.call("GrB_vxm", w, mask, self.obj(accum), self.obj(semiring), u, A,
                         self.obj(desc))

    def mxv(self, w, mask, accum, semiring, A, u, desc=None):
        return self.call("GrB_mxv", w, mask, self.obj(accum), self.obj(semiring), A, u,
                         self.obj(desc))

    def assign_all(self, w, mask, accum, u, n, desc=None):
        GrB_ALL = vp.in_dll(self.L, "GrB_ALL").value
        return self.call("GrB_Vector_assign", w, mask, self.obj(accum), u, GrB_ALL, n,
                         self.obj(desc))

    def reduce(self, A, monoid, type_code, vector=False):
        out = CTYPE[type_code]()
        name = ("GrB_Vector_reduce_" if vector else "GrB_Matrix_reduce_") + SUFFIX[type_code]
        self.call(name, ctypes.byref(out), None, self.obj(monoid), A, None)
        return out.value

    def descriptor(self, **fields):
        d = vp()
        self.call("GrB_Descriptor_new", ctypes.byref(d))
        codes = {"outp": 0, "mask": 1, "inp0": 2, "inp1": 3, "method": 7090}
        for k, v in fields.items():
            self.call("GrB_Descriptor_set", d, codes[k], v)
        return d


def _blob_lib():
    L = _lib_loader()
    if not getattr(L, "_blob_bound", False):
        L.grb_b200_blob_decode.restype = ctypes.c_int
        L.grb_b200_blob_decode.argtypes = [vp, ctypes.c_size_t, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(vp), ctypes.POINTER(vp),
                                           ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_bool)]
        L.grb_b200_blob_encode.restype = ctypes.c_int
        L.grb_b200_blob_encode.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t),
                                           ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                           vp, vp, vp, ctypes.c_bool, ctypes.c_bool]
        L._blob_bound = True
    return L


def blob_decode(blob, expected_type=0):
    """Read a serialized-matrix blob on the host (no GPU): returns
    (nrows, ncols, type_code, p, i, x, iso), CSR by row; x holds one value
    when iso.  Raises GrBError with the GrB_Info of a rejected blob."""
    L = _blob_lib()
    buf = ctypes.create_string_buffer(bytes(blob), max(len(blob), 1))
    nr, nc, t = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
    pp, ip, xp = vp(), vp(), vp()
    iso = ctypes.c_bool()
    info = L.grb_b200_blob_decode(buf, len(blob), expected_type, ctypes.byref(nr),
                                  ctypes.byref(nc), ctypes.byref(t), ctypes.byref(pp),
                                  ctypes.byref(ip), ctypes.byref(xp), ctypes.byref(iso))
    if info != 0:
        raise GrBError(info, "grb_b200_blob_decode")
    p = _take(pp.value, nr.value + 1, np.int64)
    nnz = int(p[-1])
    i = _take(ip.value, nnz, np.int64)
    x = _take(xp.value, 1 if iso.value else nnz, NP_OF[t.value])
    return nr.value, nc.value, t.value, p, i, x, iso.value


def blob_encode(nrows, ncols, type_code, p, i, x, iso=False, by_col=False):
    """Write an uncompressed serialized-matrix blob on the host (no GPU)."""
    L = _blob_lib()
    p = np.ascontiguousarray(p, np.int64)
    i = np.ascontiguousarray(i, np.int64)
    x = np.ascontiguousarray(x, NP_OF[type_code])
    n = ctypes.c_size_t()
    args = (nrows, ncols, type_code, p.ctypes.data, i.ctypes.data if i.size else None,
            x.ctypes.data if x.size else None, iso, by_col)
    info = L.grb_b200_blob_encode(None, ctypes.byref(n), *args)
    if info != 0:
        raise GrBError(info, "grb_b200_blob_encode")
    buf = ctypes.create_string_buffer(n.value)
    info = L.grb_b200_blob_encode(buf, ctypes.byref(n), *args)
    if info != 0:
        raise GrBError(info, "grb_b200_blob_encode")
    return buf.raw[:n.value]


def _copy_to_malloc(a):
    n = max(a.nbytes, 8)
    ptr = _libc.malloc(n)
    if not ptr:
        raise MemoryError
    ctypes.memmove(ptr, a.ctypes.data, a.nbytes)
    return ptr


def _take(ptr, n, dt):
    dt = np.dtype(dt)
    if n == 0 or not ptr:
        if ptr:
            _libc.free(ptr)
        return np.zeros(0, dt)
    buf = (ctypes.c_char * (n * dt.itemsize)).from_address(ptr)
    out = np.frombuffer(buf, dtype=dt).copy()
    _libc.free(ptr)
    return out
