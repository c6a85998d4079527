"""graphblas_b200: B200-native semiring sparse matrix multiply for
SuiteSparse:GraphBLAS's GrB_mxm / GrB_vxm path.

The product is the native library ``lib/libgrb_b200.so`` (CUDA kernels for
sm_100a behind the C-ABI in ``include/grb_b200.h``).  This module is a thin
ctypes front end used by the tests and the benchmark; it never computes
anything itself and fails loudly when the native library is missing.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgrb_b200.so")

# GrB_Info codes (Include/GraphBLAS.h:358-381)
SUCCESS, NO_VALUE = 0, 1
NULL_POINTER, INVALID_VALUE, DIMENSION_MISMATCH = -2, -3, -6
PANIC, OUT_OF_MEMORY = -101, -102

# GB_Type_code and GB_Opcode values (Source/builtin/include/GB_opaque.h)
TYPES = {"bool": 1, "int32": 6, "uint32": 7, "int64": 8, "uint64": 9,
         "fp32": 10, "fp64": 11}
NP_OF = {1: np.bool_, 6: np.int32, 7: np.uint32, 8: np.int64, 9: np.uint64,
         10: np.float32, 11: np.float64}
CODE_OF_NP = {np.dtype(v): k for k, v in NP_OF.items()}
OPS = {"FIRST": 72, "SECOND": 73, "ANY": 74, "PAIR": 75, "MIN": 76, "MAX": 77,
       "PLUS": 78, "MINUS": 79, "RMINUS": 80, "TIMES": 81, "DIV": 82,
       "LOR": 91, "LAND": 92, "LXOR": 93, "EQ": 102, "FIRSTI": 115,
       "FIRSTJ": 117, "SECONDI": 119, "SECONDJ": 121}


class GrBError(RuntimeError):
    def __init__(self, info, what=""):
        super().__init__("%s failed: GrB_Info %d" % (what, info))
        self.info = info


class Matrix(ctypes.Structure):
    """grb_b200_matrix: a matrix as vectors (include/grb_b200.h)."""
    _fields_ = [("vlen", ctypes.c_int64), ("vdim", ctypes.c_int64),
                ("p", ctypes.POINTER(ctypes.c_int64)),
                ("i", ctypes.POINTER(ctypes.c_int64)),
                ("x", ctypes.c_void_p), ("type", ctypes.c_int),
                ("iso", ctypes.c_bool), ("jumbled", ctypes.c_bool),
                ("nzombies", ctypes.c_int64)]


class Semiring(ctypes.Structure):
    _fields_ = [("add_opcode", ctypes.c_int), ("mult_opcode", ctypes.c_int),
                ("type", ctypes.c_int)]


def semiring(add, mult, type_name):
    return Semiring(OPS[add], OPS[mult], TYPES[type_name])


_lib = None
_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def lib():
    """The native library (loaded once).  Raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("graphblas_b200 native library missing: %s "
                               "(run python -m graphblas_b200.build)" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, ci, cb = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_bool
        PM = ctypes.POINTER(Matrix)
        PS = ctypes.POINTER(Semiring)
        L.grb_b200_init.restype = ci
        L.grb_b200_finalize.restype = ci
        L.grb_b200_set_allocator.argtypes = [vp, vp]
        L.grb_b200_debug_fail_alloc.argtypes = [i64]
        L.grb_b200_AxB_dot3_branch.restype = cb
        L.grb_b200_AxB_dot3_branch.argtypes = [PM, PM, PM, PS, cb]
        L.grb_b200_AxB_dot3.argtypes = [PM, PM, cb, PM, PM, PS, cb]
        L.grb_b200_AxB_saxpy3.argtypes = [PM, PM, cb, cb, PM, PM, PS, cb,
                                          ctypes.POINTER(cb), ci]
        L.grb_b200_reduce_to_scalar.argtypes = [vp, PM, ci]
        L.grb_b200_dmatrix_upload.argtypes = [ctypes.POINTER(vp), i64, i64, vp,
                                              vp, vp, ci, cb]
        L.grb_b200_dmatrix_download.argtypes = [vp, ctypes.POINTER(vp),
                                                ctypes.POINTER(vp),
                                                ctypes.POINTER(vp), cb]
        L.grb_b200_dmatrix_free.argtypes = [ctypes.POINTER(vp)]
        L.grb_b200_dmatrix_info.argtypes = [vp] + [ctypes.POINTER(i64)] * 4 + [
            ctypes.POINTER(ci), ctypes.POINTER(cb)]
        L.grb_b200_dmxm_dot3.argtypes = [ctypes.POINTER(vp), vp, cb, vp, vp, PS]
        L.grb_b200_dmxm_saxpy3.argtypes = [ctypes.POINTER(vp), vp, cb, cb, vp,
                                           vp, PS]
        L.grb_b200_dreduce.argtypes = [vp, vp, ci]
        L.grb_b200_dwait.argtypes = [vp]
        for name in ("grb_b200_AxB_dot3", "grb_b200_AxB_saxpy3",
                     "grb_b200_reduce_to_scalar", "grb_b200_dmatrix_upload",
                     "grb_b200_dmatrix_download", "grb_b200_dmatrix_free",
                     "grb_b200_dmatrix_info", "grb_b200_dmxm_dot3",
                     "grb_b200_dmxm_saxpy3", "grb_b200_dreduce",
                     "grb_b200_dwait"):
            getattr(L, name).restype = ci
        _optional_bindings(L)
        _lib = L
    return _lib


def _optional_bindings(L):
    """Bindings of extension entry points (present in newer builds)."""
    vp, i64, ci, cb = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_bool
    if hasattr(L, "grb_b200_set_stream"):
        L.grb_b200_set_stream.argtypes = [vp]
    if hasattr(L, "grb_b200_stream_keep_scratch"):
        L.grb_b200_stream_keep_scratch.argtypes = [vp, cb]
        L.grb_b200_stream_keep_scratch.restype = ci
    if hasattr(L, "grb_b200_profile"):
        L.grb_b200_profile.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(i64)]
        L.grb_b200_profile.restype = ci
    if hasattr(L, "grb_b200_profile_reset"):
        L.grb_b200_profile_reset.argtypes = []
    if hasattr(L, "grb_b200_profile_enable"):
        L.grb_b200_profile_enable.argtypes = [cb]
    if hasattr(L, "grb_b200_profile_select"):
        L.grb_b200_profile_select.argtypes = [ctypes.c_char_p, ci]
        L.grb_b200_profile_select.restype = ci


def check(info, what=""):
    if info != SUCCESS:
        raise GrBError(info, what)
    return info


def init():
    return check(lib().grb_b200_init(), "grb_b200_init")


# ---------------------------------------------------------------------------
# drop-in entry points: host arrays in, host arrays out
# ---------------------------------------------------------------------------

class HostMatrix:
    """A grb_b200_matrix over numpy arrays (kept alive by this object)."""

    def __init__(self, vlen, vdim, p, i, x=None, type_code=None, iso=False,
                 jumbled=False):
        self.p = np.ascontiguousarray(p, dtype=np.int64)
        self.i = np.ascontiguousarray(i, dtype=np.int64)
        self.x = None if x is None else np.ascontiguousarray(x)
        if type_code is None:
            type_code = CODE_OF_NP[self.x.dtype] if self.x is not None else 1
        self.s = Matrix(vlen, vdim,
                        self.p.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                        self.i.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                        None if self.x is None else self.x.ctypes.data,
                        type_code, iso, jumbled, 0)

    @classmethod
    def from_csr(cls, csr, type_code=None):
        """A by-row matrix (vectors = rows)."""
        return cls(csr.ncols, csr.nrows, csr.p, csr.i, csr.x, type_code)


def _take_result(C):
    """Copy a callee-allocated grb_b200_matrix into numpy and free it."""
    nnz = C.p[C.vdim] if C.vdim >= 0 else 0
    p = np.ctypeslib.as_array(C.p, shape=(C.vdim + 1,)).copy()
    i = np.ctypeslib.as_array(C.i, shape=(max(nnz, 1),))[:nnz].copy()
    x = None
    if C.x:
        dt = NP_OF[C.type]
        n = 1 if C.iso else nnz
        buf = (ctypes.c_char * (max(n, 1) * np.dtype(dt).itemsize)).from_address(C.x)
        x = np.frombuffer(buf, dtype=dt)[:n].copy()
    _libc.free(ctypes.cast(C.p, ctypes.c_void_p))
    _libc.free(ctypes.cast(C.i, ctypes.c_void_p))
    if C.x:
        _libc.free(C.x)
    return p, i, x, int(C.nzombies)


def AxB_dot3(M, A, B, sr, mask_struct=True, flipxy=False):
    """Drop-in dot3 (reference orientation).  Returns (p, i, x, nzombies)."""
    C = Matrix()
    check(lib().grb_b200_AxB_dot3(ctypes.byref(C), ctypes.byref(M.s), mask_struct,
                                  ctypes.byref(A.s), ctypes.byref(B.s),
                                  ctypes.byref(sr), flipxy), "grb_b200_AxB_dot3")
    return _take_result(C)


def AxB_saxpy3(A, B, sr, M=None, mask_comp=False, mask_struct=True, flipxy=False):
    """Drop-in saxpy3 (reference orientation).  Returns (p, i, x, applied)."""
    C = Matrix()
    applied = ctypes.c_bool(False)
    check(lib().grb_b200_AxB_saxpy3(ctypes.byref(C),
                                    ctypes.byref(M.s) if M is not None else None,
                                    mask_comp, mask_struct, ctypes.byref(A.s),
                                    ctypes.byref(B.s), ctypes.byref(sr), flipxy,
                                    ctypes.byref(applied), 0),
          "grb_b200_AxB_saxpy3")
    p, i, x, _ = _take_result(C)
    return p, i, x, applied.value


def reduce_to_scalar(A, monoid, dtype):
    out = np.zeros(1, dtype=dtype)
    check(lib().grb_b200_reduce_to_scalar(out.ctypes.data, ctypes.byref(A.s),
                                          OPS[monoid]), "reduce_to_scalar")
    return out[0]


# ---------------------------------------------------------------------------
# device-resident matrices
# ---------------------------------------------------------------------------

class DMatrix:
    """A by-row matrix resident in HBM (grb_b200_dmatrix)."""

    def __init__(self, handle):
        self.h = ctypes.c_void_p(handle)

    @classmethod
    def upload(cls, csr, type_name=None, x=None):
        L = lib()
        xv = csr.x if x is None else x
        if type_name is None:
            tc = CODE_OF_NP[np.dtype(xv.dtype)] if xv is not None else 1
        else:
            tc = TYPES[type_name]
        p = np.ascontiguousarray(csr.p, dtype=np.int64)
        i = np.ascontiguousarray(csr.i, dtype=np.int64)
        h = ctypes.c_void_p()
        xp = None
        if xv is not None:
            xv = np.ascontiguousarray(xv, dtype=NP_OF[tc])
            xp = xv.ctypes.data
        check(L.grb_b200_dmatrix_upload(ctypes.byref(h), csr.nrows, csr.ncols,
                                        p.ctypes.data, i.ctypes.data, xp, tc,
                                        False), "dmatrix_upload")
        return cls(h.value)

    def info(self):
        v = [ctypes.c_int64() for _ in range(4)]
        t = ctypes.c_int()
        iso = ctypes.c_bool()
        check(lib().grb_b200_dmatrix_info(self.h, *[ctypes.byref(a) for a in v],
                                          ctypes.byref(t), ctypes.byref(iso)))
        return dict(nrows=v[0].value, ncols=v[1].value, nnz=v[2].value,
                    nzombies=v[3].value, type=t.value, iso=iso.value)

    def download(self, prune=True):
        L = lib()
        p, i, x = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        inf = self.info()
        check(L.grb_b200_dmatrix_download(self.h, ctypes.byref(p), ctypes.byref(i),
                                          ctypes.byref(x), prune), "download")
        m = inf["nrows"]
        pa = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_int64)),
                                   shape=(m + 1,)).copy()
        nnz = int(pa[m])
        ia = np.ctypeslib.as_array(ctypes.cast(i, ctypes.POINTER(ctypes.c_int64)),
                                   shape=(max(nnz, 1),))[:nnz].copy()
        xa = None
        if x.value:
            dt = np.dtype(NP_OF[inf["type"]])
            n = 1 if inf["iso"] else nnz
            buf = (ctypes.c_char * (max(n, 1) * dt.itemsize)).from_address(x.value)
            xa = np.frombuffer(buf, dtype=dt)[:n].copy()
            if inf["iso"]:
                xa = np.full(nnz, xa[0] if n else 0, dtype=dt)
            _libc.free(x)
        _libc.free(p)
        _libc.free(i)
        return pa, ia, xa

    def free(self):
        if self.h:
            lib().grb_b200_dmatrix_free(ctypes.byref(self.h))
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def dot3(M, A, B, sr, mask_struct=True):
    h = ctypes.c_void_p()
    check(lib().grb_b200_dmxm_dot3(ctypes.byref(h), M.h, mask_struct, A.h, B.h,
                                   ctypes.byref(sr)), "dmxm_dot3")
    return DMatrix(h.value)


def saxpy3(A, B, sr, M=None, mask_comp=False, mask_struct=True):
    h = ctypes.c_void_p()
    check(lib().grb_b200_dmxm_saxpy3(ctypes.byref(h), M.h if M is not None else None,
                                     mask_comp, mask_struct, A.h, B.h,
                                     ctypes.byref(sr)), "dmxm_saxpy3")
    return DMatrix(h.value)


def reduce(D, monoid, dtype):
    out = np.zeros(1, dtype=dtype)
    check(lib().grb_b200_dreduce(out.ctypes.data, D.h, OPS[monoid]), "dreduce")
    return out[0]
