"""grb_b200_dot3_noalloc: masked dot products for callers that cannot
allocate device memory (their GPU memory belongs to another allocator, or
they must not call cudaMalloc/cudaFree because those can synchronise the
device).  The entry point keeps its work queue in a fixed array inside the
library and writes only to the caller's buffers.

Checked here against the allocating entry point (grb_b200_dmxm_dot3) on two
calls in a row with different inputs, through the C-ABI, with the same rules
as the other parity tests: integer results bit-identical, floating results
bit-identical as well (both paths fold matches in ascending k).  Inputs and
outputs are allocated by the test with torch; the entry point allocates
nothing.  This file is collected last.
"""

import ctypes

import numpy as np
import pytest

from graphblas_b200 import workloads as W
from tests.helpers import random_csr

pytestmark = pytest.mark.gpu


def _bind(L):
    f = L.grb_b200_dot3_noalloc
    vp = ctypes.c_void_p
    f.argtypes = ([ctypes.c_int64] * 3 + [vp, vp, vp, vp, vp, ctypes.c_bool,
                                          vp, vp, vp, ctypes.c_bool, vp, vp, vp,
                                          ctypes.POINTER(ctypes.c_int64), vp])
    f.restype = ctypes.c_int
    return f


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _pool_used():
    """Bytes in use in the device's default memory pool (the pool the
    allocating entry points draw from) and the device's free memory."""
    import torch
    from cuda.bindings import driver as cu
    cu.cuInit(0)
    err, dev = cu.cuDeviceGet(torch.cuda.current_device())
    assert err == cu.CUresult.CUDA_SUCCESS
    err, pool = cu.cuDeviceGetDefaultMemPool(dev)
    assert err == cu.CUresult.CUDA_SUCCESS
    err, used = cu.cuMemPoolGetAttribute(
        pool, cu.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
    assert err == cu.CUresult.CUDA_SUCCESS
    return int(used), torch.cuda.mem_get_info()[0]


def _noalloc(gb, torch, M, A, B, sr, np_t, watch=False):
    """Run the no-alloc entry point on device copies of M, A, B.  With
    `watch`, the call itself is checked to leave the default memory pool's
    usage and the device's free memory as they were."""
    f = _bind(gb.lib())
    d = {k: _dev(torch, v, np.int32) for k, v in
         (("Mp", M.p), ("Mj", M.i), ("Ap", A.p), ("Aj", A.i), ("Bp", B.p), ("Bj", B.i))}
    Ax = _dev(torch, A.x, np_t) if A.x is not None else None
    Bx = _dev(torch, B.x, np_t) if B.x is not None else None
    mnz = int(M.p[-1])
    Cj = torch.empty(max(mnz, 1), dtype=torch.int32, device="cuda")
    Cx = torch.empty(max(mnz, 1), dtype=torch.from_numpy(np.zeros(1, np_t)).dtype,
                     device="cuda")
    nz = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    before = _pool_used() if watch else None
    info = f(M.nrows, M.ncols, mnz, d["Mp"].data_ptr(), d["Mj"].data_ptr(),
             d["Ap"].data_ptr(), d["Aj"].data_ptr(),
             Ax.data_ptr() if Ax is not None else None, False,
             d["Bp"].data_ptr(), d["Bj"].data_ptr(),
             Bx.data_ptr() if Bx is not None else None, False,
             ctypes.byref(sr), Cj.data_ptr(), Cx.data_ptr(), ctypes.byref(nz),
             stream)
    assert info == 0, "grb_b200_dot3_noalloc returned %d" % info
    if watch:
        assert _pool_used() == before, "the no-alloc call allocated device memory"
    return Cj[:mnz].cpu().numpy(), Cx[:mnz].cpu().numpy(), nz.value


def _allocating(gb, M, A, B, sr, type_name):
    dM = gb.DMatrix.upload(W.Csr(M.nrows, M.ncols, M.p, M.i), "bool")
    dA = gb.DMatrix.upload(A, type_name)
    dB = gb.DMatrix.upload(B, type_name)
    C = gb.dot3(dM, dA, dB, sr)
    p, i, x = C.download(prune=False)
    nz = C.info()["nzombies"]
    for h in (dM, dA, dB, C):
        h.free()
    return p, i, x, nz


def _check(got, want, M):
    Cj, Cx, nz = got
    p, i, x, nz_w = want
    assert np.array_equal(p, M.p)
    assert nz == nz_w
    assert np.array_equal(Cj.astype(np.int64), i)
    live = Cj >= 0
    assert np.array_equal(Cx[live].view(np.uint8).reshape(-1),
                          x[live].astype(Cx.dtype).view(np.uint8).reshape(-1))


def test_noalloc_matches_allocating_dot3_twice(gpu):
    import torch
    gb = gpu
    # call 1: triangle counting (plus_pair int64) on an R-MAT graph
    S = W.rmat(12, 16, seed=21)
    L, U = W.tril_triu(S)
    sr = gb.semiring("PLUS", "PAIR", "int64")
    got = _noalloc(gb, torch, L, L, U, sr, np.int64)
    want = _allocating(gb, L, L, U, sr, "bool")
    _check(got, want, L)
    assert int(got[1][got[0] >= 0].sum()) > 0
    # call 2, right after: plus_times fp64 with values, a different mask
    A = random_csr(300, 200, 0.05, 31, np.float64)
    B = random_csr(250, 200, 0.05, 32, np.float64)
    M = random_csr(300, 250, 0.1, 33, np.bool_)
    sr2 = gb.semiring("PLUS", "TIMES", "fp64")
    got2 = _noalloc(gb, torch, M, A, B, sr2, np.float64)
    want2 = _allocating(gb, M, A, B, sr2, "fp64")
    _check(got2, want2, M)
    # the same call once more, now that the library's module is loaded: it
    # draws nothing from the default pool and takes no device memory
    got3 = _noalloc(gb, torch, M, A, B, sr2, np.float64, watch=True)
    _check(got3, want2, M)


def test_noalloc_rejects_oversize_mask(gpu):
    import torch
    gb = gpu
    f = _bind(gb.lib())
    sr = gb.semiring("PLUS", "PAIR", "int64")
    t = torch.zeros(8, dtype=torch.int32, device="cuda")
    x = torch.zeros(8, dtype=torch.int64, device="cuda")
    nz = ctypes.c_int64(-1)
    too_big = 1048568 + 1
    info = f(1, 1, too_big, t.data_ptr(), t.data_ptr(), t.data_ptr(), t.data_ptr(),
             None, False, t.data_ptr(), t.data_ptr(), None, False, ctypes.byref(sr),
             t.data_ptr(), x.data_ptr(), ctypes.byref(nz), None)
    assert info == gb.INVALID_VALUE
    assert nz.value == -1
