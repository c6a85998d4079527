"""The drop-in entry points (grb_b200_AxB_dot3 / _saxpy3 / _reduce_to_scalar)
take matrices in the reference's internal orientation: a matrix is a set of
vectors (CSC columns inside SuiteSparse:GraphBLAS).  These tests check that
orientation, the operand order of non-commutative and positional multipliers,
the zombie contract of dot3 (C keeps M's pattern, empty dot products hold
-(i)-2, C->nzombies counts them; Source/mxm/GB_AxB_dot3.c:172-197), and
mask handling of saxpy3, against a direct dense evaluation of the definitions
(C(i,j) = sum_k A(i,k) (x) B(k,j) with FIRSTI = i, FIRSTJ = k, SECONDI = k,
SECONDJ = j; Include/GraphBLAS.h positional operators).
"""

import numpy as np
import pytest

from tests.helpers import random_csr

pytestmark = pytest.mark.gpu


def _dense_vectors(vlen, vdim, p, i, x):
    """vectors -> dense (vlen x vdim) array D with D[idx, vec] = value, and a
    presence mask."""
    D = np.zeros((vlen, vdim), dtype=np.float64 if x is None else x.dtype)
    P = np.zeros((vlen, vdim), dtype=bool)
    for v in range(vdim):
        for q in range(p[v], p[v + 1]):
            D[i[q], v] = 1 if x is None else x[q]
            P[i[q], v] = True
    return D, P


def _mult(op, a, b, i, k, j):
    return {"TIMES": a * b, "PLUS": a + b, "FIRST": a, "SECOND": b, "PAIR": 1,
            "MINUS": a - b, "FIRSTI": i, "FIRSTJ": k, "SECONDI": k,
            "SECONDJ": j, "MIN": min(a, b)}[op]


def _add(op, z, t):
    return {"PLUS": z + t, "MIN": min(z, t), "MAX": max(z, t)}[op]


@pytest.mark.parametrize("add,mult,tname", [
    ("PLUS", "TIMES", "fp64"), ("PLUS", "FIRST", "fp64"),
    ("PLUS", "SECOND", "fp64"), ("MIN", "PLUS", "fp64"),
    ("MIN", "FIRSTJ", "int64"), ("MIN", "SECONDI", "int64"),
    ("MAX", "SECONDI", "int64"), ("PLUS", "PAIR", "int64"),
])
def test_dropin_dot3_orientation(gpu, add, mult, tname):
    gb = gpu
    np_t = np.float64 if tname == "fp64" else np.int64
    vlen, na, nb = 40, 30, 25
    # A: vlen x na (vectors = columns), B: vlen x nb, M: na x nb
    A = random_csr(na, vlen, 0.3, 1, np_t)     # its rows are A's vectors
    B = random_csr(nb, vlen, 0.3, 2, np_t)
    M = random_csr(nb, na, 0.4, 3, np.bool_)   # vector j of M: entries i
    hA = gb.HostMatrix(vlen, na, A.p, A.i, A.x)
    hB = gb.HostMatrix(vlen, nb, B.p, B.i, B.x)
    hM = gb.HostMatrix(na, nb, M.p, M.i, None, type_code=1)
    p, i, x, nz = gb.AxB_dot3(hM, hA, hB, gb.semiring(add, mult, tname))
    assert np.array_equal(p, M.p)                   # C keeps M's pattern
    Ad, Ap_ = _dense_vectors(vlen, na, A.p, A.i, A.x)
    Bd, Bp_ = _dense_vectors(vlen, nb, B.p, B.i, B.x)
    zombies = 0
    for j in range(nb):
        for q in range(M.p[j], M.p[j + 1]):
            ii = M.i[q]
            # C(ii,j) = A(:,ii)' * B(:,j): terms k where both present, ascending
            ks = np.nonzero(Ap_[:, ii] & Bp_[:, j])[0]
            if len(ks) == 0:
                assert i[q] == -ii - 2
                zombies += 1
                continue
            assert i[q] == ii
            z = None
            for k in ks:
                t = _mult(mult, Ad[k, ii], Bd[k, j], ii, k, j)
                z = t if z is None else _add(add, z, t)
            assert x[q] == pytest.approx(z, rel=1e-12, abs=0)
    assert nz == zombies


@pytest.mark.parametrize("add,mult,tname", [
    ("PLUS", "TIMES", "fp64"), ("PLUS", "FIRST", "fp64"),
    ("PLUS", "SECOND", "fp64"), ("MIN", "FIRSTI", "int64"),
    ("MIN", "SECONDJ", "int64"), ("MAX", "SECONDI", "int64"),
])
@pytest.mark.parametrize("masked,comp", [(False, False), (True, False), (True, True)])
def test_dropin_saxpy3_orientation(gpu, add, mult, tname, masked, comp):
    gb = gpu
    np_t = np.float64 if tname == "fp64" else np.int64
    m, kk, n = 30, 35, 28
    # C = A*B with A m x kk and B kk x n, every matrix stored as columns
    A = random_csr(kk, m, 0.25, 5, np_t)       # vectors of A (columns)
    B = random_csr(n, kk, 0.25, 6, np_t)       # vectors of B
    Mc = random_csr(n, m, 0.3, 7, np.bool_)
    hA = gb.HostMatrix(m, kk, A.p, A.i, A.x)
    hB = gb.HostMatrix(kk, n, B.p, B.i, B.x)
    hM = gb.HostMatrix(m, n, Mc.p, Mc.i, None, type_code=1) if masked else None
    p, i, x, applied = gb.AxB_saxpy3(hA, hB, gb.semiring(add, mult, tname), M=hM,
                                     mask_comp=comp)
    assert applied == masked
    Ad, Ap_ = _dense_vectors(m, kk, A.p, A.i, A.x)
    Bd, Bp_ = _dense_vectors(kk, n, B.p, B.i, B.x)
    Md, Mp_ = _dense_vectors(m, n, Mc.p, Mc.i, None)
    for j in range(n):
        want = {}
        for k in np.nonzero(Bp_[:, j])[0]:
            for ii in np.nonzero(Ap_[:, k])[0]:
                if masked and (Mp_[ii, j] == comp):
                    continue
                t = _mult(mult, Ad[ii, k], Bd[k, j], ii, k, j)
                want[ii] = t if ii not in want else _add(add, want[ii], t)
        got_i = i[p[j]:p[j + 1]]
        assert list(got_i) == sorted(want)
        for q, ii in enumerate(got_i):
            assert x[p[j] + q] == pytest.approx(want[ii], rel=1e-12, abs=0)


def test_dropin_reduce_skips_zombies(gpu):
    gb = gpu
    p = np.array([0, 2, 4], np.int64)
    i = np.array([0, -3, 1, -2], np.int64)        # two zombies
    x = np.array([5, 100, 7, 100], np.int64)
    h = gb.HostMatrix(3, 2, p, i, x)
    assert gb.reduce_to_scalar(h, "PLUS", np.int64) == 12


def test_dropin_declines_unsupported(gpu):
    gb = gpu
    A = random_csr(10, 10, 0.3, 1)
    hA = gb.HostMatrix(10, 10, A.p, A.i, A.x)
    # a semiring outside the compiled list is declined with GrB_NO_VALUE
    with pytest.raises(gb.GrBError) as e:
        gb.AxB_saxpy3(hA, hA, gb.semiring("TIMES", "MINUS", "fp64"))
    assert e.value.info == gb.NO_VALUE
