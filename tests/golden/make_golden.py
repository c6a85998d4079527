"""Regenerate the golden fixtures in this folder from the reference library.

    python tests/golden/make_golden.py

Runs SuiteSparse:GraphBLAS itself (oracle/_ref, built from the reference's
own sources by oracle/ref.mk) through its public API, single-threaded, on
small seeded inputs, and stores inputs and outputs as .npz.  The tests pin
the oracle restatement against these files, so the pin holds on machines
without the reference sources.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import Reference, TYPE_CODES, NP_TYPES   # noqa: E402
from graphblas_b200 import workloads as W            # noqa: E402
from tests.helpers import random_csr                 # noqa: E402

CASES = [
    # name, add, mult, type, method, masked, comp, transpose_b(dot3)
    ("saxpy_plus_times_fp64", "PLUS", "TIMES", "fp64", 2, False, False, False),
    ("saxpy_plus_times_fp64_hash", "PLUS", "TIMES", "fp64", 3, False, False, False),
    ("saxpy_plus_times_fp32", "PLUS", "TIMES", "fp32", 2, False, False, False),
    ("saxpy_min_plus_fp32", "MIN", "PLUS", "fp32", 0, False, False, False),
    ("saxpy_min_plus_fp32_mask", "MIN", "PLUS", "fp32", 0, True, False, False),
    ("saxpy_min_plus_fp32_cmask", "MIN", "PLUS", "fp32", 0, True, True, False),
    ("saxpy_plus_pair_int64", "PLUS", "PAIR", "int64", 0, False, False, False),
    ("saxpy_any_secondi_int64_cmask", "ANY", "SECONDI", "int64", 2, True, True, False),
    ("saxpy_plus_times_int32", "PLUS", "TIMES", "int32", 0, False, False, False),
    ("saxpy_lor_land_bool", "LOR", "LAND", "bool", 0, False, False, False),
    ("dot3_plus_pair_int64", "PLUS", "PAIR", "int64", 1, True, False, True),
    ("dot3_plus_times_fp64", "PLUS", "TIMES", "fp64", 1, True, False, True),
    ("dot3_min_plus_fp32", "MIN", "PLUS", "fp32", 1, True, False, True),
    ("dot3_any_secondi_int64", "ANY", "SECONDI", "int64", 1, True, False, True),
]


def main():
    R = Reference(nthreads=1)
    out = {}
    for k, (name, add, mult, tname, method, masked, comp, tb) in enumerate(CASES):
        tc = TYPE_CODES[tname]
        np_t = NP_TYPES[tc]
        m, kk, n = 48, 40, 44
        A = random_csr(m, kk, 0.12, 100 + k, np_t, lo=0.5 if add == "MIN" else -1.0,
                       hi=4.0 if add == "MIN" else 1.0)
        if tb:
            B = random_csr(n, kk, 0.12, 200 + k, np_t, lo=0.5, hi=4.0)
        else:
            B = random_csr(kk, n, 0.12, 200 + k, np_t, lo=0.5, hi=4.0)
        M = random_csr(m, n, 0.3, 300 + k, np.bool_) if masked else None
        Cp, Ci, Cx = R.mxm(m, kk, n, (A.p, A.i, A.x, tc), (B.p, B.i, B.x, tc),
                           add, mult, tc,
                           M=None if M is None else (M.p, M.i, None, 1),
                           mask_comp=comp, transpose_b=tb, method=method)
        d = dict(m=m, k=kk, n=n, add=add, mult=mult, type=tc, masked=masked,
                 comp=comp, dot3=tb, Ap=A.p, Ai=A.i, Ax=A.x, Bp=B.p, Bi=B.i,
                 Bx=B.x, Cp=Cp, Ci=Ci, Cx=Cx)
        if M is not None:
            d.update(Mp=M.p, Mi=M.i)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        out[name] = int(Cp[-1])
    # triangle count and BFS parents on a small R-MAT graph
    S = W.rmat(9, 16, seed=77)
    L, U = W.tril_triu(S)
    ntri, _ = R.tricount(S.nrows, L.p, L.i, U.p, U.i)
    parent, _, nlev = R.bfs(S.nrows, S.p, S.i, 1)
    np.savez_compressed(os.path.join(HERE, "rmat9_tc_bfs.npz"), n=S.nrows,
                        Sp=S.p, Si=S.i, ntri=ntri, parent=parent, src=1,
                        nlevels=nlev)
    out["rmat9_tc"] = ntri
    print(out)


if __name__ == "__main__":
    main()
