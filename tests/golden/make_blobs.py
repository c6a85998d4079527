"""Regenerate tests/golden/blobs.npz: serialized-matrix blobs written by the
reference library itself.

    python tests/golden/make_blobs.py

Runs SuiteSparse:GraphBLAS (oracle/_ref, built from the reference's own
sources by oracle/ref.mk) through GxB_Matrix_serialize on small seeded
matrices, one blob per compression method (none, LZ4, LZ4HC, ZSTD at the
default and a high level) and storage form (hypersparse, sparse, bitmap,
full; by row or by column; iso), and stores each blob with the CSR matrix it
holds.  tests/test_serialize.py decodes them with the library's blob reader,
so the pin holds on machines without the reference sources.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import Reference, NP_TYPES   # noqa: E402

# name, type code, method, sparsity control, by column, iso, dense
CASES = [
    ("fp64_sparse_row_none", 11, -1, 2, False, False, False),
    ("fp64_hyper_col_lz4", 11, 1000, 1, True, False, False),
    ("int32_bitmap_row_lz4hc", 6, 2009, 4, False, False, False),
    ("uint64_full_col_none", 9, -1, 8, True, False, True),
    ("bool_sparse_row_zstd", 1, 0, 2, False, False, False),
    ("fp32_sparse_col_zstd19", 10, 3019, 2, True, False, False),
    ("int64_hyper_row_zstd", 8, 3000, 1, False, False, False),
    ("uint32_bitmap_col_zstd", 7, 3005, 4, True, False, False),
    ("fp64_iso_sparse_row_zstd", 11, 0, 2, False, True, False),
    ("int32_full_row_zstd", 6, 0, 8, False, False, True),
]


def values(t, k, rng):
    if t == 1:
        return rng.integers(0, 2, k).astype(np.bool_)
    if t in (10, 11):
        return rng.standard_normal(k).astype(NP_TYPES[t])
    if t == 7:
        return (np.arange(k) % 5).astype(np.uint32)            # repetitive runs
    if t == 9:
        return rng.integers(0, 2**63, k, dtype=np.uint64)
    return rng.integers(-1000, 1000, k).astype(NP_TYPES[t])


def main():
    R = Reference(nthreads=2)
    rng = np.random.default_rng(20260101)
    out = {}
    for name, t, method, sparsity, by_col, iso, dense in CASES:
        m, n = (24, 20) if dense else (60, 45)
        if dense:
            mask = np.ones((m, n), bool)
        else:
            mask = rng.random((m, n)) < 0.2
            mask[7, :] = False                                   # an empty row
            mask[:, 3] = False                                   # an empty column
        p = np.concatenate([[0], np.cumsum(mask.sum(1))]).astype(np.int64)
        i = np.nonzero(mask)[1].astype(np.int64)
        x = None if iso else values(t, len(i), rng)
        blob = R.serialize(t, m, n, p, i, x, sparsity, by_col, method)
        out[name + "__blob"] = np.frombuffer(blob, np.uint8)
        out[name + "__shape"] = np.array([m, n, t, int(iso)], np.int64)
        out[name + "__p"] = p
        out[name + "__i"] = i
        out[name + "__x"] = np.ones(len(i), NP_TYPES[t]) if iso else x
    np.savez_compressed(os.path.join(HERE, "blobs.npz"), **out)
    print("wrote %d blobs" % len(CASES))


if __name__ == "__main__":
    main()
