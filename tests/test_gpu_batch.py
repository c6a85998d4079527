"""Batched products (grb_b200_batch_*): every instance of a batch equals its
own product computed by the oracle (oracle/oracle.c), bit for bit, whether
the numeric phase runs eagerly, as a replayed CUDA graph, or after the
autotuner has changed the bin configuration."""

import os

import numpy as np
import pytest

from graphblas_b200 import workloads as W
from tests.helpers import assert_exact, random_csr

pytestmark = pytest.mark.gpu


def _check(oracle, mats, got, add, mult, tc, bmats=None):
    for k, a in enumerate(mats):
        b = a if bmats is None else bmats[k]
        want = oracle.saxpy(a.nrows, b.ncols, (a.p, a.i, a.x, tc), (b.p, b.i, b.x, tc),
                            add, mult, tc)
        assert_exact(got[k], want, "instance %d" % k)


def test_batch_min_plus_graph_and_eager(gpu, oracle, tmp_path, monkeypatch):
    from graphblas_b200.batch import Batch
    monkeypatch.setenv("GRB_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    mats = W.batch_min_plus(count=60, nmin=16, nmax=900, seed=5)
    B = Batch(mats, gpu.semiring("MIN", "PLUS", "fp32"))
    B.run(use_graph=False)
    eager = B.result()
    _check(oracle, mats, eager, "MIN", "PLUS", 10)
    B.run(use_graph=True)
    B.run(use_graph=True)                       # replay
    graph = B.result()
    for e, g in zip(eager, graph):
        assert_exact(g, e, "graph replay")
    ms = B.tune(use_cache=False)
    assert ms > 0 and os.path.exists(tmp_path / "tune.json")
    B.run(use_graph=True)
    _check(oracle, mats, B.result(), "MIN", "PLUS", 10)
    # a second batch of the same size class takes the cached configuration
    B2 = Batch(mats, gpu.semiring("MIN", "PLUS", "fp32"))
    B2.tune(use_cache=True)
    B2.run(use_graph=True)
    _check(oracle, mats, B2.result(), "MIN", "PLUS", 10)
    B.free()
    B2.free()


def test_batch_plus_times_distinct_operands(gpu, oracle):
    from graphblas_b200.batch import Batch
    rng = np.random.default_rng(3)
    amats, bmats = [], []
    for k in range(40):
        m, n, p = (int(v) for v in rng.integers(5, 300, 3))
        amats.append(random_csr(m, n, 0.05, 100 + k))
        bmats.append(random_csr(n, p, 0.05, 200 + k))
    B = Batch(amats, gpu.semiring("PLUS", "TIMES", "fp64"), bmats=bmats)
    B.run(use_graph=True)
    _check(oracle, amats, B.result(), "PLUS", "TIMES", 11, bmats=bmats)
    B.free()


def test_batch_heavy_rows_and_empty_instances(gpu, oracle):
    """Instances whose rows exceed every shared-memory bin (dense accumulator)
    next to empty instances."""
    from graphblas_b200.batch import Batch
    S = W.rmat(9, 16, seed=2)
    rng = np.random.default_rng(4)
    heavy = W.Csr(S.nrows, S.ncols, S.p, S.i, (0.5 + rng.random(S.nnz)).astype(np.float32))
    empty = W.Csr(7, 7, np.zeros(8, np.int64), np.zeros(0, np.int64), np.zeros(0, np.float32))
    mats = [empty, heavy, W.poisson_minw(300, seed=9), empty]
    B = Batch(mats, gpu.semiring("MIN", "PLUS", "fp32"))
    B.run(use_graph=True)
    _check(oracle, mats, B.result(), "MIN", "PLUS", 10)
    B.free()
