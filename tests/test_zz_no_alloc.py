"""uha_query_noalloc, the entry point that allocates nothing, against uha_query.

Some callers cannot call cudaMalloc while they answer queries: a server whose
device memory is reserved up front by its own pool allocator, code that must
not allocate while other threads capture CUDA graphs, embedded callers with a
fixed device footprint. uha_query_noalloc serves them from one static device
array instead of a workspace. This file is collected last so that, if it
fails, a run that stops at the first failure has already run every other test;
it also passes on its own in a fresh process, where its first call performs
the per-device set-up.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from ultrahigh_ann_b200 import _abi, synthetic

pytestmark = pytest.mark.gpu

DIST_RTOL = 1e-5  # the tolerance every distance comparison in the GPU tests uses


def noalloc_query(index, queries_dev, n, torch):
    out = torch.zeros(n, dtype=torch.int64, device="cuda")
    dist = torch.zeros(n, dtype=torch.float64, device="cuda")
    status = _abi.load().uha_query_noalloc(
        index._handle, ctypes.c_void_p(queries_dev.data_ptr()), n,
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(dist.data_ptr()), None)
    uha.api._check(status)
    return out.cpu().numpy().astype(np.uint64), dist.cpu().numpy()


def workspace_query(index, queries, n):
    ws = index.make_query_workspace(n)
    dist = np.zeros(n, np.float64)
    out = index.query_batch(queries, n, None, ws, distances=dist)
    return out, dist


@pytest.mark.parametrize("kind", ["exact_l2", "exact_l1", "weighted_l1", "flat_l2",
                                  "flat_l1"])
def test_noalloc_matches_workspace_query_on_two_calls(kind):
    torch = pytest.importorskip("torch")
    ds = synthetic.row_dataset(rows=700, classes=9, queries=16, d=6001, seed=4)
    if kind == "weighted_l1":
        # the dense L1 scan with per-coordinate binary32 weights
        weights = np.random.default_rng(5).uniform(0.25, 4.0, ds.rows.shape[1])
        index = uha.CudaDenseL1ScanIndex(ds.rows, weights.astype(np.float32))
    elif kind.startswith("exact"):
        cls = uha.CudaExactL2Index if kind == "exact_l2" else uha.CudaExactL1Index
        index = cls(ds.rows)
    else:
        metric = kind[-2:]
        fn = (uha.compute_l2_importance_probabilities_gpu if metric == "l2"
              else uha.compute_l1_importance_probabilities_gpu)
        cls = (uha.CudaSampledCoordinateL2AnnIndex if metric == "l2"
               else uha.CudaSampledCoordinateL1AnnIndex)
        index = cls(ds.rows, fn(ds.rows).probabilities, 32, uha.MT19937_64(3))
    # two calls in a row with different queries and batch sizes: the shared
    # scratch keeps the first call's contents and must not leak into the second
    for start, n in ((0, 8), (8, 5)):
        q = ds.queries[start:start + n]
        q_dev = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        got, got_dist = noalloc_query(index, q_dev, n, torch)
        expected, expected_dist = workspace_query(index, q, n)
        assert np.array_equal(got, expected)
        assert np.allclose(got_dist, expected_dist, rtol=DIST_RTOL, atol=0)


def test_noalloc_rejects_oversized_batches_and_non_finite_queries():
    torch = pytest.importorskip("torch")
    rows = np.random.default_rng(0).standard_normal((50, 100)).astype(np.float32)
    index = uha.CudaExactL2Index(rows)
    q = torch.zeros((9, 100), dtype=torch.float32, device="cuda")
    out = torch.zeros(9, dtype=torch.int64, device="cuda")
    lib = _abi.load()
    status = lib.uha_query_noalloc(index._handle, ctypes.c_void_p(q.data_ptr()), 9,
                                   ctypes.c_void_p(out.data_ptr()), None, None)
    assert status == _abi.LENGTH_ERROR
    q[0, 3] = float("nan")
    status = lib.uha_query_noalloc(index._handle, ctypes.c_void_p(q.data_ptr()), 2,
                                   ctypes.c_void_p(out.data_ptr()), None, None)
    assert status == _abi.INVALID_ARGUMENT
    # a later valid call is unaffected by the rejected ones
    q[0, 3] = 0.0
    got, _ = noalloc_query(index, q[:2].contiguous(), 2, torch)
    expected, _ = workspace_query(index, q[:2].cpu().numpy(), 2)
    assert np.array_equal(got, expected)
