"""Precision strategies on the L2 hierarchy through the C ABI: the gathered
queries are projected on the tensor cores (BF16 or FP8-E4M3 GEMM of the
rounded p x k projection with the batch), the projected rows are scored by a
second tensor-core GEMM, and the k best candidates are re-scored by the
reference's binary64 projected distance (binary64 query projection in i
order, squared differences summed in j order).

No reference counterpart (the reference's hierarchy strategies are `direct`
and `gemm`). What is checked:
  * with at least as many candidates as rows, the answer and its distance are
    the reference CPU's (golden fixtures, and the direct path's distances);
  * with fewer candidates, every reported distance is the binary64 projected
    distance of the returned row, never below the minimum, and the answers
    agree with the exact argmin on clustered data;
  * batch-by-batch calls, query_many and a captured QueryBatch agree;
  * errors: non-finite sampled coordinates, L1 hierarchies.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, golden_inputs

pytestmark = pytest.mark.gpu

uha = pytest.importorskip("ultrahigh_ann_b200")
from ultrahigh_ann_b200 import synthetic  # noqa: E402

BF16 = uha.QueryStrategy.gemm_bf16_rerank
FP8 = uha.QueryStrategy.gemm_fp8_rerank


def run(index, queries, batch, strategy, candidates=32):
    n = queries.shape[0]
    ws = index.make_query_workspace(batch)
    ws.set_candidates(candidates)
    out = np.zeros(n, np.uint64)
    dist = np.zeros(n, np.float64)
    for s in range(0, n, batch):
        e = min(n, s + batch)
        index.query_batch(queries[s:e], e - s, out[s:e], ws, strategy, dist[s:e])
    return out, dist


def golden_index(name):
    rows, queries = golden_inputs()
    g = golden(name)
    index = uha.CudaHierarchicalL2AnnIndex(rows, int(g["repetitions"]),
                                           int(g["projection_dimension"]),
                                           uha.MT19937_64(int(g["seed"])),
                                           importance_probabilities=g["probabilities"])
    return index, queries, g


@pytest.mark.parametrize("strategy", [BF16, FP8])
@pytest.mark.parametrize("name", ["hier_l2_p16", "hier_l2_p15"])
def test_all_rows_as_candidates_equal_reference(strategy, name):
    index, queries, g = golden_index(name)
    _, want_dist = run(index, queries, 96, uha.QueryStrategy.direct)
    for batch in (1, 7, 96):
        got, dist = run(index, queries, batch, strategy, candidates=64)
        assert np.array_equal(got, g["indices"]), f"batch {batch}"
        assert np.array_equal(dist, want_dist), f"batch {batch}"


def _projected_distances(index, rows, queries, picked):
    cols = index.coordinate_sample.source_columns.astype(np.int64)
    P = np.asarray(index.projection, np.float64).reshape(-1, cols.size)
    reps = rows[:, cols].astype(np.float64) @ P.T
    y = queries[:, cols].astype(np.float64) @ P.T
    all_d = ((reps[None, :, :] - y[:, None, :]) ** 2).sum(axis=2)
    return all_d[np.arange(len(picked)), picked.astype(np.int64)], all_d.min(axis=1)


@pytest.mark.parametrize("strategy", [BF16, FP8])
@pytest.mark.parametrize("p,k", [(1, 4), (2, 8), (16, 1), (16, 8), (64, 32), (256, 8)])
def test_reported_distance_is_reference_distance_of_answer(oracle_module, strategy, p, k):
    ds = synthetic.row_dataset(rows=700, classes=9, queries=60, d=2500, seed=p + k)
    probs = oracle_module.probabilities("l2", ds.rows)
    index = uha.CudaHierarchicalL2AnnIndex(ds.rows, 16, p, uha.MT19937_64(p),
                                           importance_probabilities=probs)
    got, dist = run(index, ds.queries, 60, strategy, candidates=k)
    own, smallest = _projected_distances(index, ds.rows, ds.queries, got)
    assert np.allclose(dist, own, rtol=1e-10, atol=1e-30)
    assert np.all(dist >= smallest * (1 - 1e-10))
    if k == 32:
        expected, _ = oracle_module.hierarchical("l2", ds.rows,
                                                 index.coordinate_sample.source_columns,
                                                 index.projection, ds.queries)
        agreement = float(np.mean(got == expected))
        assert agreement >= (0.95 if strategy == BF16 else 0.9), agreement


@pytest.mark.parametrize("strategy", [BF16, FP8])
def test_query_many_and_captured_batch_equal_per_batch_calls(strategy):
    ds = synthetic.row_dataset(rows=500, classes=7, queries=40, d=3000, seed=21)
    index = uha.CudaHierarchicalL2AnnIndex(ds.rows, 16, 64, uha.MT19937_64(2))
    single, sdist = run(index, ds.queries, 8, strategy, candidates=16)
    ws = index.make_query_workspace(8)
    ws.set_candidates(16)
    dist = np.zeros(40, np.float64)
    many = index.query_many(ds.queries, 40, 8, None, ws, strategy, dist)
    assert np.array_equal(many, single) and np.array_equal(dist, sdist)
    whole, _ = run(index, ds.queries, 40, strategy, candidates=32)
    batch = uha.QueryBatch([(index, 40, strategy)], autotune=True)
    res = batch.run([ds.queries])
    assert np.array_equal(res[0][0], whole)


def test_hierarchical_precision_errors():
    rows, queries = golden_inputs()
    index, _, g = golden_index("hier_l2_p16")
    ws = index.make_query_workspace(4)
    bad = queries[:4].copy()
    bad[2, int(g["columns"][3])] = np.nan
    with pytest.raises(uha.InvalidArgument, match="sampled query coordinate"):
        index.query_batch(bad, 4, None, ws, BF16)
    # an unsampled non-finite coordinate is never read
    unsampled = np.setdiff1d(np.arange(rows.shape[1]), g["columns"])[0]
    ok = queries[:4].copy()
    ok[1, unsampled] = np.inf
    got = index.query_batch(ok, 4, None, ws, BF16)
    direct = index.query_batch(queries[:4], 4, None, ws)
    assert got.shape == direct.shape
