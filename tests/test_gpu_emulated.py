"""Certification without the FP64 units.

* The emulated replay (QueryWorkspace.set_replay(True)) of the certified path
  on exact and flat indexes: float-float distances of the candidates, then
  emulated binary64 for the candidates they cannot separate. Answers must
  equal the reference CPU (the oracle) on every query -- the small, fused and
  scan+argmin kernels, L2, L1 and weighted L1 -- including exact duplicates
  (which only the emulated binary64 can order) and one-ulp neighbours.
* The FP32 re-score strategies (gemm_bf16_rerank_fp32, gemm_fp8_rerank_fp32):
  binary32 re-score of the tensor-core candidates with a certified bound,
  near-ties settled the same way. With every row a candidate the answers are
  the oracle's; on larger indexes they equal the binary64 re-score's.
"""
from __future__ import annotations

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu

DIST_RTOL = 1e-5
S = uha.QueryStrategy


def run(index, queries, batch, emulated=True, strategy=S.direct, candidates=None):
    queries = np.ascontiguousarray(queries, np.float32).reshape(-1, index.dimension)
    ws = index.make_query_workspace(batch)
    ws.set_replay(emulated)
    if candidates is not None:
        ws.set_candidates(candidates)
    out = np.zeros(queries.shape[0], np.uint64)
    dist = np.zeros(queries.shape[0], np.float64)
    replayed = 0
    for s in range(0, queries.shape[0], batch):
        e = min(queries.shape[0], s + batch)
        index.query_batch(queries[s:e], e - s, out[s:e], ws, strategy, distances=dist[s:e])
        replayed += ws.last_stats()["replayed_queries"]
    return out, dist, replayed


def tied_rows(rng, r, d, anchor=5):
    rows = rng.standard_normal((r, d)).astype(np.float32)
    for k in (r // 3, r // 2, r - 1):
        rows[k] = rows[anchor]
    rows[r // 4] = rows[anchor]
    rows[r // 4, 3] = np.nextafter(rows[r // 4, 3], np.float32(np.inf))
    queries = np.vstack([rows[anchor], rows[r // 4], 0.5 * (rows[anchor] + rows[r // 4]),
                         rng.standard_normal((9, d))]).astype(np.float32)
    return rows, queries


@pytest.mark.parametrize("metric", ["l2", "l1"])
@pytest.mark.parametrize("shape", [(40, 300), (5000, 700), (300, 20000)])
def test_emulated_replay_exact_matches_oracle(oracle_module, metric, shape):
    # (40, 300): fused flat kernel at batch <= 8, one-CTA kernel above;
    # (5000, 700): fused flat kernel at batch <= 8, scan + argmin above;
    # (300, 20000): scan + argmin
    r, d = shape
    rows, queries = tied_rows(np.random.default_rng(r + d), r, d)
    expected, edist = oracle_module.exact(metric, rows, queries)
    cls = uha.CudaExactL2Index if metric == "l2" else uha.CudaExactL1Index
    index = cls(rows)
    for batch in (1, 5, 12):
        got, dist, replayed = run(index, queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"
        assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)
        # query 0 ties with exact duplicates of its row: no binary32 bound
        # separates them, so it is always replayed (the one-ulp neighbour is
        # separable in binary32 and need not be)
        assert replayed >= 1
        assert got[0] == 5


def test_emulated_replay_weighted_l1_matches_oracle(oracle_module):
    rng = np.random.default_rng(12)
    rows, queries = tied_rows(rng, 3000, 513)
    weights = rng.uniform(0.1, 5.0, 513).astype(np.float32)
    expected, _ = oracle_module.weighted_l1(rows, weights, queries)
    index = uha.CudaDenseL1ScanIndex(rows, weights)
    for batch in (1, 12):
        got, _, _ = run(index, queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_emulated_replay_flat_matches_oracle(oracle_module, metric):
    ds = synthetic.row_dataset(rows=3000, classes=33, queries=48, d=5003, seed=31)
    rows = ds.rows.copy()
    rows[2999] = rows[7]
    queries = np.vstack([rows[7], ds.queries]).astype(np.float32)
    probs = oracle_module.probabilities(metric, rows)
    cls = (uha.CudaSampledCoordinateL2AnnIndex if metric == "l2"
           else uha.CudaSampledCoordinateL1AnnIndex)
    index = cls(rows, probs, 32, uha.MT19937_64(2))
    cs = index.coordinate_sample
    expected, edist = oracle_module.flat(metric, rows, cs.source_columns, cs.multiplicities,
                                         cs.inverse_probabilities, queries)
    for batch in (1, 8, 49):
        got, dist, _ = run(index, queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"
        assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)
    # the binary64 replay gives the same rows
    got64, _, _ = run(index, queries, 8, emulated=False)
    assert np.array_equal(got64, expected)


@pytest.mark.parametrize("strategy", [S.gemm_bf16_rerank_fp32, S.gemm_fp8_rerank_fp32])
def test_fp32_rescore_with_all_rows_as_candidates_matches_oracle(oracle_module, strategy):
    rng = np.random.default_rng(int(strategy))
    rows, queries = tied_rows(rng, 60, 2001)
    expected, edist = oracle_module.exact("l2", rows, queries)
    index = uha.CudaExactL2Index(rows)
    for batch in (1, 12):
        got, dist, _ = run(index, queries, batch, strategy=strategy, candidates=64)
        assert np.array_equal(got, expected), f"batch {batch}"
        assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)


@pytest.mark.parametrize("fp32, fp64", [(S.gemm_bf16_rerank_fp32, S.gemm_bf16_rerank),
                                        (S.gemm_fp8_rerank_fp32, S.gemm_fp8_rerank)])
def test_fp32_rescore_equals_binary64_rescore(oracle_module, fp32, fp64):
    """Same tensor-core candidates, so the same answer whenever the reference
    row is among them, and both are certified against the reference CPU."""
    ds = synthetic.row_dataset(rows=2000, classes=33, queries=96, d=12001, seed=17)
    index = uha.CudaExactL2Index(ds.rows)
    expected, _ = oracle_module.exact("l2", ds.rows, ds.queries)
    for batch in (1, 32, 96):
        a, da, _ = run(index, ds.queries, batch, strategy=fp32, candidates=32)
        b, db, _ = run(index, ds.queries, batch, strategy=fp64, candidates=32)
        assert np.array_equal(a, b), f"batch {batch}"
        assert np.allclose(da, db, rtol=DIST_RTOL, atol=0)
        assert np.mean(a == expected) >= 0.97


def test_fp32_rescore_flat_index(oracle_module):
    ds = synthetic.row_dataset(rows=1500, classes=33, queries=40, d=9001, seed=2)
    probs = oracle_module.probabilities("l2", ds.rows)
    index = uha.CudaSampledCoordinateL2AnnIndex(ds.rows, probs, 32, uha.MT19937_64(3))
    cs = index.coordinate_sample
    expected, _ = oracle_module.flat("l2", ds.rows, cs.source_columns, cs.multiplicities,
                                     cs.inverse_probabilities, ds.queries)
    got, _, _ = run(index, ds.queries, 40, strategy=S.gemm_bf16_rerank_fp32, candidates=64)
    assert np.mean(got == expected) >= 0.97
    b, _, _ = run(index, ds.queries, 40, strategy=S.gemm_bf16_rerank, candidates=64)
    assert np.array_equal(got, b)


def test_fp32_rescore_rejects_hierarchies():
    ds = synthetic.row_dataset(rows=100, classes=4, queries=2, d=500, seed=1)
    index = uha.CudaHierarchicalL2AnnIndex(ds.rows, 8, 16, uha.MT19937_64(1),
                                           importance_probabilities=np.full(500, 0.5))
    ws = index.make_query_workspace(2)
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(ds.queries, 2, None, ws, S.gemm_bf16_rerank_fp32)
