"""Precision strategies (tensor-core BF16 / FP8-E4M3 scores, top-k, certified
re-score of the candidates) through the C ABI.

No reference counterpart: the reference's strategies are `direct` and the
binary32 `gemm` (include/ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp:17-23).
What is checked:
  * the tensor-core scores equal the binary64 dot products of the rounded
    rows and queries, within FP32 accumulation error;
  * with at least as many candidates as rows, the answer is the reference
    CPU argmin on every query (the re-score is certified);
  * with fewer candidates, the answer is the reference CPU argmin among the
    k rows with the smallest estimate ||r~||^2 - 2 r~.q~ (recomputed here from
    the engine's own scores), lowest row on ties;
  * errors: L1 indexes, candidate counts, non-finite queries.
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
DIST_RTOL = 1e-5


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even binary32 -> BF16, returned as binary32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32)


def fp8_round(x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Per-vector scale max|x| / 448 and the dequantized E4M3 values."""
    import torch
    x = np.ascontiguousarray(x, np.float32)
    amax = np.abs(x).max(axis=1)
    scale = np.where(amax > 0, amax / np.float32(448.0), np.float32(1.0)).astype(np.float32)
    y = (x / scale[:, None]).astype(np.float32)
    e = torch.from_numpy(y).to(torch.float8_e4m3fn).to(torch.float32).numpy()
    return (e * scale[:, None]).astype(np.float32), scale


def rounded(strategy, a: np.ndarray) -> np.ndarray:
    return bf16_round(a) if strategy == BF16 else fp8_round(a)[0]


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


@pytest.mark.parametrize("strategy", [BF16, FP8])
@pytest.mark.parametrize("r,d,n", [(300, 1000, 1), (300, 1000, 5), (129, 64, 17),
                                   (300, 1000, 40), (200, 2000, 100), (130, 700, 300)])
def test_scores_equal_rounded_dot_products(strategy, r, d, n):
    rng = np.random.default_rng(r + d + n)
    rows = rng.standard_normal((r, d)).astype(np.float32)
    queries = rng.standard_normal((n, d)).astype(np.float32)
    index = uha.CudaExactL2Index(rows)
    ws = index.make_query_workspace(n)
    scores, norms = index.precision_scores(queries, n, ws, strategy)
    rr = rounded(strategy, rows).astype(np.float64)
    qq = rounded(strategy, queries).astype(np.float64)
    exact = qq @ rr.T
    magnitude = np.abs(qq) @ np.abs(rr).T
    tol = (1e-5 if strategy == BF16 else 1e-4) * magnitude + 1e-30
    err = np.abs(scores.astype(np.float64) - exact)
    assert np.all(err <= tol), float((err / magnitude).max())
    assert np.allclose(norms, (rr * rr).sum(axis=1), rtol=1e-5)


@pytest.mark.parametrize("strategy", [BF16, FP8])
def test_all_rows_as_candidates_equal_reference_exact(strategy):
    rows, queries = golden_inputs()
    expected = golden("exact_l2")["indices"]
    index = uha.CudaExactL2Index(rows)
    for batch in (1, 7, 96):
        got, _ = run(index, queries, batch, strategy, candidates=64)
        assert np.array_equal(got, expected), f"batch {batch}"


@pytest.mark.parametrize("strategy", [BF16, FP8])
def test_flat_all_rows_as_candidates_equal_reference_flat(strategy):
    rows, queries = golden_inputs()
    g = golden("flat_l2_t32")
    index = uha.CudaSampledCoordinateL2AnnIndex(rows, g["probabilities"],
                                                int(g["repetitions"]),
                                                uha.MT19937_64(int(g["seed"])))
    for batch in (1, 96):
        got, _ = run(index, queries, batch, strategy, candidates=64)
        assert np.array_equal(got, g["indices"]), f"batch {batch}"


def _topk_from_scores(scores, norms, k):
    est = norms[None, :] - np.float32(2.0) * scores  # the engine's binary32 estimate
    out = []
    for e in est:
        order = np.lexsort((np.arange(e.size), e))
        out.append(np.sort(order[:k]))
    return out


@pytest.mark.parametrize("strategy", [BF16, FP8])
@pytest.mark.parametrize("k", [1, 8, 32])
def test_answer_is_reference_argmin_among_candidates(oracle_module, strategy, k):
    ds = synthetic.row_dataset(rows=700, classes=9, queries=60, d=2500, seed=3)
    index = uha.CudaExactL2Index(ds.rows)
    ws = index.make_query_workspace(60)
    scores, norms = index.precision_scores(ds.queries, 60, ws, strategy)
    got, dist = run(index, ds.queries, 60, strategy, candidates=k)
    for q, cand in enumerate(_topk_from_scores(scores, norms, k)):
        sub, sub_dist = oracle_module.exact("l2", ds.rows[cand], ds.queries[q:q + 1])
        assert got[q] == cand[int(sub[0])], q
        assert np.isclose(dist[q], sub_dist[0], rtol=DIST_RTOL, atol=1e-30)


@pytest.mark.parametrize("strategy", [BF16, FP8])
def test_agreement_with_exact_on_clustered_rows(oracle_module, strategy):
    ds = synthetic.row_dataset(rows=1500, classes=33, queries=200, d=4000, seed=11)
    expected, edist = oracle_module.exact("l2", ds.rows, ds.queries)
    index = uha.CudaExactL2Index(ds.rows)
    got, dist = run(index, ds.queries, 200, strategy, candidates=32)
    agreement = float(np.mean(got == expected))
    excess = (dist - edist) / edist
    assert np.all(excess >= -DIST_RTOL)
    assert agreement >= 0.95, agreement


def test_precision_errors():
    rows, queries = golden_inputs()
    l1 = uha.CudaExactL1Index(rows)
    ws1 = l1.make_query_workspace(2)
    # the L1 classes take no strategy (as in the reference); the C ABI refuses
    from ultrahigh_ann_b200.api import _CudaIndex
    with pytest.raises(uha.InvalidArgument):
        _CudaIndex.query_batch(l1, queries[:2], 2, None, ws1, BF16)
    index = uha.CudaExactL2Index(rows)
    ws = index.make_query_workspace(2)
    for bad in (0, 65):
        with pytest.raises(uha.InvalidArgument):
            ws.set_candidates(bad)
    q = queries[:2].copy()
    q[1, 5] = np.nan
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(q, 2, None, ws, FP8)
    # the workspace stays usable
    got = index.query_batch(queries[:2], 2, None, ws, BF16)
    assert np.array_equal(got, golden("exact_l2")["indices"][:2])
    hier = uha.CudaHierarchicalL1AnnIndex(rows, 32, 16, random_engine=uha.MT19937_64(3))
    wsh = hier.make_query_workspace(2)
    with pytest.raises(uha.InvalidArgument):
        _CudaIndex.query_batch(hier, queries[:2], 2, None, wsh, BF16)


@pytest.mark.parametrize("strategy", [BF16, FP8])
def test_query_many_pipeline_equals_per_batch_calls(strategy):
    """Calls of several batches overlap each batch's re-score with the next
    batch's scores (two candidate slots): the answers equal batch-by-batch
    calls, and a failing call leaves the workspace usable."""
    ds = synthetic.row_dataset(rows=700, classes=9, queries=50, d=2500, seed=6)
    index = uha.CudaExactL2Index(ds.rows)
    for batch in (1, 7, 16):
        ws = index.make_query_workspace(batch)
        ws.set_candidates(16)
        dist = np.zeros(50, np.float64)
        many = index.query_many(ds.queries, 50, batch, None, ws, strategy, dist)
        single, sdist = run(index, ds.queries, batch, strategy, candidates=16)
        assert np.array_equal(many, single), batch
        assert np.array_equal(dist, sdist), batch
    bad = ds.queries.copy()
    bad[23, 5] = np.inf
    ws = index.make_query_workspace(8)
    with pytest.raises(uha.InvalidArgument):
        index.query_many(bad, 50, 8, None, ws, strategy)
    again = index.query_many(ds.queries, 50, 8, None, ws, strategy)
    ref, _ = run(index, ds.queries, 8, strategy, candidates=32)
    assert np.array_equal(again, ref)
