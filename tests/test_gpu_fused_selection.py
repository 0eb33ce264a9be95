"""The fused candidate selection of the precision strategies (indexes of at
least 16,384 rows, plans of one K split): whole row tiles spread over the
index are scored as a sample, each query's k-th smallest sample estimate is
its threshold, and the
score kernel's epilogue keeps only the keys (estimate, row) at or below it; a
selection over those keys gives the candidates.

What is checked: the candidates are exactly the k smallest (estimate, row) of
the full score matrix (computed here from the engine's own tensor-core scores
and norms), so every answer is the reference CPU's argmin among them (the
oracle over the candidate rows); a list that overflows (thousands of rows tied
at the threshold) makes the engine answer the call again with the slab
selection, with the same answers; an L2 hierarchy on the precision strategy
through the fused path agrees with the oracle, alone and in a graph batch;
pipelined calls of several batches answer as batches called one at a time.
"""
from __future__ import annotations

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu

BF16 = uha.QueryStrategy.gemm_bf16_rerank
FP8 = uha.QueryStrategy.gemm_fp8_rerank
DIST_RTOL = 1e-5


def _topk_from_scores(scores, norms, k):
    # the engine's binary32 estimate: -2 S is exact, one rounding
    est = norms[None, :] - np.float32(2.0) * scores
    out = []
    for e in est:
        order = np.lexsort((np.arange(e.size), e))
        out.append(np.sort(order[:k]))
    return out


def _run(index, queries, batch, strategy, k):
    n = queries.shape[0]
    ws = index.make_query_workspace(batch)
    ws.set_candidates(k)
    out = np.zeros(n, np.uint64)
    dist = np.zeros(n, np.float64)
    for s in range(0, n, batch):
        e = min(n, s + batch)
        index.query_batch(queries[s:e], e - s, out[s:e], ws, strategy, dist[s:e])
    return out, dist


@pytest.mark.parametrize("strategy", [BF16, FP8])
@pytest.mark.parametrize("k", [1, 8, 32, 64])
def test_fused_candidates_are_the_slab_selection(oracle_module, strategy, k):
    ds = synthetic.row_dataset(rows=20000, classes=17, queries=48, d=96, seed=k)
    index = uha.CudaExactL2Index(ds.rows)
    ws = index.make_query_workspace(48)
    scores, norms = index.precision_scores(ds.queries, 48, ws, strategy)
    for batch in (1, 48):
        got, dist = _run(index, ds.queries, batch, strategy, k)
        for q, cand in enumerate(_topk_from_scores(scores, norms, k)):
            sub, sub_dist = oracle_module.exact("l2", ds.rows[cand], ds.queries[q:q + 1])
            assert got[q] == cand[int(sub[0])], (batch, q)
            assert np.isclose(dist[q], sub_dist[0], rtol=DIST_RTOL, atol=1e-30)


def test_overflowing_lists_are_answered_by_the_slab_selection(oracle_module):
    """Every row ties: every key passes the threshold, the lists overflow and
    the call is answered again by the slab path (lowest rows as candidates,
    row 0 the certified answer)."""
    rng = np.random.default_rng(5)
    row = rng.standard_normal(64).astype(np.float32)
    rows = np.tile(row, (20000, 1))
    queries = rng.standard_normal((12, 64)).astype(np.float32)
    index = uha.CudaExactL2Index(rows)
    for batch in (1, 12):
        got, _ = _run(index, queries, batch, BF16, 16)
        assert np.all(got == 0), batch
    # the workspace still takes the fused path afterwards
    ds = synthetic.row_dataset(rows=20000, classes=17, queries=8, d=96, seed=2)
    other = uha.CudaExactL2Index(ds.rows)
    ws = other.make_query_workspace(8)
    scores, norms = other.precision_scores(ds.queries, 8, ws, BF16)
    got, _ = _run(other, ds.queries, 8, BF16, 8)
    for q, cand in enumerate(_topk_from_scores(scores, norms, 8)):
        sub, _ = oracle_module.exact("l2", ds.rows[cand], ds.queries[q:q + 1])
        assert got[q] == cand[int(sub[0])]


def test_fused_hierarchy_agrees_with_oracle(oracle_module):
    ds = synthetic.row_dataset(rows=20000, classes=33, queries=96, d=3001, seed=9)
    probs = oracle_module.probabilities("l2", ds.rows[:1024])
    index = uha.CudaHierarchicalL2AnnIndex(ds.rows, 16, 64, uha.MT19937_64(4),
                                           importance_probabilities=probs)
    cs = index.coordinate_sample
    expected, _ = oracle_module.hierarchical("l2", ds.rows, cs.source_columns,
                                             index.projection, ds.queries)
    got, _ = _run(index, ds.queries, 96, BF16, 32)
    assert np.mean(got == expected) >= 0.97
    # the same pair in a graph batch (fused in the capture) answers the same
    batch = uha.QueryBatch([(index, 96, BF16)], autotune=True)
    res = batch.run([ds.queries])
    assert np.array_equal(res[0][0], got)


@pytest.mark.parametrize("strategy", [BF16, FP8])
def test_fused_selection_in_pipelined_calls(strategy):
    """One query_many call of several batches (the re-score of a batch runs on
    a second stream behind the next batch's scores) answers as the same
    batches answered one call at a time."""
    torch = pytest.importorskip("torch")
    ds = synthetic.row_dataset(rows=20000, classes=17, queries=192, d=96, seed=31)
    index = uha.CudaExactL2Index(ds.rows)
    want, want_dist = _run(index, ds.queries, 64, strategy, 16)
    ws = index.make_query_workspace(64)
    ws.set_candidates(16)
    qdev = torch.from_numpy(ds.queries).cuda()
    got = np.zeros(192, np.uint64)
    dist = np.zeros(192, np.float64)
    index.query_many(qdev.data_ptr(), 192, 64, got, ws, strategy, dist, on_device=True)
    assert np.array_equal(got, want)
    assert np.allclose(dist, want_dist, rtol=DIST_RTOL, atol=1e-30)
    host = index.query_many(ds.queries, 192, 64, None, ws, strategy)
    assert np.array_equal(host, want)
