"""Autotuned scan shapes and multi-index graph batches (uha_workspace_autotune,
uha_batch_*) through the C ABI.

No reference counterpart. What is checked: a tuned shape never changes an
answer (the certification bound follows the shape), and every pair of a
captured batch answers exactly as a query_batch of the same queries on its
index would, across graph replays with new queries.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, golden_inputs

pytestmark = pytest.mark.gpu

uha = pytest.importorskip("ultrahigh_ann_b200")
from ultrahigh_ann_b200 import synthetic  # noqa: E402

S = uha.QueryStrategy


def _individual(index, queries, strategy=S.direct, candidates=None):
    n = queries.shape[0]
    ws = index.make_query_workspace(n)
    if candidates is not None:
        ws.set_candidates(candidates)
    dist = np.zeros(n, np.float64)
    if isinstance(index, (uha.CudaDenseL1ScanIndex, uha.CudaHierarchicalL1AnnIndex)):
        out = index.query_batch(queries, n, None, ws, distances=dist)
    else:
        out = index.query_batch(queries, n, None, ws, strategy, dist)
    return out, dist


@pytest.mark.parametrize("batch", [1, 5, 8, 40, 96])
def test_autotune_keeps_reference_answers(batch):
    rows, queries = golden_inputs()
    q = queries[:batch]
    for cls, name in ((uha.CudaExactL2Index, "exact_l2"), (uha.CudaExactL1Index, "exact_l1")):
        index = cls(rows)
        ws = index.make_query_workspace(batch)
        rep = ws.autotune(batch)
        assert rep["candidates"] >= 1
        assert rep["best_ms"] <= rep["default_ms"]
        got = index.query_batch(q, batch, None, ws)
        assert np.array_equal(got, golden(name)["indices"][:batch]), (name, rep)
    g = golden("flat_l2_t32")
    flat = uha.CudaSampledCoordinateL2AnnIndex(rows, g["probabilities"], int(g["repetitions"]),
                                               uha.MT19937_64(int(g["seed"])))
    ws = flat.make_query_workspace(batch)
    for strategy in (S.direct, S.gemm_bf16_rerank):
        ws.autotune(batch, strategy)
        if strategy == S.gemm_bf16_rerank:
            ws.set_candidates(64)
        got = flat.query_batch(q, batch, None, ws, strategy)
        assert np.array_equal(got, g["indices"][:batch])


def test_autotuned_batch_sizes_match_reference(oracle_module):
    ds = synthetic.row_dataset(rows=300, classes=9, queries=40, d=3000, seed=4)
    expected, _ = oracle_module.exact("l2", ds.rows, ds.queries)
    index = uha.CudaExactL2Index(ds.rows)
    for batch in (1, 2, 4, 8, 16, 40):
        ws = index.make_query_workspace(batch)
        ws.autotune(batch)
        out = np.zeros(40, np.uint64)
        for s in range(0, 40, batch):
            e = min(40, s + batch)
            if e - s == batch:
                index.query_batch(ds.queries[s:e], batch, out[s:e], ws)
            else:
                out[s:e] = _individual(index, ds.queries[s:e])[0]
        assert np.array_equal(out, expected), batch


def _mixed_indexes():
    rows, _ = golden_inputs()
    ds = synthetic.row_dataset(rows=700, classes=9, queries=1, d=2500, seed=8)
    g8 = golden("flat_l2_t8")
    g1 = golden("flat_l1_t8")
    return [
        (uha.CudaExactL2Index(ds.rows), 37, S.direct),
        (uha.CudaExactL2Index(ds.rows), 64, S.gemm_bf16_rerank),
        (uha.CudaExactL1Index(rows), 5, S.direct),
        (uha.CudaSampledCoordinateL2AnnIndex(rows, g8["probabilities"], 8,
                                             uha.MT19937_64(int(g8["seed"]))), 96, S.direct),
        (uha.CudaSampledCoordinateL1AnnIndex(rows, g1["probabilities"], 8,
                                             uha.MT19937_64(int(g1["seed"]))), 1, S.direct),
        (uha.CudaHierarchicalL2AnnIndex(rows, 32, 16, uha.MT19937_64(3)), 19, S.direct),
        (uha.CudaHierarchicalL1AnnIndex(rows, 32, 15, uha.MT19937_64(4)), 23, S.direct),
        (uha.CudaExactL2Index(ds.rows[:1]), 3, S.direct),
    ]


@pytest.mark.parametrize("autotune", [False, True])
def test_batch_equals_individual_queries(autotune):
    pairs = _mixed_indexes()
    batch = uha.QueryBatch(pairs, autotune=autotune)
    rng = np.random.default_rng(2)
    for trial in range(2):
        queries = [np.abs(rng.standard_normal((c, ix.dimension))).astype(np.float32) * 3
                   for ix, c, _ in pairs]
        results = batch.run(queries)
        for (ix, c, strategy), q, (got, dist) in zip(pairs, queries, results):
            exp, edist = _individual(ix, q, strategy, 32)
            assert np.array_equal(got, exp), (type(ix).__name__, trial)
            assert np.allclose(dist, edist, rtol=1e-5, atol=1e-30), (type(ix).__name__, trial)
    st = batch.stats()
    assert st["pairs"] == len(pairs) and st["queries"] == sum(c for _, c, _ in pairs)
    assert st["graph_nodes"] > st["pairs"] and st["kernel_launches"] >= st["pairs"]
    assert st["device_ms"] > 0


def test_batch_reads_its_device_buffers():
    import torch
    rows, queries = golden_inputs()
    index = uha.CudaExactL2Index(rows)
    batch = uha.QueryBatch([(index, 96, S.direct)], autotune=False)
    assert batch.query_buffer(0) != 0 and batch.query_buffer(1) == 0
    src = torch.from_numpy(queries).cuda()
    torch.cuda.synchronize()
    (got, _), = batch.run([src.data_ptr()], on_device=True)
    assert np.array_equal(got, golden("exact_l2")["indices"])
    # the queries stay in the batch's buffer: a run without queries repeats it
    (again, _), = batch.run(None)
    assert np.array_equal(again, got)


def test_batch_rejects_bad_input():
    rows, queries = golden_inputs()
    index = uha.CudaExactL2Index(rows)
    with pytest.raises(uha.InvalidArgument):
        uha.QueryBatch([(index, 0, S.direct)])
    l1 = uha.CudaExactL1Index(rows)
    with pytest.raises(uha.InvalidArgument):
        uha.QueryBatch([(l1, 4, S.gemm_bf16_rerank)])
    batch = uha.QueryBatch([(index, 2, S.direct)], autotune=False)
    bad = queries[:2].copy()
    bad[0, 3] = np.inf
    with pytest.raises(uha.InvalidArgument):
        batch.run([bad])
    (got, _), = batch.run([queries[:2]])
    assert np.array_equal(got, golden("exact_l2")["indices"][:2])


@pytest.mark.parametrize("batch", [1, 3, 8, 64])
def test_autotune_median_passes_keeps_oracle_answers(oracle_module, batch):
    """The L1 hierarchy's median passes are tuned (sampled rows for the
    pruning threshold, queries per count CTA) on stand-in queries; every
    candidate shape gives the oracle's answers, and the tuned workspace
    answers as an untuned one."""
    ds = synthetic.row_dataset(rows=3000, classes=9, queries=64, d=2049, seed=12)
    probs = oracle_module.probabilities("l1", ds.rows)
    index = uha.CudaHierarchicalL1AnnIndex(ds.rows, 16, 64, uha.MT19937_64(5),
                                           importance_probabilities=probs)
    cs = index.coordinate_sample
    q = np.ascontiguousarray(ds.queries[:batch])
    expected, _ = oracle_module.hierarchical("l1", ds.rows, cs.source_columns,
                                             index.projection, q)
    ws = index.make_query_workspace(batch)
    rep = ws.autotune(batch)
    assert rep["kernel"] == "median"
    assert rep["candidates"] >= 3
    assert rep["best_ms"] <= rep["default_ms"]
    assert 32 <= rep["splits"] <= 1024  # sampled rows
    assert rep["queries_per_pass"] in (1, 2, 4, 8)
    tuned_dist = np.zeros(batch, np.float64)
    got = index.query_batch(q, batch, None, ws, distances=tuned_dist)
    assert np.array_equal(got, expected)
    want, want_dist = _individual(index, q)
    assert np.array_equal(got, want)
    assert np.allclose(tuned_dist, want_dist, rtol=1e-5, atol=1e-30)
    # a batch with autotune uses the tuned median shape in its graph and in
    # the persistent form (more than 8 queries)
    pair = [(index, batch)]
    for persistent in ((False, True) if batch > 8 else (False,)):
        b = uha.QueryBatch(pair, autotune=True, persistent=persistent)
        assert b.tuning(0)["kernel"] == "median"
        res = b.run([q])
        assert np.array_equal(res[0][0], expected)
