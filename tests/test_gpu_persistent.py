"""The persistent multi-index batch (uha_batch_create_persistent): three
cooperative kernel launches per run (gather and projection, tile scans and
median samples, late stages) that drain every pair's stages (gather,
projection, L2 tile scan or median sample / count / survivor, certified
argmin with replay, reported distances) from a device work queue, each unit
waiting only for its own pair's earlier stages.

Each unit runs the device code of the standalone kernel it replaces, so every
pair must answer exactly as query_batch of the same queries does (indices,
and distances within the tests' 1e-5 relative), which is the reference CPU's
hierarchical argmin (checked against the oracle), across runs with new
queries; the run is three kernel launches; pairs without a persistent form are
rejected; a non-finite sampled query value fails the run and the next run
answers normally; the stage clock reports every stage.
"""
from __future__ import annotations

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu

DIST_RTOL = 1e-5
CLASSES = {"l2": uha.CudaHierarchicalL2AnnIndex, "l1": uha.CudaHierarchicalL1AnnIndex}


def _alone(index, queries):
    n = queries.shape[0]
    ws = index.make_query_workspace(n)
    dist = np.zeros(n, np.float64)
    out = index.query_batch(queries, n, None, ws, distances=dist)
    return out, dist


@pytest.fixture(scope="module")
def pairs(oracle_module):
    ds = synthetic.row_dataset(rows=3000, classes=33, queries=700, d=4099, seed=6)
    specs = [("l2", 3000, 16, 64, 300), ("l1", 2000, 16, 15, 257), ("l2", 700, 32, 256, 96),
             ("l1", 3000, 32, 64, 5), ("l2", 1500, 8, 1, 17), ("l1", 700, 8, 256, 64),
             ("l1", 1024, 16, 2, 1), ("l2", 3000, 32, 33, 129)]
    probs = {m: oracle_module.probabilities(m, ds.rows) for m in ("l2", "l1")}
    out = []
    for i, (metric, r, reps, p, n) in enumerate(specs):
        ix = CLASSES[metric](ds.rows[:r], reps, p, uha.MT19937_64(40 + i),
                             importance_probabilities=probs[metric])
        out.append((metric, r, ix, n))
    return ds, out


def test_persistent_batch_equals_query_batch_and_oracle(oracle_module, pairs):
    ds, items = pairs
    batch = uha.QueryBatch([(ix, n) for _, _, ix, n in items], autotune=True, persistent=True)
    assert batch.persistent
    rng = np.random.default_rng(3)
    for run in range(3):
        queries = []
        for _, _, ix, n in items:
            pick = rng.choice(ds.queries.shape[0], n, replace=False)
            queries.append(np.ascontiguousarray(ds.queries[pick]))
        res = batch.run(queries)
        st = batch.stats()
        assert st["kernel_launches"] == 3
        stages = batch.stage_ms()
        assert len(stages) == 8 and all(t >= 0 for t in stages)
        assert sum(stages) <= st["device_ms"] * 1.5 + 1.0
        for (metric, r, ix, n), q, (got, dist) in zip(items, queries, res):
            want, wdist = _alone(ix, q)
            assert np.array_equal(got, want), (metric, r, ix.projection.shape, run)
            assert np.allclose(dist, wdist, rtol=DIST_RTOL, atol=1e-30)
            if run == 0:
                cs = ix.coordinate_sample
                expected, _ = oracle_module.hierarchical(metric, ds.rows[:r], cs.source_columns,
                                                         ix.projection, q)
                assert np.array_equal(got, expected)


def test_persistent_batch_equals_graph_batch(pairs):
    ds, items = pairs
    work = [(ix, n) for _, _, ix, n in items]
    queries = [np.ascontiguousarray(ds.queries[:n]) for _, _, _, n in items]
    a = uha.QueryBatch(work, autotune=False, persistent=True).run(queries)
    b = uha.QueryBatch(work, autotune=False).run(queries)
    for (ra, da), (rb, db) in zip(a, b):
        assert np.array_equal(ra, rb)
        assert np.allclose(da, db, rtol=DIST_RTOL, atol=1e-30)


def test_persistent_batch_rejects_pairs_without_a_persistent_form(pairs):
    ds, items = pairs
    exact = uha.CudaExactL2Index(ds.rows[:500])
    with pytest.raises(uha.InvalidArgument):
        uha.QueryBatch([(items[0][2], 16), (exact, 16)], persistent=True)
    # an L2 hierarchy with at most 8 queries uses the streaming scan
    with pytest.raises(uha.InvalidArgument):
        uha.QueryBatch([(items[0][2], 8)], persistent=True)
    with pytest.raises(uha.InvalidArgument):
        uha.QueryBatch([(items[0][2], 16, uha.QueryStrategy.gemm_bf16_rerank)],
                       persistent=True)


def test_persistent_batch_non_finite_query_fails_and_recovers(pairs):
    ds, items = pairs
    metric, r, ix, _ = items[1]
    batch = uha.QueryBatch([(ix, 32), (items[0][2], 32)], autotune=False, persistent=True)
    q0 = np.ascontiguousarray(ds.queries[:32]).copy()
    q1 = np.ascontiguousarray(ds.queries[32:64])
    q0[4, int(ix.coordinate_sample.source_columns[0])] = np.nan
    with pytest.raises(uha.InvalidArgument):
        batch.run([q0, q1])
    q0 = np.ascontiguousarray(ds.queries[:32])
    res = batch.run([q0, q1])
    assert np.array_equal(res[0][0], _alone(ix, q0)[0])
    assert np.array_equal(res[1][0], _alone(items[0][2], q1)[0])
