"""Parity of the hierarchical indexes (binary32 projection + L2 scan or
median-|diff| scan, certified, binary64 replay) with the reference CPU
HierarchicalL{2,1}AnnIndex, through the C ABI on the GPU.

Expectations follow tests/hnsvw25/l2/hierarchical/
cuda_hierarchical_l2_ann_index_test.cpp and its L1 sibling, held to
bit-exact indices against the reference CPU on every query.
"""
from __future__ import annotations

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from conftest import engine_state, golden, golden_inputs
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu

DIST_RTOL = 1e-5
BATCHES = (1, 2, 3, 5, 8, 9, 64, 96)
CLASSES = {"l2": uha.CudaHierarchicalL2AnnIndex, "l1": uha.CudaHierarchicalL1AnnIndex}


def run(index, queries, batch):
    queries = np.ascontiguousarray(queries, np.float32).reshape(-1, index.dimension)
    ws = index.make_query_workspace(batch)
    out = np.zeros(queries.shape[0], np.uint64)
    dist = np.zeros(queries.shape[0], np.float64)
    for s in range(0, queries.shape[0], batch):
        e = min(queries.shape[0], s + batch)
        index.query_batch(queries[s:e], e - s, out[s:e], ws, distances=dist[s:e])
    return out, dist


@pytest.mark.parametrize("name", ["hier_l2_p16", "hier_l2_p15", "hier_l1_p16",
                                  "hier_l1_p15"])
def test_hierarchical_golden_all_batches(name):
    rows, queries = golden_inputs()
    g = golden(name)
    metric = name[5:7]
    rng = uha.MT19937_64(int(g["seed"]))
    index = CLASSES[metric](rows, int(g["repetitions"]), int(g["projection_dimension"]),
                            rng, importance_probabilities=g["probabilities"])
    # the same randomness as the reference constructor, consumed identically
    assert np.array_equal(index.coordinate_sample.source_columns, g["columns"])
    assert np.array_equal(index.projection, g["projection"])
    assert rng.state() == engine_state(g["engine_state_after"])
    for batch in BATCHES:
        got, _ = run(index, queries, batch)
        assert np.array_equal(got, g["indices"]), f"batch {batch}"


@pytest.mark.parametrize("metric", ["l2", "l1"])
@pytest.mark.parametrize("p", [1, 2, 7, 16, 33, 64, 256])
def test_hierarchical_random_parity(oracle_module, metric, p):
    ds = synthetic.row_dataset(rows=211, classes=6, queries=70, d=2500, seed=p)
    probs = oracle_module.probabilities(metric, ds.rows)
    index = CLASSES[metric](ds.rows, 8, p, uha.MT19937_64(p + 5),
                            importance_probabilities=probs)
    s = index.coordinate_sample
    expected, edist = oracle_module.hierarchical(metric, ds.rows, s.source_columns,
                                                 index.projection, ds.queries)
    for batch in (1, 8, 70):
        got, dist = run(index, ds.queries, batch)
        assert np.array_equal(got, expected), batch
        assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_hierarchical_duplicate_rows_take_the_lowest_index(oracle_module, metric):
    rng = np.random.default_rng(11)
    rows = rng.standard_normal((40, 300)).astype(np.float32)
    rows[25] = rows[7]
    rows[31] = rows[7]
    queries = np.vstack([rows[7], rows[7] + 1e-3, rng.standard_normal((6, 300))]
                        ).astype(np.float32)
    sample = uha.CoordinateSample(np.arange(0, 300, 3), np.ones(100, np.uint64),
                                  np.full(100, 3.0))
    index = CLASSES[metric](rows, None, 12, uha.MT19937_64(4),
                            coordinate_sample=sample)
    expected, _ = oracle_module.hierarchical(metric, rows, sample.source_columns,
                                             index.projection, queries)
    got, _ = run(index, queries, queries.shape[0])
    assert np.array_equal(got, expected)
    assert got[0] == 7


def test_hierarchical_l2_reference_fixture(oracle_module):
    rows = np.array([[0.0, 99.0, 0.0, -5.0], [4.0, -99.0, 1.0, -5.0],
                     [2.0, 0.0, 5.0, -5.0]], np.float32)
    probs = np.array([1.0, 0.0, 1.0, 0.0])
    index = uha.CudaHierarchicalL2AnnIndex(rows, 1, 7, uha.MT19937_64(1729),
                                           importance_probabilities=probs)
    ws = index.make_query_workspace(4)
    usage = index.space_usage()
    assert usage.index_payload_bytes == 3 * 7 * 4 + 3 * 4 + 2 * 24 + 7 * 2 * 4
    assert usage.query_workspace_payload_bytes == 0
    assert usage.unique_query_coordinates == 2 and usage.sampled_multiplicity == 2
    assert ws.payload_bytes() == (2 * (4 * 2 * 4) + 2 * (4 * 7 * 4) + 4 +
                                  4 * 3 * 4 + 4 * 4 + 4 * 8)
    queries = np.array([0.2, 10.0, 0.1, 20.0, 3.9, -10.0, 1.1, 20.0,
                        2.1, 10.0, 4.8, 20.0, 1.0, -10.0, 2.0, 20.0], np.float32)
    expected, _ = oracle_module.hierarchical(
        "l2", rows, index.coordinate_sample.source_columns, index.projection, queries)
    assert np.array_equal(index.query_batch(queries, 4, None, ws), expected)
    assert np.array_equal(index.query_batch(queries, 4, None, ws, uha.QueryStrategy.gemm),
                          expected)
    # unsampled non-finite values are ignored; sampled ones are rejected
    unsampled = np.array([0.2, np.nan, 0.1, np.inf], np.float32)
    assert index.query(unsampled, ws) == expected[0]
    assert index.query(unsampled, ws, uha.QueryStrategy.gemm) == expected[0]
    with pytest.raises(uha.InvalidArgument):
        index.query(np.array([np.nan, 0.0, 0.25, 0.0], np.float32), ws)
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(np.zeros(20, np.float32), 5, None, ws)
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(np.zeros(7, np.float32), 2, None, ws)
    other = uha.CudaHierarchicalL2AnnIndex(rows, 1, 7, uha.MT19937_64(1729),
                                           importance_probabilities=probs)
    with pytest.raises(uha.InvalidArgument):
        other.query(queries[:4], ws)


def test_hierarchical_l1_space_formulas():
    rows = np.array([[0.0, 1.0], [3.0, 4.0]], np.float32)
    index = uha.CudaHierarchicalL1AnnIndex(
        rows, None, 5, uha.MT19937_64(3),
        coordinate_sample=uha.CoordinateSample([1], [1], [1.0]))
    ws = index.make_query_workspace(4)
    assert index.space_usage().index_payload_bytes == 24 + 5 * 4 + 2 * 5 * 4
    assert ws.payload_bytes() == (2 * (4 * 4) + 4 * 5 * 4 + 4 + 4 * 2 * 4 + 4 * 8 + 4)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_hierarchical_wide_fixture_returns_own_rows(metric):
    d, r, p = 513, 4, 31
    col = np.arange(d)
    rows = np.stack([2.0 * row + 0.01 * ((col % 7) - 3) for row in range(r)]).astype(
        np.float32)
    sample = uha.CoordinateSample(col, np.ones(d, np.uint64), np.ones(d))
    index = CLASSES[metric](rows, None, p, uha.MT19937_64(1729),
                            coordinate_sample=sample)
    ws = index.make_query_workspace(r)
    assert list(index.query_batch(rows, r, None, ws)) == list(range(r))
    if metric == "l2":
        assert list(index.query_batch(rows, r, None, ws, uha.QueryStrategy.gemm)) == \
            list(range(r))


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_hierarchical_edge_cases(metric):
    cls = CLASSES[metric]
    rows = np.array([[1.0, 2.0, 3.0]], np.float32)
    one = cls(rows, None, 4, uha.MT19937_64(1),
              coordinate_sample=uha.CoordinateSample([0], [1], [1.0]))
    ws = one.make_query_workspace(2)
    # a one-row hierarchy answers row 0 without reading the query
    nan_q = np.full(6, np.nan, np.float32)
    assert list(one.query_batch(nan_q, 2, None, ws)) == [0, 0]
    two = np.array([[1.0, 2.0, 3.0], [2.0, 2.0, 2.0]], np.float32)
    with pytest.raises(uha.InvalidArgument):
        cls(two, None, 0, uha.MT19937_64(1),
            coordinate_sample=uha.CoordinateSample([0], [1], [1.0]))
    with pytest.raises(uha.CudaRuntimeError):
        cls(two, None, 3, uha.MT19937_64(1), coordinate_sample=uha.CoordinateSample())


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_hierarchical_near_ties_match_reference(oracle_module, metric):
    """Groups of six rows equal up to relative 1e-6 noise: their projected
    distances differ far below the binary32 bounds, so most queries take the
    binary64 replay (and, for L1, the per-pair median bounds must not
    exclude the reference's row)."""
    rng = np.random.default_rng(3)
    base = (np.abs(rng.standard_normal((20, 500))) * 10).astype(np.float32)
    rows = np.repeat(base, 6, axis=0)
    rows = (rows * (1 + 1e-6 * rng.standard_normal(rows.shape))).astype(np.float32)
    queries = (base[:12] + 0.05 * rng.standard_normal((12, 500))).astype(np.float32)
    sample = uha.CoordinateSample(np.arange(0, 500, 2), np.ones(250, np.uint64),
                                  np.full(250, 2.0))
    for p in (16, 64, 255):
        index = CLASSES[metric](rows, None, p, uha.MT19937_64(p),
                                coordinate_sample=sample)
        expected, edist = oracle_module.hierarchical(metric, rows, sample.source_columns,
                                                     index.projection, queries)
        for batch in (1, 12):
            got, dist = run(index, queries, batch)
            assert np.array_equal(got, expected), (p, batch)
            assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)


@pytest.mark.parametrize("p", [1, 16, 64, 256])
def test_gaussian_jl_hierarchy_matches_oracle(oracle_module, p):
    """The seeded Gaussian JL mode (not in the reference) runs the same
    certified path as the Rademacher one: its answers are the binary64
    projected argmin of the oracle given the same matrix, on every query and
    with every strategy, lowest row on ties."""
    ds = synthetic.row_dataset(rows=300, classes=6, queries=70, d=2500, seed=p + 40)
    probs = oracle_module.probabilities("l2", ds.rows)
    index = uha.CudaHierarchicalL2AnnIndex(ds.rows, 16, p, uha.MT19937_64(p),
                                           importance_probabilities=probs,
                                           projection="gaussian")
    assert index.projection_kind == "gaussian"
    cs = index.coordinate_sample
    expected, edist = oracle_module.hierarchical("l2", ds.rows, cs.source_columns,
                                                 index.projection, ds.queries)
    for batch in (1, 8, 70):
        got, dist = run(index, ds.queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"
        assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)
    ws = index.make_query_workspace(70)
    ws.set_candidates(64)
    got = index.query_batch(ds.queries, 70, None, ws, uha.QueryStrategy.gemm_bf16_rerank)
    # with 64 candidates per query every near row is re-scored in binary64
    assert np.mean(got == expected) >= 0.98
