"""The fused single-launch query of flat (and small exact) indexes at batches of
at most 8 queries: gather, scan and certified argmin in one kernel with many
CTAs per query (the last CTA of a query merges and replays near-ties in
binary64). Indices must equal the reference CPU's (the oracle: binary64 scan,
strict <, lowest row on ties) on every query, for every lane width the plan
picks (8, 16 and 32 lanes per row), for L2, L1 and weighted L1, on planted
ties, across consecutive calls that reuse the workspace scratch, with host
and device queries; the query's non-finite sampled values fail the call.
"""
from __future__ import annotations

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu

DIST_RTOL = 1e-5


def run(index, queries, batch):
    queries = np.ascontiguousarray(queries, np.float32).reshape(-1, index.dimension)
    ws = index.make_query_workspace(batch)
    out = np.zeros(queries.shape[0], np.uint64)
    dist = np.zeros(queries.shape[0], np.float64)
    for s in range(0, queries.shape[0], batch):
        e = min(queries.shape[0], s + batch)
        index.query_batch(queries[s:e], e - s, out[s:e], ws, distances=dist[s:e])
    return out, dist


def flat_index(metric, rows, probs, reps, seed):
    cls = (uha.CudaSampledCoordinateL2AnnIndex if metric == "l2"
           else uha.CudaSampledCoordinateL1AnnIndex)
    return cls(rows, probs, reps, uha.MT19937_64(seed))


@pytest.mark.parametrize("metric", ["l2", "l1"])
@pytest.mark.parametrize("reps", [4, 16, 64])
def test_fused_flat_matches_oracle_all_small_batches(oracle_module, metric, reps):
    ds = synthetic.row_dataset(rows=5000, classes=33, queries=40, d=9001, seed=reps)
    probs = oracle_module.probabilities(metric, ds.rows)
    index = flat_index(metric, ds.rows, probs, reps, reps + 1)
    cs = index.coordinate_sample
    expected, edist = oracle_module.flat(metric, ds.rows, cs.source_columns,
                                         cs.multiplicities, cs.inverse_probabilities,
                                         ds.queries)
    for batch in (1, 2, 3, 5, 8):
        got, dist = run(index, ds.queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"
        assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)


@pytest.mark.parametrize("metric", ["l2", "l1"])
@pytest.mark.parametrize("dim", [7, 100, 300, 1000, 8190])
def test_fused_exact_small_dimension_matches_oracle(oracle_module, metric, dim):
    # exact indexes of at most 8192 padded columns (the smaller ones also fit
    # the one-CTA kernel, which now serves only batches above 8)
    rng = np.random.default_rng(dim)
    rows = rng.standard_normal((6000, dim)).astype(np.float32)
    queries = rng.standard_normal((24, dim)).astype(np.float32)
    expected, edist = oracle_module.exact(metric, rows, queries)
    cls = uha.CudaExactL2Index if metric == "l2" else uha.CudaExactL1Index
    index = cls(rows)
    for batch in (1, 4, 8):
        got, dist = run(index, queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"
        assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)


def test_fused_weighted_l1_matches_oracle(oracle_module):
    rng = np.random.default_rng(3)
    rows = rng.standard_normal((9000, 700)).astype(np.float32)
    weights = rng.uniform(0.1, 3.0, 700).astype(np.float32)
    queries = rng.standard_normal((16, 700)).astype(np.float32)
    expected, _ = oracle_module.weighted_l1(rows, weights, queries)
    index = uha.CudaDenseL1ScanIndex(rows, weights)
    for batch in (1, 8):
        got, _ = run(index, queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_fused_planted_ties_take_the_lowest_row(oracle_module, metric):
    rng = np.random.default_rng(8)
    rows = rng.standard_normal((7000, 520)).astype(np.float32)
    # exact duplicates and one-ulp neighbours of row 123 in other CTAs' blocks
    for r in (900, 4000, 6999):
        rows[r] = rows[123]
    rows[5000] = rows[123]
    rows[5000, 17] = np.nextafter(rows[5000, 17], np.float32(np.inf))
    queries = np.vstack([rows[123], rows[5000], 0.5 * (rows[123] + rows[5000]),
                         rng.standard_normal((5, 520))]).astype(np.float32)
    expected, _ = oracle_module.exact(metric, rows, queries)
    cls = uha.CudaExactL2Index if metric == "l2" else uha.CudaExactL1Index
    index = cls(rows)
    ws = index.make_query_workspace(1)
    got = np.zeros(queries.shape[0], np.uint64)
    for i in range(queries.shape[0]):
        index.query_batch(queries[i], 1, got[i:i + 1], ws)
    assert np.array_equal(got, expected)
    assert got[0] == 123


def test_fused_many_calls_device_and_host_queries(oracle_module):
    """query_many at batch 1 over device queries (consecutive fused launches)
    and host queries agree with the oracle; the workspace scratch stays
    consistent across calls."""
    torch = pytest.importorskip("torch")
    ds = synthetic.row_dataset(rows=7028, classes=33, queries=300, d=6007, seed=5)
    probs = oracle_module.probabilities("l2", ds.rows)
    index = flat_index("l2", ds.rows, probs, 32, 7)
    cs = index.coordinate_sample
    expected, _ = oracle_module.flat("l2", ds.rows, cs.source_columns, cs.multiplicities,
                                     cs.inverse_probabilities, ds.queries)
    qdev = torch.from_numpy(ds.queries).cuda()
    for batch in (1, 3, 8):
        ws = index.make_query_workspace(batch)
        for _ in range(2):
            out = np.zeros(300, np.uint64)
            index.query_many(qdev.data_ptr(), 300, batch, out, ws, on_device=True)
            assert np.array_equal(out, expected), batch
            assert ws.last_stats()["kernel_launches"] == -(-300 // batch)
        host = index.query_many(ds.queries, 300, batch, None, ws)
        assert np.array_equal(host, expected)


def test_fused_non_finite_sampled_value_fails_and_recovers():
    ds = synthetic.row_dataset(rows=6000, classes=9, queries=4, d=3001, seed=2)
    probs = uha.compute_l2_importance_probabilities_gpu(ds.rows).probabilities
    index = flat_index("l2", ds.rows, probs, 32, 1)
    col = int(index.coordinate_sample.source_columns[0])
    q = ds.queries.copy()
    q[1, col] = np.nan
    ws = index.make_query_workspace(4)
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(q, 4, None, ws)
    # an unsampled non-finite value is never read
    unsampled = np.setdiff1d(np.arange(ds.rows.shape[1]),
                             index.coordinate_sample.source_columns)[0]
    q = ds.queries.copy()
    q[2, unsampled] = np.inf
    good = index.query_batch(ds.queries, 4, None, ws)
    assert np.array_equal(index.query_batch(q, 4, None, ws), good)
