"""Parity of the engine's exact and flat (sampled-coordinate) scans with the
reference CPU implementation, through the C ABI on the GPU.

Expectations follow the reference's own CUDA tests
(tests/exact/l2/cuda_exact_l2_index_test.cpp, tests/exact/l1/
cuda_exact_l1_index_test.cpp, tests/coordinate_sampling/
cuda_sampled_coordinate_l{1,2}_ann_index_test.cpp), except that the `direct`
strategy is held to the stronger bar of bit-exact indices against the
reference CPU binary64 scan on every query (the oracle), including planted
near-ties. Distances are compared within 1e-5 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from conftest import golden, golden_inputs
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu

DIST_RTOL = 1e-5
BATCHES = (1, 2, 3, 5, 8, 9, 64, 96)

FIX_ROWS = np.array([[0.0, 0.0], [5.0, 0.0], [2.0, 4.0]], np.float32)
FIX_QUERIES = np.array([1.0, 0.0, 3.0, 3.0, 2.5, 0.0, 5.0, 0.0], np.float32)


def run(index, queries, batch, strategy=uha.QueryStrategy.direct):
    queries = np.ascontiguousarray(queries, np.float32).reshape(-1, index.dimension)
    ws = index.make_query_workspace(batch)
    out = np.zeros(queries.shape[0], np.uint64)
    dist = np.zeros(queries.shape[0], np.float64)
    for s in range(0, queries.shape[0], batch):
        e = min(queries.shape[0], s + batch)
        index.query_batch(queries[s:e], e - s, out[s:e], ws, strategy,
                          distances=dist[s:e])
    return out, dist


def test_runtime_info_reports_b200():
    info = uha.cuda_runtime_info(0)
    assert info is not None
    assert info.compute_capability_major == 10
    assert info.device_name
    assert uha.cuda_available()


def test_exact_l2_reference_fixture(oracle_module):
    index = uha.CudaExactL2Index(FIX_ROWS)
    scan = uha.CudaDenseL2ScanIndex(FIX_ROWS)
    ws = index.make_query_workspace(4)
    assert index.device() == 0 and index.device_name()
    assert ws.maximum_batch_size() == 4
    assert index.space_usage().index_payload_bytes == 6 * 4 + 3 * 4
    assert ws.payload_bytes() == 4 * 2 * 4 + 4 * 3 * 4 + 4 * 4 + 4 * 8
    expected, _ = oracle_module.exact("l2", FIX_ROWS, FIX_QUERIES)
    direct = index.query_batch(FIX_QUERIES, 4, None, ws)
    assert np.array_equal(direct, expected) and direct[2] == 0
    gemm = index.query_batch(FIX_QUERIES, 4, None, ws, uha.QueryStrategy.gemm)
    assert np.array_equal(gemm, expected) and gemm[2] == 0
    sws = scan.make_query_workspace(4)
    assert np.array_equal(scan.query_batch(FIX_QUERIES, 4, None, sws), direct)
    assert index.query(FIX_QUERIES[:2], ws) == 0


def test_exact_l2_cancellation_fixture():
    base = np.float32(1048576.0)
    rows = np.array([[base + np.float32(0.25)], [base + np.float32(0.125)]], np.float32)
    scan = uha.CudaDenseL2ScanIndex(rows)
    ws = scan.make_query_workspace(1)
    q = np.array([base], np.float32)
    assert scan.query_batch(q, 1, None, ws, uha.QueryStrategy.direct)[0] == 1
    # the norm-identity strategy keeps the reference's unrefined binary32 answer
    assert scan.query_batch(q, 1, None, ws, uha.QueryStrategy.gemm)[0] == 0


def test_exact_l2_errors():
    index = uha.CudaExactL2Index(FIX_ROWS)
    ws = index.make_query_workspace(4)
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(np.zeros(10, np.float32), 5, None, ws)
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(np.zeros(3, np.float32), 2, None, ws)
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(FIX_QUERIES, 4, np.zeros(1, np.uint64), ws)
    with pytest.raises(uha.InvalidArgument):
        index.query(np.array([np.nan, 0.0], np.float32), ws)
    other = uha.CudaExactL2Index(FIX_ROWS)
    with pytest.raises(uha.InvalidArgument):
        other.query(FIX_QUERIES[:2], ws)
    with pytest.raises(uha.InvalidArgument):
        uha.CudaExactL2Index(np.array([[np.inf, 0.0]], np.float32))
    with pytest.raises(uha.InvalidArgument):
        uha.CudaExactL2Index(np.zeros((0, 3), np.float32))
    with pytest.raises(uha.InvalidArgument):
        index.make_query_workspace(0)
    # the workspace stays usable after a rejected query
    assert np.array_equal(index.query_batch(FIX_QUERIES, 4, None, ws),
                          np.array([0, 2, 0, 1], np.uint64))


def test_exact_l1_reference_fixture(oracle_module):
    index = uha.CudaExactL1Index(FIX_ROWS)
    ws = index.make_query_workspace(4)
    assert index.space_usage().index_payload_bytes == 6 * 4
    assert ws.payload_bytes() == 4 * 2 * 4 + 4 * 3 * 4 + 4 * 8
    expected, _ = oracle_module.exact("l1", FIX_ROWS, FIX_QUERIES)
    got = index.query_batch(FIX_QUERIES, 4, None, ws)
    assert np.array_equal(got, expected) and got[2] == 0
    weights = np.array([2.0, 0.5], np.float32)
    weighted = uha.CudaDenseL1ScanIndex(FIX_ROWS, weights)
    assert weighted.space_usage().index_payload_bytes == 6 * 4 + 2 * 4
    wws = weighted.make_query_workspace(4)
    expected_w, _ = oracle_module.weighted_l1(FIX_ROWS, weights, FIX_QUERIES)
    assert np.array_equal(weighted.query_batch(FIX_QUERIES, 4, None, wws), expected_w)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_exact_golden_all_batches(metric):
    rows, queries = golden_inputs()
    expected = golden(f"exact_{metric}")["indices"]
    cls = uha.CudaExactL2Index if metric == "l2" else uha.CudaExactL1Index
    index = cls(rows)
    for batch in BATCHES:
        got, _ = run(index, queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"


@pytest.mark.parametrize("metric", ["l2", "l1"])
@pytest.mark.parametrize("shape", [(1, 5), (7, 1), (33, 1003), (130, 4099), (257, 64)])
def test_exact_random_parity(oracle_module, metric, shape):
    r, d = shape
    rng = np.random.default_rng(r * 7 + d)
    rows = rng.standard_normal((r, d)).astype(np.float32)
    queries = rng.standard_normal((40, d)).astype(np.float32)
    expected, edist = oracle_module.exact(metric, rows, queries)
    cls = uha.CudaExactL2Index if metric == "l2" else uha.CudaExactL1Index
    index = cls(rows)
    for batch in (1, 8, 40):
        got, dist = run(index, queries, batch)
        assert np.array_equal(got, expected), f"batch {batch}"
        assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_exact_planted_ties_take_replay_path(oracle_module, metric):
    rng = np.random.default_rng(5)
    base = rng.standard_normal((20, 300)).astype(np.float32)
    # duplicates and one-ulp neighbours of row 4, scattered at higher indices
    rows = base.copy()
    rows[11] = rows[4]
    rows[17] = rows[4]
    rows[19] = rows[4]
    rows[19, 7] = np.nextafter(rows[19, 7], np.float32(np.inf))
    queries = np.vstack([rows[4], rows[19], 0.5 * (rows[4] + rows[19]),
                         rng.standard_normal((5, 300))]).astype(np.float32)
    expected, _ = oracle_module.exact(metric, rows, queries)
    cls = uha.CudaExactL2Index if metric == "l2" else uha.CudaExactL1Index
    index = cls(rows)
    ws = index.make_query_workspace(queries.shape[0])
    got = index.query_batch(queries, queries.shape[0], None, ws)
    assert np.array_equal(got, expected)
    assert got[0] == 4
    assert ws.last_stats()["replayed_queries"] >= 1


SAMPLE = uha.CoordinateSample([0, 2], [2, 1], [0.5, 4.0])
SAMPLED_ROWS = np.array([[0.0, 99.0, 0.0, -5.0], [4.0, -99.0, 1.0, -5.0],
                         [2.0, 0.0, 5.0, -5.0]], np.float32)
SAMPLED_QUERIES = np.array([0.5, 10.0, 0.25, 20.0, 3.8, -10.0, 1.1, 20.0,
                            2.0, 10.0, 0.5, 20.0, 2.0, -10.0, 5.0, 20.0], np.float32)


def test_sampled_l2_reference_fixture(oracle_module):
    index = uha.CudaSampledCoordinateL2AnnIndex(SAMPLED_ROWS, coordinate_sample=SAMPLE)
    ws = index.make_query_workspace(4)
    usage = index.space_usage()
    assert usage.index_payload_bytes == 3 * 2 * 4 + 3 * 4 + 2 * 8 + 2 * 4
    assert usage.unique_query_coordinates == 2 and usage.sampled_multiplicity == 3
    assert ws.payload_bytes() == 2 * (4 * 2 * 4) + 4 * 3 * 4 + 4 * 4 + 4 * 8
    expected, _ = oracle_module.flat("l2", SAMPLED_ROWS, SAMPLE.source_columns,
                                     SAMPLE.multiplicities,
                                     SAMPLE.inverse_probabilities, SAMPLED_QUERIES)
    direct = index.query_batch(SAMPLED_QUERIES, 4, None, ws)
    gemm = index.query_batch(SAMPLED_QUERIES, 4, None, ws, uha.QueryStrategy.gemm)
    assert np.array_equal(direct, expected) and np.array_equal(gemm, expected)
    assert direct[2] == 0 and gemm[2] == 0
    # unsampled non-finite coordinates are neither read nor validated
    q = np.array([0.5, np.nan, 0.25, np.inf], np.float32)
    assert index.query(q, ws, uha.QueryStrategy.gemm) == index.query(q, ws) == 0
    # sampled non-finite coordinates are rejected
    with pytest.raises(uha.InvalidArgument):
        index.query(np.array([np.nan, 0.0, 0.25, 0.0], np.float32), ws)
    # empty sample: row 0 for every query
    empty = uha.CudaSampledCoordinateL2AnnIndex(SAMPLED_ROWS,
                                                coordinate_sample=uha.CoordinateSample())
    ews = empty.make_query_workspace(2)
    assert list(empty.query_batch(SAMPLED_QUERIES[:8], 2, None, ews)) == [0, 0]
    # errors
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(np.zeros(20, np.float32), 5, None, ws)
    with pytest.raises(uha.InvalidArgument):
        index.query_batch(np.zeros(7, np.float32), 2, None, ws)
    other = uha.CudaSampledCoordinateL2AnnIndex(SAMPLED_ROWS, coordinate_sample=SAMPLE)
    with pytest.raises(uha.InvalidArgument):
        other.query(SAMPLED_QUERIES[:4], ws)
    with pytest.raises(uha.InvalidArgument):
        uha.CudaSampledCoordinateL2AnnIndex(
            SAMPLED_ROWS, coordinate_sample=uha.CoordinateSample([0], [0], [1.0]))
    with pytest.raises(uha.OutOfRange):
        uha.CudaSampledCoordinateL2AnnIndex(
            SAMPLED_ROWS, coordinate_sample=uha.CoordinateSample([9], [1], [1.0]))


def test_sampled_l1_reference_fixture(oracle_module):
    index = uha.CudaSampledCoordinateL1AnnIndex(SAMPLED_ROWS, coordinate_sample=SAMPLE)
    ws = index.make_query_workspace(4)
    usage = index.space_usage()
    assert usage.index_payload_bytes == 3 * 2 * 4 + 2 * 4 + 2 * 8
    assert ws.payload_bytes() == 2 * (4 * 2 * 4) + 4 * 3 * 4 + 4 * 8
    expected, _ = oracle_module.flat("l1", SAMPLED_ROWS, SAMPLE.source_columns,
                                     SAMPLE.multiplicities,
                                     SAMPLE.inverse_probabilities, SAMPLED_QUERIES)
    assert np.array_equal(index.query_batch(SAMPLED_QUERIES, 4, None, ws), expected)
    q = np.array([0.5, np.nan, 0.25, np.inf], np.float32)
    assert index.query(q, ws) == oracle_module.flat(
        "l1", SAMPLED_ROWS, SAMPLE.source_columns, SAMPLE.multiplicities,
        SAMPLE.inverse_probabilities, q)[0][0]
    with pytest.raises(uha.InvalidArgument):
        index.query(np.array([0.5, 0.0, np.inf, 0.0], np.float32), ws)


@pytest.mark.parametrize("name", ["flat_l2_t8", "flat_l1_t8", "flat_l2_t32"])
def test_flat_golden_all_batches(name):
    rows, queries = golden_inputs()
    g = golden(name)
    cls = (uha.CudaSampledCoordinateL2AnnIndex if "l2" in name
           else uha.CudaSampledCoordinateL1AnnIndex)
    rng = uha.MT19937_64(int(g["seed"]))
    index = cls(rows, g["probabilities"], int(g["repetitions"]), rng)
    assert np.array_equal(index.coordinate_sample.source_columns, g["columns"])
    for batch in BATCHES:
        got, _ = run(index, queries, batch)
        assert np.array_equal(got, g["indices"]), f"batch {batch}"


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_flat_synthetic_parity_against_reference(oracle_module, metric):
    ds = synthetic.row_dataset(rows=300, classes=9, queries=200, d=3000, seed=21)
    probs = oracle_module.probabilities(metric, ds.rows)
    cls = (uha.CudaSampledCoordinateL2AnnIndex if metric == "l2"
           else uha.CudaSampledCoordinateL1AnnIndex)
    for reps in (8, 64):
        index = cls(ds.rows, probs, reps, uha.MT19937_64(reps))
        s = index.coordinate_sample
        expected, edist = oracle_module.flat(metric, ds.rows, s.source_columns,
                                             s.multiplicities, s.inverse_probabilities,
                                             ds.queries)
        for batch in (1, 7, 64, 200):
            got, dist = run(index, ds.queries, batch)
            assert np.array_equal(got, expected), (reps, batch)
            assert np.allclose(dist, edist, rtol=DIST_RTOL, atol=1e-30)


def test_gpu_probabilities_match_cpu(oracle_module):
    rows = np.array([[0.0, 0.0], [3.0, 4.0]], np.float32)
    p2 = uha.compute_l2_importance_probabilities_gpu(rows).probabilities
    p1 = uha.compute_l1_importance_probabilities_gpu(rows).probabilities
    assert np.allclose(p2, [9 / 25, 16 / 25], rtol=0, atol=1e-12)
    assert np.allclose(p1, [3 / 7, 4 / 7], rtol=0, atol=1e-12)
    rows, _ = golden_inputs()
    for metric, fn in (("l2", uha.compute_l2_importance_probabilities_gpu),
                       ("l1", uha.compute_l1_importance_probabilities_gpu)):
        res = fn(rows)
        expected = golden(f"probabilities_{metric}")["probabilities"]
        assert np.allclose(res.probabilities, expected, rtol=1e-12, atol=1e-15)
        assert res.pair_count == rows.shape[0] * (rows.shape[0] - 1) // 2
    ds = synthetic.row_dataset(rows=97, classes=4, queries=1, d=2100, seed=8)
    for metric, fn in (("l2", uha.compute_l2_importance_probabilities_gpu),
                       ("l1", uha.compute_l1_importance_probabilities_gpu)):
        assert np.allclose(fn(ds.rows).probabilities,
                           oracle_module.probabilities(metric, ds.rows),
                           rtol=1e-12, atol=1e-15)


def test_flat_facade_defaults_to_gpu_probabilities(oracle_module):
    probs = uha.compute_l2_importance_probabilities_gpu(SAMPLED_ROWS).probabilities
    a = uha.CudaFlatL2AnnIndex(SAMPLED_ROWS, 2, uha.MT19937_64(77))
    b = uha.CudaSampledCoordinateL2AnnIndex(SAMPLED_ROWS, probs, 2, uha.MT19937_64(77))
    assert np.array_equal(a.coordinate_sample.source_columns,
                          b.coordinate_sample.source_columns)
    wa = a.make_query_workspace(4)
    wb = b.make_query_workspace(4)
    assert np.array_equal(a.query_batch(SAMPLED_QUERIES, 4, None, wa),
                          b.query_batch(SAMPLED_QUERIES, 4, None, wb))


@pytest.mark.parametrize("kind", ["exact_l2", "exact_l1", "flat_l2", "hier_l1"])
def test_query_many_equals_per_batch_calls(oracle_module, kind):
    ds = synthetic.row_dataset(rows=300, classes=5, queries=45, d=2000, seed=31)
    if kind.startswith("exact"):
        index = (uha.CudaExactL2Index if kind == "exact_l2" else uha.CudaExactL1Index)(ds.rows)
    elif kind == "flat_l2":
        probs = oracle_module.probabilities("l2", ds.rows)
        index = uha.CudaSampledCoordinateL2AnnIndex(ds.rows, probs, 16, uha.MT19937_64(1))
    else:
        probs = oracle_module.probabilities("l1", ds.rows)
        index = uha.CudaHierarchicalL1AnnIndex(ds.rows, 8, 16, uha.MT19937_64(2),
                                               importance_probabilities=probs)
    for batch in (1, 4, 9):
        ws = index.make_query_workspace(batch)
        dist = np.zeros(45, np.float64)
        many = index.query_many(ds.queries, 45, batch, None, ws, distances=dist)
        single, sdist = run(index, ds.queries, batch)
        assert np.array_equal(many, single)
        assert np.array_equal(dist, sdist)
    with pytest.raises(uha.InvalidArgument):
        index.query_many(ds.queries, 45, 10, None, index.make_query_workspace(9))
    bad = ds.queries.copy()
    bad[30, :] = np.nan
    with pytest.raises(uha.InvalidArgument):
        index.query_many(bad, 45, 4, None, index.make_query_workspace(4))


def test_timing_samples_every_stride_batch():
    ds = synthetic.row_dataset(rows=300, classes=5, queries=20, d=4000, seed=2)
    index = uha.CudaExactL2Index(ds.rows)
    ws = index.make_query_workspace(1)
    ws.set_timing(True, stride=8)
    got = index.query_many(ds.queries, 20, 1, None, ws)
    st = ws.last_stats()
    assert st["timed_scans"] == 3 and st["scan_ms"] > 0 and st["device_ms"] > 0
    ws.set_timing(True)
    assert np.array_equal(index.query_many(ds.queries, 20, 1, None, ws), got)
    assert ws.last_stats()["timed_scans"] == 20
    ws.set_timing(False)
    index.query_many(ds.queries, 20, 1, None, ws)
    assert ws.last_stats()["timed_scans"] == 0
    with pytest.raises(uha.InvalidArgument):
        ws.set_timing(True, stride=0)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_binary32_overflowing_distances_match_reference(oracle_module, metric):
    """Distances above the binary32 range (finite in the CPU's binary64) have
    no finite upper bound: the query is replayed and the CPU's row returned,
    both when one row overflows and when every row does."""
    rng = np.random.default_rng(5)
    rows = rng.standard_normal((50, 64)).astype(np.float32)
    queries = rng.standard_normal((12, 64)).astype(np.float32)
    scale = np.float32(4e18 if metric == "l2" else 1e37)
    one = rows.copy()
    one[7] *= scale
    everything = rows * scale
    cls = uha.CudaExactL2Index if metric == "l2" else uha.CudaExactL1Index
    for r, q in ((one, queries), (everything, queries * scale)):
        expected, edist = oracle_module.exact(metric, r, q)
        assert np.all(np.isfinite(edist))
        for batch in (1, 12):
            got, _ = run(cls(r), q, batch)
            assert np.array_equal(got, expected), batch
