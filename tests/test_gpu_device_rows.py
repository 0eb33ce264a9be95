"""Indexes built from a representative matrix already on the device
(uha_*_index_create_device): binary32 or BF16 rows, with a row stride. Each
must equal the index built from the host binary32 matrix of the same values
(answers, reported distances, space usage) and fail with the host form's
errors; only the sampled columns are read or validated."""
from __future__ import annotations

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _answers(index, queries, batch=16, strategy=uha.QueryStrategy.direct):
    ws = index.make_query_workspace(batch)
    n = queries.shape[0]
    out = np.zeros(n, np.uint64)
    dist = np.zeros(n, np.float64)
    for s in range(0, n, batch):
        e = min(n, s + batch)
        index.query_batch(queries[s:e], e - s, out[s:e], ws, strategy, distances=dist[s:e])
    return out, dist


def _usage(index):
    u = index.space_usage()
    return (u.index_payload_bytes, u.unique_query_coordinates, u.sampled_multiplicity)


@pytest.fixture(scope="module")
def data():
    ds = synthetic.row_dataset(rows=300, classes=6, queries=40, d=2050, seed=11)
    wide = torch.zeros((300, 2056 + 24), dtype=torch.float32, device="cuda")
    wide[:, 24:24 + 2050] = torch.from_numpy(ds.rows).cuda()
    strided = wide[:, 24:24 + 2050]          # row stride 2080 elements
    bf16 = torch.from_numpy(ds.rows).cuda().to(torch.bfloat16)
    decoded = bf16.to(torch.float32).cpu().numpy()
    return ds, strided, bf16, decoded


def _pairs(data):
    ds, strided, bf16, decoded = data
    return ((ds.rows, strided), (decoded, bf16))


@pytest.mark.parametrize("cls", [uha.CudaExactL2Index, uha.CudaExactL1Index])
def test_exact_from_device_rows(data, cls):
    ds = data[0]
    for host, dev in _pairs(data):
        want = cls(host)
        got = cls(dev)
        assert _usage(got) == _usage(want)
        a, da = _answers(want, ds.queries)
        b, db = _answers(got, ds.queries)
        assert np.array_equal(a, b) and np.array_equal(da, db)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_sampled_from_device_rows(data, metric):
    ds = data[0]
    cls = (uha.CudaSampledCoordinateL2AnnIndex if metric == "l2"
           else uha.CudaSampledCoordinateL1AnnIndex)
    for host, dev in _pairs(data):
        probs = uha.compute_importance_probabilities_host(metric, host)
        want = cls(host, probs, 24, uha.MT19937_64(5))
        got = cls(dev, probs, 24, uha.MT19937_64(5))
        assert np.array_equal(want.coordinate_sample.source_columns,
                              got.coordinate_sample.source_columns)
        assert _usage(got) == _usage(want)
        a, da = _answers(want, ds.queries)
        b, db = _answers(got, ds.queries)
        assert np.array_equal(a, b) and np.array_equal(da, db)


@pytest.mark.parametrize("metric,p", [("l2", 16), ("l1", 9)])
def test_hierarchical_from_device_rows(data, metric, p):
    ds = data[0]
    cls = (uha.CudaHierarchicalL2AnnIndex if metric == "l2"
           else uha.CudaHierarchicalL1AnnIndex)
    for host, dev in _pairs(data):
        probs = uha.compute_importance_probabilities_host(metric, host)
        want = cls(host, 24, p, uha.MT19937_64(8), importance_probabilities=probs)
        got = cls(dev, 24, p, uha.MT19937_64(8), importance_probabilities=probs)
        assert np.array_equal(want.projection, got.projection)
        assert _usage(got) == _usage(want)
        a, da = _answers(want, ds.queries)
        b, db = _answers(got, ds.queries)
        assert np.array_equal(a, b) and np.array_equal(da, db)
        if metric == "l2":
            bf16 = uha.QueryStrategy.gemm_bf16_rerank
            a, da = _answers(want, ds.queries, strategy=bf16)
            b, db = _answers(got, ds.queries, strategy=bf16)
            assert np.array_equal(a, b) and np.array_equal(da, db)


def test_device_rows_need_probabilities(data):
    with pytest.raises(uha.InvalidArgument, match="host representative matrix"):
        uha.CudaFlatL2AnnIndex(data[1], 8, uha.MT19937_64(1))


def test_device_rows_validation():
    rows = torch.ones((4, 6), dtype=torch.float32, device="cuda")
    rows[2, 3] = float("inf")
    with pytest.raises(uha.InvalidArgument, match="representatives must be finite"):
        uha.CudaExactL2Index(rows)
    sample = uha.CoordinateSample([1, 3], [1, 1], [2.0, 2.0])
    with pytest.raises(uha.InvalidArgument, match="sampled representatives must be finite"):
        uha.CudaSampledCoordinateL1AnnIndex(rows, coordinate_sample=sample)
    # an unsampled non-finite column is never read
    ok = uha.CudaSampledCoordinateL2AnnIndex(
        rows, coordinate_sample=uha.CoordinateSample([0, 5], [1, 1], [2.0, 2.0]))
    assert ok.row_count == 4
    # the scaled binary32 value overflows only at (row 1, column 5), before
    # the non-finite source value at (row 2, column 3): host order decides
    big = torch.ones((4, 6), dtype=torch.float32, device="cuda")
    big[1, 5] = 3.0e38
    big[2, 3] = float("nan")
    with pytest.raises(uha.InvalidArgument, match="transformed representatives must be finite"):
        uha.CudaSampledCoordinateL2AnnIndex(
            big, coordinate_sample=uha.CoordinateSample([3, 5], [1, 1], [4.0, 4.0]))
    host = np.ones((4, 6), np.float32)
    with pytest.raises(uha.InvalidArgument, match="not memory of the index's device"):
        uha.CudaExactL2Index(uha.DeviceMatrix(host.ctypes.data, 4, 6))
    with pytest.raises(uha.InvalidArgument, match="aligned"):
        uha.CudaExactL2Index(uha.DeviceMatrix(rows.data_ptr() + 2, 3, 5))
    with pytest.raises(uha.InvalidArgument, match="row stride"):
        uha.CudaExactL2Index(uha.DeviceMatrix(rows.data_ptr(), 4, 6, row_stride=5))
    with pytest.raises(uha.InvalidArgument, match="at least one representative"):
        uha.CudaExactL2Index(uha.DeviceMatrix(rows.data_ptr(), 0, 6))
