"""Request loop (uha_server_*) through the C ABI: continuous batching over
several device-resident indexes, HBM-budget admission, per-request errors.

No reference counterpart. The central check: every answer is the same when
its query runs alone and when it runs in a mix of requests to several indexes
that arrive while other batches are on the GPU (rows equal, distances within
the 1e-5 relative tolerance of the query contract).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, golden_inputs

pytestmark = pytest.mark.gpu

uha = pytest.importorskip("ultrahigh_ann_b200")
from ultrahigh_ann_b200 import synthetic  # noqa: E402

S = uha.QueryStrategy
DIST_RTOL = 1e-5


def _indexes():
    rows, _ = golden_inputs()
    ds = synthetic.row_dataset(rows=700, classes=9, queries=1, d=2500, seed=8)
    g = golden("flat_l2_t32")
    return [
        (uha.CudaExactL2Index(ds.rows), S.direct),
        (uha.CudaExactL2Index(ds.rows), S.gemm_bf16_rerank),
        (uha.CudaExactL1Index(rows), S.direct),
        (uha.CudaSampledCoordinateL2AnnIndex(rows, g["probabilities"], 32,
                                             uha.MT19937_64(int(g["seed"]))), S.direct),
        (uha.CudaHierarchicalL1AnnIndex(rows, 32, 15, uha.MT19937_64(4)), S.direct),
    ]


def _queries(pairs, per_index, seed):
    rng = np.random.default_rng(seed)
    return [np.abs(rng.standard_normal((per_index, ix.dimension))).astype(np.float32) * 3
            for ix, _ in pairs]


def _by_tag(results):
    order = np.argsort(results["tag"])
    return results[order]


def _alone(server, ids, queries):
    out = []
    for tag, (i, q) in enumerate(zip(ids, queries)):
        server.submit(int(i), q, tag)
        server.drain()
        out.append(server.poll())
    return _by_tag(np.concatenate(out))


def _mixed_load(pairs, per_index, seed):
    qs = _queries(pairs, per_index, seed)
    ids = np.repeat(np.arange(len(pairs)), per_index)
    flat = [q for per in qs for q in per]
    perm = np.random.default_rng(seed + 1).permutation(len(ids))
    return ids[perm], [flat[k] for k in perm]


@pytest.mark.parametrize("on_device", [False, True])
def test_same_result_alone_and_in_the_mix(on_device):
    import torch
    pairs = _indexes()
    ids, queries = _mixed_load(pairs, 40, seed=5)
    if on_device:
        dev = [torch.from_numpy(q).cuda() for q in queries]
        torch.cuda.synchronize()
        handles = [t.data_ptr() for t in dev]
    else:
        handles = queries
    server = uha.Server(hbm_budget_bytes=4 << 30, max_batch=16, slots=4,
                        queries_on_device=on_device)
    sid = [server.add_index(ix, st) for ix, st in pairs]
    assert sid == list(range(len(pairs)))
    assert server.reserve(0, 2) == 2
    alone = _alone(server, ids, handles)
    assert np.all(alone["status"] == 0)
    server.reset_stats()
    # open-loop arrivals, 2 us apart: batches form while others run
    arrival = np.arange(len(ids), dtype=np.float64) * 2.0
    server.replay(ids, handles, arrival, np.arange(len(ids)))
    server.drain()
    mixed = _by_tag(server.poll())
    assert len(mixed) == len(ids)
    assert np.all(mixed["status"] == 0)
    assert np.array_equal(mixed["index_id"], alone["index_id"])
    assert np.array_equal(mixed["row"], alone["row"])
    assert np.allclose(mixed["distance"], alone["distance"], rtol=DIST_RTOL, atol=1e-30)
    st = server.stats()
    assert st["completed"] == len(ids) and st["failed"] == 0
    assert st["mean_batch"] > 1.0 and st["batches"] < len(ids)
    assert st["peak_in_flight"] >= 2
    assert 0 < st["p50_us"] <= st["p99_us"] <= st["max_us"]
    # and the same as the index API, one query at a time
    for (ix, strategy), k in zip(pairs, range(len(pairs))):
        sel = np.nonzero(ids == k)[0][:5]
        ws = ix.make_query_workspace(1)
        for j in sel:
            q = queries[j]
            if isinstance(ix, (uha.CudaDenseL1ScanIndex, uha.CudaHierarchicalL1AnnIndex)):
                want = ix.query_batch(q, 1, None, ws)[0]
            else:
                want = ix.query_batch(q, 1, None, ws, strategy)[0]
            assert mixed["row"][j] == want


def _workspace_bytes(index, strategy, max_batch):
    probe = uha.Server(hbm_budget_bytes=64 << 30, max_batch=max_batch, slots=1)
    probe.add_index(index, strategy)
    return probe.stats()["workspace_bytes"]


def test_budget_admission_keeps_answers():
    pairs = _indexes()[:3]
    sizes = [_workspace_bytes(ix, st, 8) for ix, st in pairs]
    budget = max(sizes) + 1  # every index fits alone, not all together
    assert sum(sizes) > budget
    ids, queries = _mixed_load(pairs, 30, seed=9)
    server = uha.Server(hbm_budget_bytes=budget, max_batch=8, slots=3)
    for ix, st in pairs:
        server.add_index(ix, st)
    alone = _alone(server, ids, queries)
    server.reset_stats()
    server.replay(ids, queries, np.zeros(len(ids)), np.arange(len(ids)))
    server.drain()
    mixed = _by_tag(server.poll())
    assert np.array_equal(mixed["row"], alone["row"])
    assert np.all(mixed["status"] == 0)
    st = server.stats()
    assert st["peak_workspace_bytes"] <= budget
    assert st["admission_waits"] + st["evictions"] > 0


def test_budget_below_one_workspace_is_rejected():
    rows, _ = golden_inputs()
    index = uha.CudaExactL2Index(rows)
    server = uha.Server(hbm_budget_bytes=1024, max_batch=64, slots=2)
    with pytest.raises(uha.LengthError):
        server.add_index(index)


def test_bad_query_fails_alone():
    rows, queries = golden_inputs()
    index = uha.CudaExactL2Index(rows)
    server = uha.Server(hbm_budget_bytes=1 << 30, max_batch=32, slots=2)
    server.add_index(index)
    qs = [queries[i].copy() for i in range(20)]
    qs[7][11] = np.nan
    server.replay(np.zeros(20, np.uint32), qs, np.zeros(20), np.arange(20))
    server.drain()
    res = _by_tag(server.poll())
    assert res["status"][7] == 1  # UHA_INVALID_ARGUMENT
    ok = np.delete(np.arange(20), 7)
    assert np.all(res["status"][ok] == 0)
    assert np.array_equal(res["row"][ok], golden("exact_l2")["indices"][ok])
    assert server.stats()["failed"] == 1
