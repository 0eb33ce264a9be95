"""Index equality with the reference's own CPU library (oracle/_ref) at a
larger scale than the golden fixtures: 2,048 rows of the TCGA-shaped synthetic
generator (log2(1 + Gamma) values, 40 % all-zero columns, 33 latent classes)
at d = 30,011, every index form and both metrics, batches 1, 64 and 256.

The flat and hierarchical indexes sample from the engine's GPU probabilities,
which equal the reference CPU's bit for bit, so the engine's coordinate sample
is the reference sampler's for the same seed; the reference indexes are built
from the CPU probabilities and the reference sampler (their constructors
taking probabilities), i.e. the reference path end to end. Indices must be
equal on every query; the bench repeats the exact and flat checks at
r = 7,028, d = 60,660 and the hierarchical one at the 65,536-row sizes.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def data():
    return synthetic.row_dataset(rows=2048, classes=33, queries=256, d=30011, seed=21)


@pytest.fixture(scope="module")
def ref(oracle_module):
    if not oracle_module.ref_available():
        pytest.skip("reference library oracle/_ref is not built")
    return oracle_module


def _answers(index, queries, batch, strategy=uha.QueryStrategy.direct):
    ws = index.make_query_workspace(batch)
    out = np.zeros(queries.shape[0], np.uint64)
    for s in range(0, queries.shape[0], batch):
        e = min(queries.shape[0], s + batch)
        index.query_batch(queries[s:e], e - s, out[s:e], ws, strategy)
    return out


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_exact_equals_reference_at_scale(ref, data, metric):
    want = ref.ref_exact(metric, data.rows, data.queries, THREADS)
    cls = uha.CudaExactL2Index if metric == "l2" else uha.CudaExactL1Index
    index = cls(data.rows)
    for batch in (1, 64, 256):
        assert np.array_equal(_answers(index, data.queries, batch), want), batch


@pytest.mark.parametrize("metric", ["l2", "l1"])
@pytest.mark.parametrize("repetitions", [32, 128])
def test_flat_equals_reference_at_scale(ref, data, metric, repetitions):
    cpu_probs = ref.ref_probabilities(metric, data.rows)
    fn = (uha.compute_l2_importance_probabilities_gpu if metric == "l2"
          else uha.compute_l1_importance_probabilities_gpu)
    gpu_probs = fn(data.rows).probabilities
    assert gpu_probs.tobytes() == cpu_probs.tobytes()
    cls = (uha.CudaSampledCoordinateL2AnnIndex if metric == "l2"
           else uha.CudaSampledCoordinateL1AnnIndex)
    index = cls(data.rows, gpu_probs, repetitions, uha.MT19937_64(5))
    cols, mult, invp, _ = ref.ref_sample(cpu_probs, repetitions, 5)
    assert np.array_equal(index.coordinate_sample.source_columns, cols)
    want = ref.ref_sampled(metric, data.rows, cols, mult, invp, data.queries, THREADS)
    for batch in (1, 64, 256):
        assert np.array_equal(_answers(index, data.queries, batch), want), batch


@pytest.mark.parametrize("metric", ["l2", "l1"])
@pytest.mark.parametrize("p", [16, 64])
def test_hierarchical_equals_reference_at_scale(ref, data, metric, p):
    cpu_probs = ref.ref_probabilities(metric, data.rows)
    rows, queries = data.rows[:1500], data.queries[:96]
    want, _ = ref.ref_hierarchical(metric, rows, cpu_probs, 32, p, 9, queries, THREADS)
    cls = (uha.CudaHierarchicalL2AnnIndex if metric == "l2"
           else uha.CudaHierarchicalL1AnnIndex)
    index = cls(rows, 32, p, uha.MT19937_64(9), importance_probabilities=cpu_probs)
    for batch in (1, 64, 96):
        assert np.array_equal(_answers(index, queries, batch), want), batch
