"""The engine's importance probabilities against the reference CPU's, bit for bit.

The direct pair backend performs the reference CPU's own binary64 operations
in its order (src/hnsvw25/l2/importance_sampling.cpp:19-45 with
src/core/l2_distance.cpp:9-25; src/hnsvw25/l1/importance_sampling.cpp:19-47
with src/core/l1_distance.cpp:12-28), so its probabilities, and the coordinate
sample drawn from them for a seed, equal the reference's: an index built from
GPU probabilities samples the same multiset I as the reference's
FlatL2AnnIndex / L1AnnIndex with CPU probabilities. The Gram backend (the
reference's cuBLAS form) is held to the reference's own GPU tolerance, 1e-6
(tests/hnsvw25/l2/importance_sampling_test.cpp:131-134).
"""
from __future__ import annotations

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from conftest import golden_inputs
from ultrahigh_ann_b200 import synthetic

pytestmark = pytest.mark.gpu

GPU_FN = {"l2": uha.compute_l2_importance_probabilities_gpu,
          "l1": uha.compute_l1_importance_probabilities_gpu}


def _ref(oracle_module):
    if not oracle_module.ref_available():
        pytest.skip("reference library oracle/_ref is not built")
    return oracle_module


def _cases():
    rows, _ = golden_inputs()
    yield "golden", rows
    # dimensions that are not a multiple of four (the L1 sum's tail) and not a
    # multiple of the 64-column slab
    yield "r97_d2103", synthetic.row_dataset(rows=97, classes=4, queries=1, d=2103,
                                             seed=8).rows
    ds = synthetic.row_dataset(rows=301, classes=9, queries=1, d=4097, seed=11).rows
    ds[17] = ds[3]  # a zero-distance pair contributes nothing
    yield "r301_d4097_duplicate", ds
    yield "r2_d3", np.array([[0.0, 1.0, 2.0], [3.0, -1.0, 2.5]], np.float32)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_direct_probabilities_bit_identical_to_reference_cpu(oracle_module, metric):
    O = _ref(oracle_module)
    for name, rows in _cases():
        got = GPU_FN[metric](rows).probabilities
        want = O.ref_probabilities(metric, rows)
        assert got.tobytes() == want.tobytes(), name


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_direct_probabilities_bit_identical_across_pair_chunks(oracle_module, metric):
    O = _ref(oracle_module)
    rows = synthetic.row_dataset(rows=200, classes=5, queries=1, d=1001, seed=2).rows
    want = O.ref_probabilities(metric, rows).tobytes()
    for chunks in (1, 3, 64):
        fn = GPU_FN[metric]
        got = fn(rows, pair_chunks=chunks).probabilities
        assert got.tobytes() == want, chunks


def test_gram_probabilities_within_reference_gpu_tolerance(oracle_module):
    O = _ref(oracle_module)
    rows = synthetic.row_dataset(rows=150, classes=5, queries=1, d=3000, seed=6).rows
    got = uha.compute_l2_importance_probabilities_gpu(rows, distance_backend="gram")
    want = O.ref_probabilities("l2", rows)
    assert np.allclose(got.probabilities, want, rtol=0, atol=1e-6)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_index_from_gpu_probabilities_samples_the_reference_set(oracle_module, metric):
    """The engine's flat index built with GPU probabilities holds the same
    coordinate sample as the reference sampler given CPU probabilities."""
    O = _ref(oracle_module)
    rows = synthetic.row_dataset(rows=400, classes=7, queries=1, d=6007, seed=12).rows
    probs = GPU_FN[metric](rows).probabilities
    cls = (uha.CudaSampledCoordinateL2AnnIndex if metric == "l2"
           else uha.CudaSampledCoordinateL1AnnIndex)
    index = cls(rows, probs, 32, uha.MT19937_64(21))
    cols, mult, invp, _ = O.ref_sample(O.ref_probabilities(metric, rows), 32, 21)
    s = index.coordinate_sample
    assert np.array_equal(s.source_columns, cols)
    assert np.array_equal(s.multiplicities, mult)
    assert s.inverse_probabilities.tobytes() == np.asarray(invp, np.float64).tobytes()


@pytest.mark.parametrize("metric, backend", [("l2", "direct"), ("l2", "gram"),
                                             ("l1", "direct")])
def test_binary32_maxima_within_reference_gpu_tolerance(oracle_module, metric, backend):
    """maxima="binary32" (the full-size build's form): the same pair distances,
    the per-column maxima in binary32, within the reference GPU path's 1e-6
    and within 3e-7 relative of the binary64 maxima."""
    O = _ref(oracle_module)
    rows = synthetic.row_dataset(rows=300, classes=6, queries=1, d=4099, seed=21).rows
    want = O.ref_probabilities(metric, rows)
    kwargs = {"distance_backend": backend} if metric == "l2" else {}
    got = GPU_FN[metric](rows, maxima="binary32", pair_chunks=3, **kwargs).probabilities
    assert np.allclose(got, want, rtol=0, atol=1e-6)
    assert np.all(np.abs(got - want) <= 3e-7 * np.abs(want) + 1e-30)


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_device_matrix_input_equals_host_input(metric):
    torch = pytest.importorskip("torch")
    rows = synthetic.row_dataset(rows=120, classes=5, queries=1, d=1031, seed=4).rows
    host = GPU_FN[metric](rows).probabilities
    dev = GPU_FN[metric](torch.from_numpy(rows).cuda()).probabilities
    assert dev.tobytes() == host.tobytes()
    bad = torch.from_numpy(rows).cuda()
    bad[7, 3] = float("nan")
    with pytest.raises(uha.InvalidArgument):
        GPU_FN[metric](bad)
