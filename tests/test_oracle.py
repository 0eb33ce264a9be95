"""Pins the oracle (oracle/uha_oracle.cpp) before anything is checked against
it: against the golden fixtures made by the reference itself, against the
reference's CPU library (oracle/_ref) on fresh seeded inputs, and against the
reference tests' known answers (tests/hnsvw25/l2/importance_sampling_test.cpp:
63-95, tests/hnsvw25/l1/importance_sampling_test.cpp:60-92,
tests/exact/l2/exact_l2_index_test.cpp:45-96)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import engine_state, golden, golden_inputs
from ultrahigh_ann_b200 import synthetic


def test_oracle_matches_golden_exact(oracle_module):
    rows, queries = golden_inputs()
    for metric in ("l2", "l1"):
        idx, _ = oracle_module.exact(metric, rows, queries)
        assert np.array_equal(idx, golden(f"exact_{metric}")["indices"])


def test_oracle_matches_golden_probabilities(oracle_module):
    rows, _ = golden_inputs()
    for metric in ("l2", "l1"):
        p = oracle_module.probabilities(metric, rows)
        assert np.array_equal(p, golden(f"probabilities_{metric}")["probabilities"])


@pytest.mark.parametrize("name", ["flat_l2_t8", "flat_l1_t8", "flat_l2_t32"])
def test_oracle_matches_golden_flat(oracle_module, name):
    rows, queries = golden_inputs()
    g = golden(name)
    cols, mult, inv, state = oracle_module.sample(g["probabilities"],
                                                  int(g["repetitions"]), int(g["seed"]))
    assert np.array_equal(cols, g["columns"])
    assert np.array_equal(mult, g["multiplicities"])
    assert np.array_equal(inv, g["inverse_probabilities"])
    assert state == engine_state(g["engine_state"])
    idx, _ = oracle_module.flat(name[5:7], rows, cols, mult, inv, queries)
    assert np.array_equal(idx, g["indices"])


@pytest.mark.parametrize("name", ["hier_l2_p16", "hier_l2_p15", "hier_l1_p16",
                                  "hier_l1_p15"])
def test_oracle_matches_golden_hierarchical(oracle_module, name):
    rows, queries = golden_inputs()
    g = golden(name)
    metric = name[5:7]
    p = int(g["projection_dimension"])
    cols, mult, inv, state = oracle_module.sample(g["probabilities"],
                                                  int(g["repetitions"]), int(g["seed"]))
    draw = oracle_module.jl_matrix if metric == "l2" else oracle_module.cauchy_matrix
    matrix = draw(mult, inv, p, state)
    assert np.array_equal(matrix, g["projection"])
    assert np.array_equal(oracle_module.project_rows(rows, cols, matrix),
                          g["projected_rows"])
    idx, _ = oracle_module.hierarchical(metric, rows, cols, matrix, queries)
    assert np.array_equal(idx, g["indices"])


def test_oracle_matches_reference_library_fresh_inputs(oracle_module):
    if not oracle_module.ref_available():
        pytest.skip("reference library not built in this tree")
    ds = synthetic.row_dataset(rows=61, classes=5, queries=50, d=1500, seed=99)
    for metric in ("l2", "l1"):
        ref = oracle_module.ref_exact(metric, ds.rows, ds.queries, threads=2)
        assert np.array_equal(ref, oracle_module.exact(metric, ds.rows, ds.queries)[0])
        probs = oracle_module.ref_probabilities(metric, ds.rows)
        assert np.array_equal(probs, oracle_module.probabilities(metric, ds.rows))
        cols, mult, inv, _ = oracle_module.ref_sample(probs, 16, 3)
        ref = oracle_module.ref_sampled(metric, ds.rows, cols, mult, inv, ds.queries,
                                        threads=2)
        assert np.array_equal(
            ref, oracle_module.flat(metric, ds.rows, cols, mult, inv, ds.queries)[0])


def test_known_answer_probabilities(oracle_module):
    # two rows differing by (3, 4): L2 p = (9/25, 16/25), L1 p = (3/7, 4/7)
    rows = np.array([[0.0, 0.0], [3.0, 4.0]], np.float32)
    assert np.allclose(oracle_module.probabilities("l2", rows), [9 / 25, 16 / 25],
                       rtol=0, atol=1e-15)
    assert np.allclose(oracle_module.probabilities("l1", rows), [3 / 7, 4 / 7],
                       rtol=0, atol=1e-15)


def test_ties_resolve_to_lowest_row(oracle_module):
    # tests/exact/l2/cuda_exact_l2_index_test.cpp:58-61, 94-124
    rows = np.array([[0, 0], [5, 0], [2, 4]], np.float32)
    queries = np.array([[1, 0], [3, 3], [2.5, 0], [5, 0]], np.float32)
    l2, _ = oracle_module.exact("l2", rows, queries)
    l1, _ = oracle_module.exact("l1", rows, queries)
    assert l2[2] == 0 and l1[2] == 0
    assert list(l2) == [0, 2, 0, 1]


def test_l1_grouped_summation_differs_from_sequential(oracle_module):
    # The reference's exact L1 uses std::transform_reduce, which adds groups of
    # four before accumulating; the oracle must follow that grouping, not a
    # left-to-right sum. Planted so the two orders round differently.
    big = 2.0 ** 60  # binary64 ulp 256: +100 rounds away, +200 rounds up
    q = np.array([[big, 100.0, 100.0, 100.0]], np.float32)
    rows = np.zeros((1, 4), np.float32)
    _, dist = oracle_module.exact("l1", rows, q)
    grouped = (big + 100.0) + (100.0 + 100.0)
    sequential = ((big + 100.0) + 100.0) + 100.0
    assert grouped != sequential
    assert dist[0] == grouped


@pytest.mark.parametrize("metric", ["l2", "l1"])
def test_reference_hierarchy_on_sampled_columns_equals_full_matrix(oracle_module, metric):
    """The full-size parity check runs the reference's hierarchical index over
    the sampled columns only (the full 65,536 x 262,144 matrix does not fit host
    memory). That index must answer exactly as the reference index over the
    full matrix, whatever the thread count of its row-block projection."""
    O = oracle_module
    if not O.ref_available():
        pytest.skip("reference library oracle/_ref is not built")
    ds = synthetic.row_dataset(rows=230, classes=6, queries=40, d=3001, seed=15)
    probs = O.ref_probabilities(metric, ds.rows)
    for reps, p, seed in ((8, 15, 3), (32, 16, 4), (16, 64, 5)):
        full, _ = O.ref_hierarchical(metric, ds.rows, probs, reps, p, seed, ds.queries)
        cols, mult, invp, state = O.ref_sample(probs, reps, seed)
        cols = cols.astype(np.int64)
        for threads in (1, 3, 8):
            got = O.ref_hierarchical_sampled(metric, ds.rows[:, cols], mult, invp, p,
                                             state, ds.queries[:, cols], threads)
            assert np.array_equal(got, full), (reps, p, threads)
