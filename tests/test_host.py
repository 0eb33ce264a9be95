"""Host-side logic of the engine that needs no GPU: the C-ABI library loads
and exports every entry point include/uha_b200.h declares, the host sampler
and projection draws reproduce the reference's (same engine, same
distributions, same order), and errors map onto the reference's exception
types."""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

import ultrahigh_ann_b200 as uha
from conftest import ROOT, engine_state, golden, golden_inputs
from ultrahigh_ann_b200 import _abi


def declared_functions() -> set[str]:
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(uha_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    declared = declared_functions()
    assert declared, "no declarations found"
    for name in sorted(declared):
        assert hasattr(lib, name), f"{name} declared but not exported"
    assert declared == set(_abi.SIGNATURES), "ctypes table and header differ"


def test_library_is_built_for_sm100a():
    from ultrahigh_ann_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert _abi.LIBRARY_PATH.exists()


def test_device_matrix_descriptor_needs_no_device():
    m = uha.DeviceMatrix(4096, 3, 5, "bfloat16", row_stride=8)
    st = m._struct()
    assert (st.data, st.type, st.rows, st.columns, st.row_stride) == (4096, _abi.VALUES_BF16,
                                                                      3, 5, 8)
    assert uha.DeviceMatrix(64, 2, 7)._struct().row_stride == 7
    with pytest.raises(uha.InvalidArgument):
        uha.DeviceMatrix(64, 2, 7, "float16")._struct()
    torch = pytest.importorskip("torch")
    with pytest.raises(uha.InvalidArgument):
        uha.DeviceMatrix.from_torch(torch.zeros((2, 3)))
    # a host-side operation on a device matrix names what it needs
    with pytest.raises(uha.InvalidArgument, match="host representative matrix"):
        uha.compute_importance_probabilities_host("l2", m)


def test_no_device_is_reported_as_runtime_error_or_none():
    if uha.cuda_available():
        pytest.skip("a CUDA device is visible")
    assert uha.cuda_runtime_info() is None
    with pytest.raises(uha.CudaRuntimeError):
        uha.CudaExactL2Index(np.zeros((3, 2), np.float32))


@pytest.mark.parametrize("name", ["flat_l2_t8", "flat_l1_t8", "flat_l2_t32"])
def test_host_sampler_reproduces_reference_sample(name):
    g = golden(name)
    rng = uha.MT19937_64(int(g["seed"]))
    sample = uha.build_coordinate_sample(g["probabilities"], int(g["repetitions"]), rng)
    assert np.array_equal(sample.source_columns, g["columns"])
    assert np.array_equal(sample.multiplicities, g["multiplicities"])
    assert np.array_equal(sample.inverse_probabilities, g["inverse_probabilities"])
    assert rng.state() == engine_state(g["engine_state"])


@pytest.mark.parametrize("name", ["hier_l2_p16", "hier_l2_p15", "hier_l1_p16",
                                  "hier_l1_p15"])
def test_host_projection_draws_reproduce_reference(name):
    g = golden(name)
    rng = uha.MT19937_64(int(g["seed"]))
    sample = uha.build_coordinate_sample(g["probabilities"], int(g["repetitions"]), rng)
    p = int(g["projection_dimension"])
    draw = uha.build_jl_matrix if "l2" in name else uha.build_cauchy_matrix
    matrix = draw(sample, p, rng)
    assert np.array_equal(matrix, g["projection"])
    # one engine through sampling and projection, as the reference constructor
    assert rng.state() == engine_state(g["engine_state_after"])


def test_sampler_rejects_invalid_probabilities_as_domain_error():
    rng = uha.MT19937_64(1)
    with pytest.raises(uha.DomainError):
        uha.build_coordinate_sample(np.array([0.5, 1.5]), 4, rng)
    with pytest.raises(uha.DomainError):
        uha.build_coordinate_sample(np.array([np.nan]), 4, rng)
    with pytest.raises(uha.DomainError):
        uha.build_coordinate_sample(np.array([-0.1]), 4, rng)


def test_sampler_edge_cases():
    rng = uha.MT19937_64(1234)
    # p = 1 -> multiplicity T and 1/p = 1 (tests/hnsvw25/l2/importance_sampling_test.cpp:290-319)
    s = uha.build_coordinate_sample(np.array([1.0, 0.0, 1.0]), 7, rng)
    assert list(s.source_columns) == [0, 2]
    assert list(s.multiplicities) == [7, 7]
    assert list(s.inverse_probabilities) == [1.0, 1.0]
    # zero repetitions or all-zero probabilities -> empty sample
    assert len(uha.build_coordinate_sample(np.array([0.5, 0.5]), 0, rng)) == 0
    assert len(uha.build_coordinate_sample(np.zeros(10), 8, rng)) == 0
    assert len(uha.build_coordinate_sample(np.zeros(0), 8, rng)) == 0


def test_engine_state_roundtrip():
    a = uha.MT19937_64(77)
    uha.build_coordinate_sample(np.full(100, 0.3), 5, a)
    b = uha.MT19937_64(0)
    b.set_state(a.state())
    assert a == b
    with pytest.raises(uha.InvalidArgument):
        b.set_state("not an engine state")


def test_projection_rejects_zero_dimension():
    s = uha.CoordinateSample([0], [1], [2.0])
    with pytest.raises(uha.InvalidArgument):
        uha.build_jl_matrix(s, 0, uha.MT19937_64(1))


def test_golden_inputs_are_consistent():
    rows, queries = golden_inputs()
    assert rows.dtype == np.float32 and queries.dtype == np.float32
    assert rows.shape[1] == queries.shape[1]


@pytest.mark.parametrize("threads", [1, 3, 8])
def test_host_probabilities_are_the_reference_cpu_policy(threads):
    rows, _ = golden_inputs()
    for metric in ("l2", "l1"):
        p = uha.compute_importance_probabilities_host(metric, rows, threads)
        assert np.array_equal(p, golden(f"probabilities_{metric}")["probabilities"])


def test_host_probabilities_edge_cases():
    one = np.ones((1, 5), np.float32)
    assert np.array_equal(uha.compute_importance_probabilities_host("l2", one), np.zeros(5))
    same = np.ones((3, 4), np.float32)  # every pair at distance zero is skipped
    assert np.array_equal(uha.compute_importance_probabilities_host("l1", same), np.zeros(4))
    with pytest.raises(uha.InvalidArgument):
        uha.compute_importance_probabilities_host(
            "l2", np.array([[np.nan, 0.0], [1.0, 1.0]], np.float32))


def test_gaussian_jl_matrix_is_seeded_binary32_with_rademacher_variance():
    s = uha.CoordinateSample([0, 5, 9], [1, 4, 9], [2.0, 0.5, 1.25])
    p = 4096
    a = uha.build_gaussian_jl_matrix(s, p, uha.MT19937_64(3))
    b = uha.build_gaussian_jl_matrix(s, p, uha.MT19937_64(3))
    assert a.shape == (p, 3) and np.array_equal(a, b)
    assert np.array_equal(a, a.astype(np.float32).astype(np.float64))
    assert not np.array_equal(a, uha.build_gaussian_jl_matrix(s, p, uha.MT19937_64(4)))
    # the aggregated Rademacher entry's variance m (1/p_j) / p
    want = np.array([1 * 2.0, 4 * 0.5, 9 * 1.25]) / p
    assert np.allclose(a.var(axis=0), want, rtol=0.1)
    assert np.allclose(a.mean(axis=0), 0.0, atol=4 * np.sqrt(want / p))
    with pytest.raises(uha.InvalidArgument):
        uha.build_gaussian_jl_matrix(s, 0, uha.MT19937_64(1))
    with pytest.raises(uha.InvalidArgument):
        uha.CudaHierarchicalL1AnnIndex(np.ones((2, 3), np.float32), 4, 2,
                                       uha.MT19937_64(1), projection="gaussian")
