"""The reference's own CUDA-device test programs, unmodified, against the
engine.

oracle/Makefile compiles the reference library with its CUDA translation units
(and the four facades that pack queries on the host) replaced by the engine's
reference-side binding (ultrahigh_ann_b200/shim/), and links the reference's
eight "cuda-device" test programs (tests/exact/l{1,2}/cuda_exact_l{1,2}_index_test.cpp,
tests/hnsvw25/l{1,2}/importance_sampling_test.cpp,
tests/coordinate_sampling/cuda_sampled_coordinate_l{1,2}_ann_index_test.cpp,
tests/hnsvw25/l{1,2}/hierarchical/cuda_hierarchical_l{1,2}_ann_index_test.cpp)
against it. Each program exits 0 when every expectation holds, 1 on a failed
expectation and 77 when no CUDA device is usable.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
TESTS = ROOT / "oracle" / "_ref" / "tests"
PROGRAMS = [
    "exact/l1/cuda_exact_l1_index_test",
    "exact/l2/cuda_exact_l2_index_test",
    "hnsvw25/l1/importance_sampling_test",
    "hnsvw25/l2/importance_sampling_test",
    "coordinate_sampling/cuda_sampled_coordinate_l1_ann_index_test",
    "coordinate_sampling/cuda_sampled_coordinate_l2_ann_index_test",
    "hnsvw25/l1/hierarchical/cuda_hierarchical_l1_ann_index_test",
    "hnsvw25/l2/hierarchical/cuda_hierarchical_l2_ann_index_test",
]


def run(program: str) -> subprocess.CompletedProcess:
    path = TESTS / program
    if not path.exists():
        pytest.skip(f"{path} not built (the reference sources were not present)")
    return subprocess.run([str(path)], capture_output=True, text=True, timeout=600)


@pytest.mark.gpu
@pytest.mark.parametrize("program", PROGRAMS)
def test_reference_cuda_program_passes_on_the_engine(program):
    res = run(program)
    assert res.returncode == 0, f"{program} exited {res.returncode}\n{res.stdout}\n{res.stderr}"


@pytest.mark.parametrize("program", PROGRAMS)
def test_reference_cuda_program_skips_without_a_device(program):
    import ultrahigh_ann_b200 as uha
    if uha.cuda_available():
        pytest.skip("a CUDA device is visible")
    assert run(program).returncode == 77
