"""Shared test set-up: the `gpu` marker, import paths and golden fixtures.

Tests marked `gpu` need a CUDA device and call the engine through its C ABI;
everything else runs on the CPU (oracle pinning, host-side logic, library
exports, gloo multi-process plumbing).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as data:
        return {k: data[k] for k in data.files}


def golden_inputs() -> tuple[np.ndarray, np.ndarray]:
    g = golden("inputs")
    return g["rows"], g["queries"]


def engine_state(array: np.ndarray) -> str:
    return array.tobytes().decode()


@pytest.fixture(scope="session")
def oracle_module():
    from oracle import oracle as O
    if not O.ORACLE_LIB.exists():
        O.build()
    return O
