"""Data files on the path: the versioned importance-probability file bound to
its representative matrix by SHA-256, and the NPY files of a transformed
dataset directory. Python mirror of include/ultrahigh_ann/io/
importance_probability_io.hpp, include/ultrahigh_ann/io/sha256.hpp and
include/ultrahigh_ann/datasets/representative_query_dataset.hpp; the file
formats are parsed and written by the engine library (csrc/io.cpp).
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _abi
from .api import _check


class ImportanceProbabilityKind(enum.IntEnum):
    """include/ultrahigh_ann/io/importance_probability_io.hpp:12-15."""

    l1 = _abi.L1
    l2 = _abi.L2


@dataclass
class ImportanceProbabilityFile:
    kind: ImportanceProbabilityKind
    representative_count: int
    representatives_sha256: bytes
    probabilities: np.ndarray


def sha256(data: bytes) -> bytes:
    out = (ctypes.c_uint8 * 32)()
    buf = bytes(data)
    _check(_abi.load().uha_sha256(ctypes.c_char_p(buf), ctypes.c_uint64(len(buf)), out))
    return bytes(out)


def sha256_file(path) -> bytes:
    """SHA-256 of the exact bytes stored in a file (sha256.hpp:14)."""
    out = (ctypes.c_uint8 * 32)()
    _check(_abi.load().uha_sha256_file(str(path).encode(), out))
    return bytes(out)


def sha256_hex(digest: bytes) -> str:
    return bytes(digest).hex()


def save_importance_probabilities(path, kind, representative_count: int,
                                  representatives_sha256: bytes, probabilities) -> None:
    """importance_probability_io.hpp:27-31."""
    if len(representatives_sha256) != 32:
        raise ValueError("a SHA-256 digest has 32 bytes")
    p = np.ascontiguousarray(probabilities, dtype=np.float64).reshape(-1)
    digest = (ctypes.c_uint8 * 32)(*bytes(representatives_sha256))
    _check(_abi.load().uha_probabilities_save(
        str(path).encode(), int(kind), ctypes.c_uint64(representative_count), digest,
        ctypes.c_void_p(p.ctypes.data if p.size else 0), ctypes.c_uint64(p.size)))


def load_importance_probabilities(path) -> ImportanceProbabilityFile:
    """importance_probability_io.hpp:33-34."""
    kind = ctypes.c_int()
    reps = ctypes.c_uint64()
    count = ctypes.c_uint64()
    digest = (ctypes.c_uint8 * 32)()
    lib = _abi.load()
    _check(lib.uha_probabilities_load(str(path).encode(), ctypes.byref(kind),
                                      ctypes.byref(reps), digest, None, 0,
                                      ctypes.byref(count)))
    out = np.zeros(count.value, dtype=np.float64)
    _check(lib.uha_probabilities_load(str(path).encode(), ctypes.byref(kind),
                                      ctypes.byref(reps), digest,
                                      ctypes.c_void_p(out.ctypes.data if out.size else 0),
                                      ctypes.c_uint64(out.size), ctypes.byref(count)))
    return ImportanceProbabilityFile(ImportanceProbabilityKind(kind.value), reps.value,
                                     bytes(digest), out)


def importance_probability_source_matches(file: ImportanceProbabilityFile, kind,
                                          representative_count: int,
                                          coordinate_count: int,
                                          representatives_sha256: bytes) -> bool:
    """importance_probability_io.hpp:36-39."""
    return (file.kind == kind and file.representative_count == representative_count
            and file.probabilities.size == coordinate_count
            and file.representatives_sha256 == bytes(representatives_sha256))


def load_float_matrix_npy(path) -> np.ndarray:
    """A two-dimensional little-endian float32 NPY matrix
    (representative_query_dataset.hpp:19-21)."""
    rows = ctypes.c_uint64()
    cols = ctypes.c_uint64()
    lib = _abi.load()
    _check(lib.uha_npy_load_f32(str(path).encode(), None, 0, ctypes.byref(rows),
                                ctypes.byref(cols)))
    out = np.zeros((rows.value, cols.value), dtype=np.float32)
    _check(lib.uha_npy_load_f32(str(path).encode(),
                                ctypes.c_void_p(out.ctypes.data if out.size else 0),
                                ctypes.c_uint64(out.size), ctypes.byref(rows),
                                ctypes.byref(cols)))
    return out


def load_label_vector_npy(path) -> np.ndarray:
    """A one-dimensional little-endian uint16 NPY label array
    (representative_query_dataset.hpp:23-25), as uint64."""
    count = ctypes.c_uint64()
    lib = _abi.load()
    _check(lib.uha_npy_load_u16(str(path).encode(), None, 0, ctypes.byref(count)))
    out = np.zeros(count.value, dtype=np.uint64)
    _check(lib.uha_npy_load_u16(str(path).encode(),
                                ctypes.c_void_p(out.ctypes.data if out.size else 0),
                                ctypes.c_uint64(out.size), ctypes.byref(count)))
    return out


@dataclass
class RepresentativeQueryDataset:
    representatives: np.ndarray
    queries: np.ndarray
    representative_labels: np.ndarray
    query_labels: np.ndarray


def load_representative_matrix(directory) -> np.ndarray:
    """reference_vectors.npy of a transformed dataset directory
    (src/datasets/representative_query_dataset.cpp:336-348)."""
    reps = load_float_matrix_npy(Path(directory) / "reference_vectors.npy")
    if reps.shape[0] == 0:
        raise RuntimeError("dataset has no reference vectors")
    if reps.shape[1] == 0:
        raise RuntimeError("dataset has no features")
    return reps


def load_representative_query_dataset(directory) -> RepresentativeQueryDataset:
    """The files of a transformed dataset directory, with the reference's
    checks; row indices are the labels when reference_labels.npy is absent
    (src/datasets/representative_query_dataset.cpp:350-403)."""
    d = Path(directory)
    reps = load_representative_matrix(d)
    queries = load_float_matrix_npy(d / "queries.npy")
    query_labels = load_label_vector_npy(d / "query_labels.npy")
    rl = d / "reference_labels.npy"
    if rl.is_file():
        rep_labels = load_label_vector_npy(rl)
    else:
        rep_labels = np.arange(reps.shape[0], dtype=np.uint64)
    if queries.shape[0] == 0:
        raise RuntimeError("dataset has no queries")
    if reps.shape[1] != queries.shape[1]:
        raise RuntimeError("reference-vector and query dimensions do not match")
    if query_labels.size != queries.shape[0]:
        raise RuntimeError("query label count does not match query row count")
    if rep_labels.size != reps.shape[0]:
        raise RuntimeError(
            "reference label count does not match reference-vector row count")
    if not np.isin(query_labels, rep_labels).all():
        raise RuntimeError("query label has no representative")
    return RepresentativeQueryDataset(reps, queries, rep_labels, query_labels)
