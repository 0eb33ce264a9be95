"""Data files on the CPU: SHA-256, the versioned importance-probability file
and the NPY dataset loader, pinned to the reference's own implementations
(src/io/*.cpp, src/datasets/representative_query_dataset.cpp compiled into
oracle/_ref) and to published SHA-256 test vectors (FIPS 180-4 examples).
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

uha = pytest.importorskip("ultrahigh_ann_b200")
from ultrahigh_ann_b200 import _abi  # noqa: E402
from ultrahigh_ann_b200 import io as uio  # noqa: E402

if not _abi.LIBRARY_PATH.exists():
    pytest.skip("engine library not built", allow_module_level=True)


def _ref(oracle_module):
    if not oracle_module.ref_available():
        pytest.skip("reference library not built here")
    return oracle_module


@pytest.mark.parametrize("message,digest", [
    (b"", "e3b0c44298fc1c149afbf4c8996fb92427ae41e4649b934ca495991b7852b855"),
    (b"abc", "ba7816bf8f01cfea414140de5dae2223b00361a396177a9cb410ff61f20015ad"),
    (b"abcdbcdecdefdefgefghfghighijhijkijkljklmklmnlmnomnopnopq",
     "248d6a61d20638b8e5c026930c3e6039a33ce45964ff2167f6ecedd419db06c1"),
])
def test_sha256_known_answers(message, digest):
    assert uio.sha256_hex(uio.sha256(message)) == digest


def test_sha256_matches_hashlib_at_every_padding_length():
    rng = np.random.default_rng(0)
    for n in list(range(0, 130)) + [1000, 4096, 1 << 20]:
        data = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert uio.sha256(data) == hashlib.sha256(data).digest(), n


def test_sha256_file_matches_reference(tmp_path, oracle_module):
    O = _ref(oracle_module)
    p = tmp_path / "m.bin"
    p.write_bytes(np.random.default_rng(1).bytes(3_000_001))
    assert uio.sha256_file(p) == hashlib.sha256(p.read_bytes()).digest()
    assert uio.sha256_file(p) == O.ref_sha256_file(p)


def _probs(n, seed=2):
    p = np.random.default_rng(seed).random(n)
    p[0], p[-1] = 0.0, 1.0
    return p


@pytest.mark.parametrize("kind", [uio.ImportanceProbabilityKind.l1,
                                  uio.ImportanceProbabilityKind.l2])
def test_probability_file_identical_to_reference(tmp_path, oracle_module, kind):
    O = _ref(oracle_module)
    sha = hashlib.sha256(b"representatives").digest()
    p = _probs(777)
    ours, theirs = tmp_path / "a" / "ours.bin", tmp_path / "b" / "theirs.bin"
    uio.save_importance_probabilities(ours, kind, 48, sha, p)
    O.ref_probabilities_save(theirs, int(kind), 48, sha, p)
    assert ours.read_bytes() == theirs.read_bytes()
    f = uio.load_importance_probabilities(theirs)
    assert f.kind == kind and f.representative_count == 48
    assert f.representatives_sha256 == sha
    assert np.array_equal(f.probabilities.view(np.uint64), p.view(np.uint64))
    k, reps, d, vals = O.ref_probabilities_load(ours)
    assert k == int(kind) and reps == 48 and d == sha and np.array_equal(vals, p)
    assert uio.importance_probability_source_matches(f, kind, 48, 777, sha)
    assert not uio.importance_probability_source_matches(f, kind, 47, 777, sha)
    assert not uio.importance_probability_source_matches(f, kind, 48, 776, sha)
    other = uio.ImportanceProbabilityKind.l2 if kind == uio.ImportanceProbabilityKind.l1 \
        else uio.ImportanceProbabilityKind.l1
    assert not uio.importance_probability_source_matches(f, other, 48, 777, sha)


def _corrupt_files(tmp_path, good: bytes):
    cases = {
        "magic": b"UHANNPR1" + good[8:],
        "kind": good[:8] + b"\x03" + good[9:],
        "reserved": good[:10] + b"\x01" + good[11:],
        "truncated_header": good[:20],
        "truncated_values": good[:-3],
        "trailing": good + b"\x00",
        "range": good[:-8] + np.float64(1.5).tobytes(),
        "nan": good[:-8] + np.float64(np.nan).tobytes(),
        "empty": b"",
    }
    out = {}
    for name, data in cases.items():
        f = tmp_path / f"{name}.bin"
        f.write_bytes(data)
        out[name] = f
    out["missing"] = tmp_path / "does-not-exist.bin"
    return out


def test_probability_file_errors_match_reference(tmp_path, oracle_module):
    O = _ref(oracle_module)
    good = tmp_path / "good.bin"
    uio.save_importance_probabilities(good, uio.ImportanceProbabilityKind.l2, 3,
                                      bytes(range(32)), _probs(9))
    for name, path in _corrupt_files(tmp_path, good.read_bytes()).items():
        with pytest.raises(RuntimeError) as ours:
            uio.load_importance_probabilities(path)
        with pytest.raises(O.ReferenceError_) as theirs:
            O.ref_probabilities_load(path)
        assert str(ours.value) == str(theirs.value).split(": ", 1)[1], name
    with pytest.raises(RuntimeError):
        uio.save_importance_probabilities(tmp_path / "bad.bin",
                                          uio.ImportanceProbabilityKind.l1, 1,
                                          bytes(32), [0.5, -0.1])


def test_npy_matrices_and_labels_match_reference(tmp_path, oracle_module):
    O = _ref(oracle_module)
    rng = np.random.default_rng(3)
    m = rng.standard_normal((17, 33)).astype(np.float32)
    np.save(tmp_path / "m.npy", m)
    got = uio.load_float_matrix_npy(tmp_path / "m.npy")
    assert got.dtype == np.float32 and np.array_equal(got, m)
    assert np.array_equal(O.ref_npy_f32(tmp_path / "m.npy"), m)
    labels = rng.integers(0, 65535, 41).astype(np.uint16)
    np.save(tmp_path / "l.npy", labels)
    assert np.array_equal(uio.load_label_vector_npy(tmp_path / "l.npy"), labels)
    assert np.array_equal(O.ref_npy_u16(tmp_path / "l.npy"), labels)
    # format version 2 header
    with open(tmp_path / "v2.npy", "wb") as f:
        np.lib.format.write_array(f, m, version=(2, 0))
    assert np.array_equal(uio.load_float_matrix_npy(tmp_path / "v2.npy"), m)


def test_npy_errors_match_reference(tmp_path, oracle_module):
    O = _ref(oracle_module)
    m = np.arange(12, dtype=np.float32).reshape(3, 4)
    cases = {}
    np.save(tmp_path / "fortran.npy", np.asfortranarray(m))
    cases["fortran"] = tmp_path / "fortran.npy"
    np.save(tmp_path / "f64.npy", m.astype(np.float64))
    cases["f64"] = tmp_path / "f64.npy"
    np.save(tmp_path / "one_d.npy", m.reshape(-1))
    cases["one_d"] = tmp_path / "one_d.npy"
    bad = m.copy()
    bad[1, 2] = np.inf
    np.save(tmp_path / "inf.npy", bad)
    cases["inf"] = tmp_path / "inf.npy"
    good = (tmp_path / "fortran.npy").read_bytes()
    np.save(tmp_path / "ok.npy", m)
    ok = (tmp_path / "ok.npy").read_bytes()
    (tmp_path / "trunc.npy").write_bytes(ok[:-4])
    cases["trunc"] = tmp_path / "trunc.npy"
    (tmp_path / "trail.npy").write_bytes(ok + b"\x00" * 4)
    cases["trail"] = tmp_path / "trail.npy"
    (tmp_path / "magic.npy").write_bytes(b"\x93NUMPX" + ok[6:])
    cases["magic"] = tmp_path / "magic.npy"
    (tmp_path / "version.npy").write_bytes(ok[:6] + b"\x04\x00" + ok[8:])
    cases["version"] = tmp_path / "version.npy"
    cases["missing"] = tmp_path / "missing.npy"
    assert good != ok
    for name, path in cases.items():
        with pytest.raises(RuntimeError) as ours:
            uio.load_float_matrix_npy(path)
        with pytest.raises(O.ReferenceError_) as theirs:
            O.ref_npy_f32(path)
        assert str(ours.value) == str(theirs.value).split(": ", 1)[1], name


def test_dataset_directory(tmp_path):
    rng = np.random.default_rng(4)
    reps = rng.random((5, 7)).astype(np.float32)
    queries = rng.random((9, 7)).astype(np.float32)
    np.save(tmp_path / "reference_vectors.npy", reps)
    np.save(tmp_path / "queries.npy", queries)
    np.save(tmp_path / "query_labels.npy", rng.integers(0, 5, 9).astype(np.uint16))
    ds = uio.load_representative_query_dataset(tmp_path)
    assert np.array_equal(ds.representatives, reps) and np.array_equal(ds.queries, queries)
    assert np.array_equal(ds.representative_labels, np.arange(5))
    np.save(tmp_path / "reference_labels.npy", np.array([1, 1, 2, 2, 3], np.uint16))
    with pytest.raises(RuntimeError, match="query label has no representative"):
        uio.load_representative_query_dataset(tmp_path)
    np.save(tmp_path / "query_labels.npy", np.ones(8, np.uint16))
    with pytest.raises(RuntimeError, match="query label count"):
        uio.load_representative_query_dataset(tmp_path)
    np.save(tmp_path / "queries.npy", rng.random((8, 6)).astype(np.float32))
    with pytest.raises(RuntimeError, match="dimensions do not match"):
        uio.load_representative_query_dataset(tmp_path)
