"""ORACLE — test infrastructure only (tests/, smoke() and bench.py's
cpu_baseline leg). ctypes access to

* liboracle.so — the CPU restatement in uha_oracle.cpp, and
* _ref/libref.so — the reference's own CPU library (built here from its
  sources by the Makefile; present wherever the built tree travels).

The engine never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_char_p, c_double, c_int, c_int64, c_uint64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref.so"

_oracle = None
_ref = None


REFERENCE_TREE_ENV = "UHA_REFERENCE_DIR"
DEFAULT_REFERENCE_TREE = "/root/reference"


def build() -> None:
    """Builds liboracle.so and, when the reference sources exist, _ref/.

    The reference tree is UHA_REFERENCE_DIR when set, else the container's
    read-only checkout; the Makefile itself has no default for it."""
    tree = os.environ.get(REFERENCE_TREE_ENV, DEFAULT_REFERENCE_TREE)
    cmd = ["make", "-s", "-C", str(HERE), "-j8"]
    if (Path(tree) / "src").is_dir():
        cmd.append(f"REF={tree}")
    subprocess.run(cmd, check=True)


def _p(a):
    return c_void_p(a.ctypes.data) if a is not None and a.size else c_void_p(0)


def oracle_lib() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            build()
        lib = ctypes.CDLL(str(ORACLE_LIB))
        lib.oracle_sample.restype = c_int64
        lib.oracle_sample.argtypes = [c_void_p, c_uint64, c_uint64, c_uint64, c_void_p,
                                      c_void_p, c_void_p, c_char_p, c_uint64]
        for name in ("oracle_jl_matrix", "oracle_cauchy_matrix"):
            fn = getattr(lib, name)
            fn.restype = None
            fn.argtypes = [c_void_p, c_void_p, c_uint64, c_uint64, c_char_p, c_uint64,
                           c_void_p]
        for name in ("oracle_exact_l2", "oracle_exact_l1"):
            fn = getattr(lib, name)
            fn.restype = None
            fn.argtypes = [c_void_p, c_uint64, c_uint64, c_void_p, c_uint64, c_void_p,
                           c_void_p]
        lib.oracle_weighted_l1.restype = None
        lib.oracle_weighted_l1.argtypes = [c_void_p, c_uint64, c_uint64, c_void_p,
                                           c_void_p, c_uint64, c_void_p, c_void_p]
        for name in ("oracle_flat_l2", "oracle_flat_l1"):
            fn = getattr(lib, name)
            fn.restype = c_int
            fn.argtypes = [c_void_p, c_uint64, c_uint64, c_void_p, c_void_p, c_void_p,
                           c_uint64, c_void_p, c_uint64, c_void_p, c_void_p]
        lib.oracle_project_rows.restype = None
        lib.oracle_project_rows.argtypes = [c_void_p, c_uint64, c_uint64, c_void_p,
                                            c_uint64, c_void_p, c_uint64, c_void_p]
        for name in ("oracle_hier_l2", "oracle_hier_l1"):
            fn = getattr(lib, name)
            fn.restype = c_int
            fn.argtypes = [c_void_p, c_uint64, c_void_p, c_uint64, c_uint64, c_void_p,
                           c_uint64, c_void_p, c_uint64, c_void_p, c_void_p]
        lib.oracle_probabilities.restype = None
        lib.oracle_probabilities.argtypes = [c_int, c_void_p, c_uint64, c_uint64,
                                             c_void_p]
        lib.oracle_threads.restype = c_int
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return REF_LIB.exists()


def reference_dir():
    """The reference source tree the _ref library was built from (recorded by
    the Makefile), or None when it is not present on this machine."""
    marker = REF_LIB.parent / "reference_dir"
    if not marker.exists():
        return None
    d = Path(marker.read_text().strip())
    return d if d.is_dir() else None


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} is missing (build it where the reference "
                               "sources are present: make -C oracle)")
        lib = ctypes.CDLL(str(REF_LIB))
        lib.ref_last_error.restype = c_char_p
        lib.ref_sample.restype = c_int
        lib.ref_sample.argtypes = [c_void_p, c_uint64, c_uint64, c_uint64, c_void_p,
                                   c_void_p, c_void_p, c_void_p, c_char_p, c_uint64]
        lib.ref_probabilities.restype = c_int
        lib.ref_probabilities.argtypes = [c_int, c_void_p, c_uint64, c_uint64, c_int,
                                          c_void_p]
        for name in ("ref_exact_l2", "ref_exact_l1"):
            fn = getattr(lib, name)
            fn.restype = c_int
            fn.argtypes = [c_void_p, c_uint64, c_uint64, c_void_p, c_uint64, c_int,
                           c_void_p]
        for name in ("ref_sampled_l2", "ref_sampled_l1"):
            fn = getattr(lib, name)
            fn.restype = c_int
            fn.argtypes = [c_void_p, c_uint64, c_uint64, c_void_p, c_void_p, c_void_p,
                           c_uint64, c_void_p, c_uint64, c_int, c_void_p]
        lib.ref_hierarchical.restype = c_int
        lib.ref_hierarchical.argtypes = [c_int, c_void_p, c_uint64, c_uint64, c_void_p,
                                         c_uint64, c_uint64, c_uint64, c_void_p,
                                         c_uint64, c_int, c_void_p, c_char_p, c_uint64]
        lib.ref_projection.restype = c_int
        lib.ref_projection.argtypes = [c_int, c_void_p, c_uint64, c_uint64, c_void_p,
                                       c_void_p, c_void_p, c_uint64, c_uint64, c_char_p,
                                       c_uint64, c_void_p, c_void_p]
        lib.ref_exact_create.restype = c_void_p
        lib.ref_exact_create.argtypes = [c_int, c_void_p, c_uint64, c_uint64]
        lib.ref_exact_destroy.restype = None
        lib.ref_exact_destroy.argtypes = [c_void_p]
        lib.ref_exact_query.restype = c_int
        lib.ref_exact_query.argtypes = [c_void_p, c_void_p, c_uint64, c_int, c_void_p]
        lib.ref_exact_query_batched.restype = c_int
        lib.ref_exact_query_batched.argtypes = [c_void_p, c_void_p, c_uint64, c_uint64,
                                                c_int, c_void_p]
        lib.ref_sha256_file.restype = c_int
        lib.ref_sha256_file.argtypes = [c_char_p, c_void_p]
        lib.ref_probabilities_save.restype = c_int
        lib.ref_probabilities_save.argtypes = [c_char_p, c_int, c_uint64, c_void_p,
                                               c_void_p, c_uint64]
        lib.ref_probabilities_load.restype = c_int
        lib.ref_probabilities_load.argtypes = [c_char_p, c_void_p, c_void_p, c_void_p,
                                               c_void_p, c_uint64, c_void_p]
        lib.ref_npy_f32.restype = c_int
        lib.ref_npy_f32.argtypes = [c_char_p, c_void_p, c_uint64, c_void_p, c_void_p]
        lib.ref_parse_setup.restype = c_int
        lib.ref_parse_setup.argtypes = [c_char_p, c_void_p, c_uint64, c_void_p]
        lib.ref_npy_u16.restype = c_int
        lib.ref_npy_u16.argtypes = [c_char_p, c_void_p, c_uint64, c_void_p]
        _ref = lib
    return _ref


class ReferenceError_(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"reference error {code}: {message}")
        self.code = code


def _ref_check(code: int) -> None:
    if code != 0:
        raise ReferenceError_(code, ref_lib().ref_last_error().decode())


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------ restatement
def sample(probs, repetitions: int, seed: int):
    """(cols, mult, invp, engine_state) — coordinate_sampling.cpp:14-45."""
    p = np.ascontiguousarray(probs, dtype=np.float64)
    d = p.size
    cols = np.empty(d, np.uint64)
    mult = np.empty(d, np.uint64)
    inv = np.empty(d, np.float64)
    state = ctypes.create_string_buffer(1 << 16)
    k = oracle_lib().oracle_sample(_p(p), d, repetitions, seed, _p(cols), _p(mult),
                                   _p(inv), state, len(state))
    if k < 0:
        raise ValueError("invalid sampling probability")
    return cols[:k].copy(), mult[:k].copy(), inv[:k].copy(), state.value.decode()


def jl_matrix(mult, invp, p: int, state: str | None = None, seed: int = 5489):
    k = len(mult)
    out = np.empty((p, k), np.float64)
    oracle_lib().oracle_jl_matrix(_p(np.asarray(mult, np.uint64)),
                                  _p(np.asarray(invp, np.float64)), k, p,
                                  state.encode() if state else None, seed, _p(out))
    return out


def cauchy_matrix(mult, invp, p: int, state: str | None = None, seed: int = 5489):
    k = len(mult)
    out = np.empty((p, k), np.float64)
    oracle_lib().oracle_cauchy_matrix(_p(np.asarray(mult, np.uint64)),
                                      _p(np.asarray(invp, np.float64)), k, p,
                                      state.encode() if state else None, seed, _p(out))
    return out


def exact(metric: str, rows, queries):
    """(indices, binary64 distances) of ExactL2Index / ExactL1Index."""
    rows = _f32(rows)
    q = _f32(queries).reshape(-1, rows.shape[1])
    out = np.zeros(q.shape[0], np.uint64)
    dist = np.zeros(q.shape[0], np.float64)
    fn = oracle_lib().oracle_exact_l2 if metric == "l2" else oracle_lib().oracle_exact_l1
    fn(_p(rows), rows.shape[0], rows.shape[1], _p(q), q.shape[0], _p(out), _p(dist))
    return out, dist


def weighted_l1(rows, weights, queries):
    rows = _f32(rows)
    q = _f32(queries).reshape(-1, rows.shape[1])
    w = _f32(weights)
    out = np.zeros(q.shape[0], np.uint64)
    dist = np.zeros(q.shape[0], np.float64)
    oracle_lib().oracle_weighted_l1(_p(rows), rows.shape[0], rows.shape[1], _p(w),
                                    _p(q), q.shape[0], _p(out), _p(dist))
    return out, dist


def flat(metric: str, rows, cols, mult, invp, queries):
    rows = _f32(rows)
    q = _f32(queries).reshape(-1, rows.shape[1])
    cols = np.ascontiguousarray(cols, np.uint64)
    mult = np.ascontiguousarray(mult, np.uint64)
    invp = np.ascontiguousarray(invp, np.float64)
    out = np.zeros(q.shape[0], np.uint64)
    dist = np.zeros(q.shape[0], np.float64)
    fn = oracle_lib().oracle_flat_l2 if metric == "l2" else oracle_lib().oracle_flat_l1
    status = fn(_p(rows), rows.shape[0], rows.shape[1], _p(cols), _p(mult), _p(invp),
                cols.size, _p(q), q.shape[0], _p(out), _p(dist))
    if status != 0:
        raise ValueError("sampled query coordinate must be finite")
    return out, dist


def project_rows(rows, cols, proj):
    rows = _f32(rows)
    cols = np.ascontiguousarray(cols, np.uint64)
    proj = np.ascontiguousarray(proj, np.float64)
    out = np.empty((rows.shape[0], proj.shape[0]), np.float64)
    oracle_lib().oracle_project_rows(_p(rows), rows.shape[0], rows.shape[1], _p(cols),
                                     cols.size, _p(proj), proj.shape[0], _p(out))
    return out


def hierarchical(metric: str, rows, cols, proj, queries):
    rows = _f32(rows)
    reps = project_rows(rows, cols, proj)
    q = _f32(queries).reshape(-1, rows.shape[1])
    cols = np.ascontiguousarray(cols, np.uint64)
    proj = np.ascontiguousarray(proj, np.float64)
    out = np.zeros(q.shape[0], np.uint64)
    dist = np.zeros(q.shape[0], np.float64)
    fn = oracle_lib().oracle_hier_l2 if metric == "l2" else oracle_lib().oracle_hier_l1
    status = fn(_p(reps), rows.shape[0], _p(q), q.shape[0], rows.shape[1], _p(cols),
                cols.size, _p(proj), proj.shape[0], _p(out), _p(dist))
    if status == -1:
        raise ValueError("sampled query coordinate must be finite")
    if status == -2:
        raise OverflowError("projected query is not finite")
    return out, dist


def probabilities(metric: str, rows):
    rows = _f32(rows)
    out = np.zeros(rows.shape[1], np.float64)
    oracle_lib().oracle_probabilities(0 if metric == "l2" else 1, _p(rows),
                                      rows.shape[0], rows.shape[1], _p(out))
    return out


# -------------------------------------------------------------- reference
def ref_sample(probs, repetitions: int, seed: int):
    p = np.ascontiguousarray(probs, dtype=np.float64)
    d = p.size
    cols = np.empty(d, np.uint64)
    mult = np.empty(d, np.uint64)
    inv = np.empty(d, np.float64)
    k = c_uint64()
    state = ctypes.create_string_buffer(1 << 16)
    _ref_check(ref_lib().ref_sample(_p(p), d, repetitions, seed, _p(cols), _p(mult),
                                    _p(inv), ctypes.byref(k), state, len(state)))
    n = k.value
    return cols[:n].copy(), mult[:n].copy(), inv[:n].copy(), state.value.decode()


def ref_probabilities(metric: str, rows, parallel: bool = True):
    rows = _f32(rows)
    out = np.zeros(rows.shape[1], np.float64)
    _ref_check(ref_lib().ref_probabilities(0 if metric == "l2" else 1, _p(rows),
                                           rows.shape[0], rows.shape[1],
                                           1 if parallel else 0, _p(out)))
    return out


def ref_exact(metric: str, rows, queries, threads: int = 1):
    """ExactL2Index::query_batch (parallel_queries when threads > 1) or
    ExactL1Index::query on `threads` threads."""
    rows = _f32(rows)
    q = _f32(queries).reshape(-1, rows.shape[1])
    out = np.zeros(q.shape[0], np.uint64)
    if metric == "l2":
        _ref_check(ref_lib().ref_exact_l2(_p(rows), rows.shape[0], rows.shape[1], _p(q),
                                          q.shape[0], 1 if threads > 1 else 0, _p(out)))
    else:
        _ref_check(ref_lib().ref_exact_l1(_p(rows), rows.shape[0], rows.shape[1], _p(q),
                                          q.shape[0], threads, _p(out)))
    return out


class RefExactIndex:
    """A persistent reference ExactL2Index / ExactL1Index (CPU)."""

    def __init__(self, metric: str, rows):
        self._rows = _f32(rows)
        self.dimension = self._rows.shape[1]
        self._h = ref_lib().ref_exact_create(0 if metric == "l2" else 1, _p(self._rows),
                                             self._rows.shape[0], self._rows.shape[1])
        if not self._h:
            raise ReferenceError_(1, ref_lib().ref_last_error().decode())

    def query_batch(self, queries, threads: int) -> np.ndarray:
        q = _f32(queries).reshape(-1, self.dimension)
        out = np.zeros(q.shape[0], np.uint64)
        _ref_check(ref_lib().ref_exact_query(self._h, _p(q), q.shape[0], threads,
                                             _p(out)))
        return out

    def query_in_batches(self, queries, batch: int, threads: int) -> np.ndarray:
        """L2: query_batch calls of `batch` queries with the reference's
        automatic strategy (parallel over rows for one query)."""
        q = _f32(queries).reshape(-1, self.dimension)
        out = np.zeros(q.shape[0], np.uint64)
        _ref_check(ref_lib().ref_exact_query_batched(self._h, _p(q), q.shape[0], batch,
                                                     threads, _p(out)))
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            ref_lib().ref_exact_destroy(self._h)
            self._h = None


def ref_sampled(metric: str, rows, cols, mult, invp, queries, threads: int = 1):
    rows = _f32(rows)
    q = _f32(queries).reshape(-1, rows.shape[1])
    cols = np.ascontiguousarray(cols, np.uint64)
    mult = np.ascontiguousarray(mult, np.uint64)
    invp = np.ascontiguousarray(invp, np.float64)
    out = np.zeros(q.shape[0], np.uint64)
    fn = ref_lib().ref_sampled_l2 if metric == "l2" else ref_lib().ref_sampled_l1
    arg = (1 if threads > 1 else 0) if metric == "l2" else threads
    _ref_check(fn(_p(rows), rows.shape[0], rows.shape[1], _p(cols), _p(mult), _p(invp),
                  cols.size, _p(q), q.shape[0], arg, _p(out)))
    return out


def ref_hierarchical(metric: str, rows, probs, repetitions: int, p: int, seed: int,
                     queries, threads: int = 1):
    """(indices, engine state after construction)."""
    rows = _f32(rows)
    q = _f32(queries).reshape(-1, rows.shape[1])
    pr = np.ascontiguousarray(probs, np.float64)
    out = np.zeros(q.shape[0], np.uint64)
    state = ctypes.create_string_buffer(1 << 16)
    _ref_check(ref_lib().ref_hierarchical(0 if metric == "l2" else 1, _p(rows),
                                          rows.shape[0], rows.shape[1], _p(pr),
                                          repetitions, p, seed, _p(q), q.shape[0],
                                          threads, _p(out), state, len(state)))
    return out, state.value.decode()


def ref_projection(metric: str, rows, cols, mult, invp, p: int, state: str | None,
                   seed: int = 5489):
    rows = _f32(rows)
    cols = np.ascontiguousarray(cols, np.uint64)
    mult = np.ascontiguousarray(mult, np.uint64)
    invp = np.ascontiguousarray(invp, np.float64)
    mat = np.empty((p, cols.size), np.float64)
    reps = np.empty((rows.shape[0], p), np.float64)
    _ref_check(ref_lib().ref_projection(0 if metric == "l2" else 1, _p(rows),
                                        rows.shape[0], rows.shape[1], _p(cols), _p(mult),
                                        _p(invp), cols.size, p,
                                        state.encode() if state else None, seed,
                                        _p(mat), _p(reps)))
    return mat, reps


def ref_hierarchical_sampled(metric: str, sampled_rows, mult, invp, p: int, state: str,
                             sampled_queries, threads: int = 1) -> np.ndarray:
    """The reference's hierarchical index (its own constructor and query())
    over the r x k sampled columns with the sample renumbered 0..k-1; equal to
    the index over the full matrix (ref_hier_capi.cpp)."""
    lib = ref_lib()
    if not getattr(lib, "_hier_typed", False):
        lib.ref_hier_last_error.restype = c_char_p
        lib.ref_hierarchical_sampled.restype = c_int
        lib.ref_hierarchical_sampled.argtypes = [c_int, c_void_p, c_uint64, c_uint64,
                                                 c_void_p, c_void_p, c_uint64, c_char_p,
                                                 c_void_p, c_uint64, c_int, c_void_p]
        lib._hier_typed = True
    rows = _f32(sampled_rows)
    q = _f32(sampled_queries).reshape(-1, rows.shape[1])
    mult = np.ascontiguousarray(mult, np.uint64)
    invp = np.ascontiguousarray(invp, np.float64)
    out = np.zeros(q.shape[0], np.uint64)
    code = lib.ref_hierarchical_sampled(0 if metric == "l2" else 1, _p(rows),
                                        rows.shape[0], rows.shape[1], _p(mult), _p(invp),
                                        p, state.encode(), _p(q), q.shape[0], threads,
                                        _p(out))
    if code != 0:
        raise ReferenceError_(code, lib.ref_hier_last_error().decode())
    return out


# ------------------------------------------------- reference data-file code

def ref_sha256_file(path) -> bytes:
    out = (ctypes.c_uint8 * 32)()
    _ref_check(ref_lib().ref_sha256_file(str(path).encode(), out))
    return bytes(out)


def ref_probabilities_save(path, kind: int, reps: int, sha: bytes, probs) -> None:
    """kind: 0 = L2, 1 = L1."""
    p = np.ascontiguousarray(probs, np.float64)
    d = (ctypes.c_uint8 * 32)(*sha)
    _ref_check(ref_lib().ref_probabilities_save(str(path).encode(), kind, reps, d, _p(p),
                                                p.size))


def ref_probabilities_load(path):
    kind = ctypes.c_int()
    reps = ctypes.c_uint64()
    n = ctypes.c_uint64()
    d = (ctypes.c_uint8 * 32)()
    _ref_check(ref_lib().ref_probabilities_load(str(path).encode(), ctypes.byref(kind),
                                                ctypes.byref(reps), d, None, 0,
                                                ctypes.byref(n)))
    out = np.zeros(n.value, np.float64)
    _ref_check(ref_lib().ref_probabilities_load(str(path).encode(), ctypes.byref(kind),
                                                ctypes.byref(reps), d, _p(out), out.size,
                                                ctypes.byref(n)))
    return kind.value, reps.value, bytes(d), out


def ref_npy_f32(path) -> np.ndarray:
    r = ctypes.c_uint64()
    c = ctypes.c_uint64()
    _ref_check(ref_lib().ref_npy_f32(str(path).encode(), None, 0, ctypes.byref(r),
                                     ctypes.byref(c)))
    out = np.zeros((r.value, c.value), np.float32)
    _ref_check(ref_lib().ref_npy_f32(str(path).encode(), _p(out), out.size, ctypes.byref(r),
                                     ctypes.byref(c)))
    return out


def ref_npy_u16(path) -> np.ndarray:
    n = ctypes.c_uint64()
    _ref_check(ref_lib().ref_npy_u16(str(path).encode(), None, 0, ctypes.byref(n)))
    out = np.zeros(n.value, np.uint64)
    _ref_check(ref_lib().ref_npy_u16(str(path).encode(), _p(out), out.size, ctypes.byref(n)))
    return out


def ref_parse_setup(path) -> dict:
    """The reference's load_benchmark_setup of a setup file, as a dict."""
    import json
    n = ctypes.c_uint64()
    _ref_check(ref_lib().ref_parse_setup(str(path).encode(), None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    _ref_check(ref_lib().ref_parse_setup(str(path).encode(), buf, n.value + 1,
                                         ctypes.byref(n)))
    return json.loads(buf.value.decode())
