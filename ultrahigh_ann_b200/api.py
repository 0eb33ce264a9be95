"""Python mirror of the reference's CUDA index API over the engine's C ABI.

Class and method names, argument meaning and error types follow the
reference's C++ headers under include/ultrahigh_ann/ (for example
core/cuda_dense_l2_scan_index.hpp, coordinate_sampling/
cuda_sampled_coordinate_l2_ann_index.hpp, hnsvw25/l2/flat/cuda_l2_ann_index.hpp,
hnsvw25/l2/hierarchical/cuda_hierarchical_l2_ann_index.hpp). C++ exception
types map onto Python exceptions:

    std::invalid_argument -> InvalidArgument     std::length_error -> LengthError
    std::runtime_error    -> CudaRuntimeError    std::overflow_error -> ResultOverflowError
    std::out_of_range     -> OutOfRange          std::domain_error -> DomainError
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi


class InvalidArgument(ValueError):
    """std::invalid_argument."""


class LengthError(ValueError):
    """std::length_error."""


class CudaRuntimeError(RuntimeError):
    """std::runtime_error (CUDA failure or no usable device)."""


class ResultOverflowError(OverflowError):
    """std::overflow_error (non-finite projected or median results)."""


class OutOfRange(IndexError):
    """std::out_of_range."""


class DomainError(ValueError):
    """std::domain_error."""


class LogicError(RuntimeError):
    """std::logic_error."""


_ERRORS = {
    _abi.INVALID_ARGUMENT: InvalidArgument,
    _abi.LENGTH_ERROR: LengthError,
    _abi.RUNTIME_ERROR: CudaRuntimeError,
    _abi.OVERFLOW_ERROR: ResultOverflowError,
    _abi.OUT_OF_RANGE: OutOfRange,
    _abi.DOMAIN_ERROR: DomainError,
    _abi.LOGIC_ERROR: LogicError,
}


def _check(status: int) -> None:
    if status != _abi.OK:
        message = _abi.load().uha_last_error().decode(errors="replace")
        raise _ERRORS.get(status, CudaRuntimeError)(message)


def _ptr(array: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(array.ctypes.data) if array.size else ctypes.c_void_p(0)


class QueryStrategy(enum.IntEnum):
    """CudaDenseL2QueryStrategy and siblings
    (include/ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp:17-23)."""

    direct = _abi.DIRECT
    gemm = _abi.GEMM
    # precision forms (appended; exact, flat and hierarchical L2 indexes):
    # tensor-core scores of rounded rows/queries (hierarchies: and of the
    # projection), then a binary64 re-score of the best candidates per query
    # (QueryWorkspace.set_candidates)
    gemm_bf16_rerank = _abi.GEMM_BF16_RERANK
    gemm_fp8_rerank = _abi.GEMM_FP8_RERANK
    # the same scores and candidates re-scored in binary32 with a certified
    # bound, near-ties settled without FP64 instructions (exact and flat L2)
    gemm_bf16_rerank_fp32 = _abi.GEMM_BF16_RERANK_FP32
    gemm_fp8_rerank_fp32 = _abi.GEMM_FP8_RERANK_FP32


CudaDenseL2QueryStrategy = QueryStrategy
CudaExactL2QueryStrategy = QueryStrategy
CudaSampledCoordinateL2QueryStrategy = QueryStrategy
CudaHierarchicalL2QueryStrategy = QueryStrategy
CudaHierarchicalL1QueryStrategy = QueryStrategy


class ExecutionPolicy(enum.Enum):
    """include/ultrahigh_ann/hnsvw25/execution_policy.hpp:7-12. The engine
    builds probabilities on the device for the gpu policies."""

    sequential = "sequential"
    cpu_parallel = "cpu_parallel"
    gpu_fp32 = "gpu_fp32"
    gpu_cublas_fp32 = "gpu_cublas_fp32"


@dataclass(frozen=True)
class IndexSpaceUsage:
    """include/ultrahigh_ann/core/index_space_usage.hpp:9-14."""

    index_payload_bytes: int
    query_workspace_payload_bytes: int
    unique_query_coordinates: int
    sampled_multiplicity: int


@dataclass(frozen=True)
class CudaRuntimeInfo:
    """include/ultrahigh_ann/core/cuda_runtime_info.hpp:9-18."""

    device: int
    device_name: str
    compute_capability_major: int
    compute_capability_minor: int
    total_global_memory_bytes: int
    compiled_runtime_version: int
    runtime_version: int
    driver_version: int


def cuda_runtime_info(device: int = 0) -> Optional[CudaRuntimeInfo]:
    """Device metadata, or None without a usable device
    (include/ultrahigh_ann/core/cuda_runtime_info.hpp:20-23)."""
    info = _abi.DeviceInfo()
    if _abi.load().uha_device_info_get(device, ctypes.byref(info)) != _abi.OK:
        return None
    return CudaRuntimeInfo(info.device, info.device_name.decode(),
                           info.compute_capability_major,
                           info.compute_capability_minor,
                           info.total_global_memory_bytes,
                           info.compiled_runtime_version, info.runtime_version,
                           info.driver_version)


def cuda_available() -> bool:
    return bool(_abi.load().uha_cuda_available())


class MT19937_64:
    """std::mt19937_64 shared by the host-side draws (sampling, projections).
    The default seed is the standard's 5489."""

    def __init__(self, seed: int = 5489):
        handle = ctypes.c_void_p()
        _check(_abi.load().uha_rng_create(ctypes.c_uint64(seed), ctypes.byref(handle)))
        self._handle = handle

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle:
            self._handle = None
            try:
                _abi.load().uha_rng_destroy(handle)
            except Exception:  # interpreter shutdown: the module is gone
                pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._handle

    def state(self) -> str:
        lib = _abi.load()
        length = ctypes.c_uint64()
        _check(lib.uha_rng_state(self._handle, None, 0, ctypes.byref(length)))
        buf = ctypes.create_string_buffer(length.value)
        _check(lib.uha_rng_state(self._handle, buf, length.value, ctypes.byref(length)))
        return buf.value.decode()

    def set_state(self, state: str) -> None:
        _check(_abi.load().uha_rng_set_state(self._handle, state.encode()))

    def __eq__(self, other: object) -> bool:
        return isinstance(other, MT19937_64) and self.state() == other.state()


@dataclass(frozen=True)
class SampledColumn:
    """include/ultrahigh_ann/coordinate_sampling/coordinate_sample.hpp:10-14."""

    source_column: int
    multiplicity: int
    inverse_probability: float


class CoordinateSample:
    """The multiset I as three parallel arrays in ascending column order
    (include/ultrahigh_ann/coordinate_sampling/coordinate_sample.hpp:16-18)."""

    def __init__(self, columns=(), multiplicities=(), inverse_probabilities=()):
        self.source_columns = np.ascontiguousarray(columns, dtype=np.uint64)
        self.multiplicities = np.ascontiguousarray(multiplicities, dtype=np.uint64)
        self.inverse_probabilities = np.ascontiguousarray(inverse_probabilities,
                                                          dtype=np.float64)
        if not (self.source_columns.shape == self.multiplicities.shape
                == self.inverse_probabilities.shape):
            raise InvalidArgument("coordinate sample arrays differ in length")

    @classmethod
    def from_columns(cls, columns) -> "CoordinateSample":
        cols = list(columns)
        return cls([c.source_column for c in cols], [c.multiplicity for c in cols],
                   [c.inverse_probability for c in cols])

    @property
    def columns(self) -> list[SampledColumn]:
        return [SampledColumn(int(c), int(m), float(p)) for c, m, p in
                zip(self.source_columns, self.multiplicities, self.inverse_probabilities)]

    def __len__(self) -> int:
        return int(self.source_columns.size)

    def sampled_multiplicity(self) -> int:
        return int(self.multiplicities.sum())


def build_coordinate_sample(probabilities, repetitions: int,
                            random_engine: MT19937_64) -> CoordinateSample:
    """include/ultrahigh_ann/coordinate_sampling/coordinate_sampling.hpp:13-16."""
    p = np.ascontiguousarray(probabilities, dtype=np.float64)
    d = p.size
    cols = np.empty(d, dtype=np.uint64)
    mult = np.empty(d, dtype=np.uint64)
    inv = np.empty(d, dtype=np.float64)
    k = ctypes.c_uint64()
    _check(_abi.load().uha_sample_coordinates(
        _ptr(p), d, ctypes.c_uint64(repetitions), random_engine.handle,
        _ptr(cols), _ptr(mult), _ptr(inv), ctypes.byref(k)))
    n = k.value
    return CoordinateSample(cols[:n], mult[:n], inv[:n])


build_l2_importance_sample = build_coordinate_sample
build_l1_importance_sample = build_coordinate_sample


def build_jl_matrix(sample: CoordinateSample, projection_dimension: int,
                    random_engine: MT19937_64) -> np.ndarray:
    """p x k aggregated Rademacher-JL matrix in the reference's draw order
    (src/hnsvw25/l2/hierarchical/l2_hierarchical_projection.cpp:53-77)."""
    out = np.empty((projection_dimension, len(sample)), dtype=np.float64)
    _check(_abi.load().uha_jl_matrix(
        _ptr(sample.multiplicities), _ptr(sample.inverse_probabilities),
        len(sample), projection_dimension, random_engine.handle, _ptr(out)))
    return out


def build_gaussian_jl_matrix(sample: CoordinateSample, projection_dimension: int,
                             random_engine: MT19937_64) -> np.ndarray:
    """p x k Gaussian JL matrix with binary32 entries Z * sqrt(m (1/p) / p),
    the variance of the aggregated Rademacher entry (uha_gaussian_jl_matrix);
    an extra projection mode, not in the reference."""
    out = np.empty((projection_dimension, len(sample)), dtype=np.float64)
    _check(_abi.load().uha_gaussian_jl_matrix(
        _ptr(sample.multiplicities), _ptr(sample.inverse_probabilities),
        len(sample), projection_dimension, random_engine.handle, _ptr(out)))
    return out


def build_cauchy_matrix(sample: CoordinateSample, projection_dimension: int,
                        random_engine: MT19937_64) -> np.ndarray:
    """p x k Cauchy matrix in the reference's draw order
    (src/hnsvw25/l1/hierarchical/l1_hierarchical_projection.cpp:54-77)."""
    out = np.empty((projection_dimension, len(sample)), dtype=np.float64)
    _check(_abi.load().uha_cauchy_matrix(
        _ptr(sample.multiplicities), _ptr(sample.inverse_probabilities),
        len(sample), projection_dimension, random_engine.handle, _ptr(out)))
    return out


@dataclass
class ProbabilityResult:
    """L{1,2}GpuProbabilityResult (include/ultrahigh_ann/hnsvw25/l2/
    importance_sampling.hpp:31-41)."""

    probabilities: np.ndarray
    device_name: str
    device: int
    pair_count: int
    pair_chunks: int
    device_working_set_bytes: int
    host_to_device_ms: float
    inverse_distance_ms: float
    coordinate_maximum_ms: float
    device_to_host_ms: float
    total_ms: float


def _matrix(values) -> np.ndarray:
    if isinstance(values, DeviceMatrix) or _is_cuda_tensor(values):
        raise InvalidArgument("this operation needs a host representative matrix")
    m = np.ascontiguousarray(values, dtype=np.float32)
    if m.ndim != 2:
        raise InvalidArgument("representative matrix must be two-dimensional")
    return m


def _is_cuda_tensor(values) -> bool:
    return type(values).__module__.startswith("torch") and \
        getattr(getattr(values, "device", None), "type", None) == "cuda"


@dataclass(frozen=True)
class DeviceMatrix:
    """A row-major representative matrix already on a CUDA device: row i
    starts at element i * row_stride of `pointer`; values binary32 or BF16
    (decoded exactly). Index constructors given one read it on the device
    (uha_*_index_create_device) instead of copying a host matrix; only the
    sampled columns are read by sampled and hierarchical indexes. The memory
    must stay valid while the constructor runs."""
    pointer: int
    rows: int
    columns: int
    dtype: str = "float32"
    row_stride: Optional[int] = None

    @classmethod
    def from_torch(cls, tensor) -> "DeviceMatrix":
        import torch
        if tensor.dim() != 2 or tensor.device.type != "cuda":
            raise InvalidArgument("a device matrix is a two-dimensional CUDA tensor")
        if tensor.dtype not in (torch.float32, torch.bfloat16) or tensor.stride(1) != 1:
            raise InvalidArgument("a device matrix holds float32 or bfloat16 rows "
                                  "with unit column stride")
        return cls(tensor.data_ptr(), tensor.shape[0], tensor.shape[1],
                   "bfloat16" if tensor.dtype == torch.bfloat16 else "float32",
                   tensor.stride(0))

    @property
    def shape(self) -> tuple:
        return (self.rows, self.columns)

    def _struct(self) -> "_abi.DeviceMatrix":
        if self.dtype not in ("float32", "bfloat16"):
            raise InvalidArgument("a device matrix holds float32 or bfloat16 values")
        return _abi.DeviceMatrix(ctypes.c_void_p(int(self.pointer)),
                                 _abi.VALUES_BF16 if self.dtype == "bfloat16"
                                 else _abi.VALUES_F32,
                                 int(self.rows), int(self.columns),
                                 int(self.columns if self.row_stride is None
                                     else self.row_stride))


def _rows_input(values):
    """A host matrix (as binary32 numpy) or a DeviceMatrix."""
    if isinstance(values, DeviceMatrix):
        return values
    if _is_cuda_tensor(values):
        return DeviceMatrix.from_torch(values)
    return _matrix(values)


def _probabilities_gpu(metric: int, representatives, device: int,
                       gram: bool = False, pair_chunks: int = 128,
                       maxima: str = "binary64") -> ProbabilityResult:
    if maxima not in ("binary64", "binary32"):
        raise InvalidArgument("column maxima are binary64 or binary32")
    single = maxima == "binary32"
    backend = ((_abi.PAIRS_GRAM_MAX32 if single else _abi.PAIRS_GRAM) if gram
               else (_abi.PAIRS_DIRECT_MAX32 if single else _abi.PAIRS_DIRECT))
    rep = _abi.ProbabilityReport()
    if isinstance(representatives, DeviceMatrix) or _is_cuda_tensor(representatives):
        # a matrix on the device: no host copy (float32, densely packed rows)
        m = _rows_input(representatives)
        if m.dtype != "float32" or (m.row_stride not in (None, m.columns)):
            raise InvalidArgument("device representatives must be dense float32 rows")
        out = np.zeros(int(m.columns), dtype=np.float64)
        _check(_abi.load().uha_importance_probabilities_device(
            device, metric, ctypes.c_void_p(int(m.pointer)), int(m.rows), int(m.columns),
            backend, ctypes.c_uint64(pair_chunks), _ptr(out), ctypes.byref(rep)))
    else:
        rows = _matrix(representatives)
        out = np.zeros(rows.shape[1], dtype=np.float64)
        _check(_abi.load().uha_importance_probabilities(
            device, metric, _ptr(rows), rows.shape[0], rows.shape[1], backend,
            ctypes.c_uint64(pair_chunks), _ptr(out), ctypes.byref(rep)))
    info = cuda_runtime_info(device)
    return ProbabilityResult(out, info.device_name if info else "", device,
                             rep.pair_count, rep.pair_chunks, rep.device_working_set_bytes,
                             rep.host_to_device_ms, rep.inverse_distance_ms,
                             rep.coordinate_maximum_ms, rep.device_to_host_ms,
                             rep.total_ms)


def compute_l2_importance_probabilities_gpu(representatives, device: int = 0,
                                            pair_chunks: int = 128,
                                            distance_backend: str = "direct",
                                            maxima: str = "binary64"
                                            ) -> ProbabilityResult:
    """include/ultrahigh_ann/hnsvw25/l2/importance_sampling.hpp:49-52;
    distance_backend "direct" or "gram" (the reference's "cublas" backend).
    Appended: representatives may be a DeviceMatrix or CUDA tensor (no host
    copy), and maxima="binary32" forms the per-column maxima in binary32
    (within 3e-7 relative; for full-size builds)."""
    if pair_chunks <= 0:
        raise InvalidArgument("GPU pair chunk count must be positive")
    if distance_backend not in ("direct", "gram", "cublas"):
        raise InvalidArgument("unknown L2 GPU distance backend")
    return _probabilities_gpu(_abi.L2, representatives, device,
                              gram=distance_backend != "direct", pair_chunks=pair_chunks,
                              maxima=maxima)


def compute_l1_importance_probabilities_gpu(representatives, device: int = 0,
                                            pair_chunks: int = 128,
                                            maxima: str = "binary64") -> ProbabilityResult:
    """include/ultrahigh_ann/hnsvw25/l1/importance_sampling.hpp:45-48 (device
    input and binary32 maxima as for L2)."""
    if pair_chunks <= 0:
        raise InvalidArgument("GPU pair chunk count must be positive")
    return _probabilities_gpu(_abi.L1, representatives, device, pair_chunks=pair_chunks,
                              maxima=maxima)


def _tune_dict(r) -> dict:
    kernel = ("stream", "tile", "tensor", "median")[r.kernel] if r.candidates else "fixed"
    return {"candidates": r.candidates, "kernel": kernel,
            "queries_per_pass": r.queries_per_pass, "tile_queries": r.tile_queries,
            "splits": r.splits, "best_ms": r.best_ms, "default_ms": r.default_ms}


class QueryWorkspace:
    """Per-caller device buffers sized for a maximum batch
    (e.g. include/ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp:28-45)."""

    def __init__(self, index: "_CudaIndex", maximum_batch_size: int):
        handle = ctypes.c_void_p()
        if maximum_batch_size < 0:
            raise InvalidArgument("workspace batch size must be positive")
        _check(_abi.load().uha_workspace_create(index._handle,
                                                ctypes.c_uint64(maximum_batch_size),
                                                ctypes.byref(handle)))
        self._handle = handle
        self._index = index  # keeps the index alive while the workspace lives

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle:
            self._handle = None
            try:
                _abi.load().uha_workspace_destroy(handle)
            except Exception:  # interpreter shutdown: the module is gone
                pass

    def maximum_batch_size(self) -> int:
        b = ctypes.c_uint64()
        _check(_abi.load().uha_workspace_info(self._handle, ctypes.byref(b), None))
        return b.value

    def payload_bytes(self) -> int:
        p = ctypes.c_uint64()
        _check(_abi.load().uha_workspace_info(self._handle, None, ctypes.byref(p)))
        return p.value

    def last_stats(self) -> dict:
        s = _abi.QueryStats()
        _check(_abi.load().uha_workspace_last_stats(self._handle, ctypes.byref(s)))
        return {"query_count": s.query_count, "certified_queries": s.certified_queries,
                "replayed_queries": s.replayed_queries,
                "kernel_launches": s.kernel_launches, "scan_ms": s.scan_ms,
                "device_ms": s.device_ms, "timed_scans": s.timed_scans}

    def stream_handle(self) -> int:
        """cudaStream_t of the workspace as an integer."""
        return int(_abi.load().uha_workspace_stream(self._handle) or 0)

    def set_timing(self, enabled, stride: int = 1) -> None:
        """Records CUDA events around the device pipeline of every call and
        around the scan kernel of every stride-th batch (see last_stats():
        scan_ms covers timed_scans launches)."""
        value = int(stride) if enabled else 0
        if enabled and value < 1:
            raise InvalidArgument("timing stride must be positive")
        _check(_abi.load().uha_workspace_set_timing(self._handle, value))

    def autotune(self, batch: int, strategy=QueryStrategy.direct) -> dict:
        """Times every candidate scan shape for batches of exactly `batch`
        queries and keeps the fastest for this workspace."""
        r = _abi.TuneReport()
        _check(_abi.load().uha_workspace_autotune(self._handle, ctypes.c_uint64(batch),
                                                  int(strategy), ctypes.byref(r)))
        return _tune_dict(r)

    def set_replay(self, emulated: bool) -> None:
        """Arithmetic of the certified path's replay on exact and flat
        indexes: binary64 on the FP64 units (default) or, with emulated=True,
        no FP64 instruction (float-float, then emulated binary64). Both give
        the reference CPU's row."""
        _check(_abi.load().uha_workspace_set_replay(
            self._handle, _abi.REPLAY_EMULATED if emulated else _abi.REPLAY_BINARY64))

    def set_candidates(self, candidates: int) -> None:
        """Candidates per query re-scored by the precision strategies (1-64)."""
        if not 1 <= int(candidates) <= 64:
            raise InvalidArgument("candidate count must be between 1 and 64")
        _check(_abi.load().uha_workspace_set_candidates(self._handle,
                                                        ctypes.c_uint32(int(candidates))))


class _CudaIndex:
    _handle: ctypes.c_void_p = None
    _dimension: int = 0

    def _adopt(self, handle: ctypes.c_void_p, dimension: int, rows: int) -> None:
        self._handle = handle
        self._dimension = dimension
        self._rows = rows

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle:
            self._handle = None
            try:
                _abi.load().uha_index_destroy(handle)
            except Exception:  # interpreter shutdown: the module is gone
                pass

    @property
    def dimension(self) -> int:
        return self._dimension

    @property
    def row_count(self) -> int:
        return self._rows

    def make_query_workspace(self, maximum_batch_size: int) -> QueryWorkspace:
        return QueryWorkspace(self, maximum_batch_size)

    def _run(self, queries_ptr: int, query_count: int, on_device: bool,
             output: np.ndarray, workspace: QueryWorkspace, strategy,
             distances: Optional[np.ndarray]) -> None:
        if not isinstance(workspace, QueryWorkspace):
            raise InvalidArgument("CUDA workspace belongs to a different index")
        dist_ptr = ctypes.c_void_p(distances.ctypes.data) if distances is not None else None
        _check(_abi.load().uha_query(self._handle, workspace._handle,
                                     ctypes.c_void_p(queries_ptr),
                                     ctypes.c_uint64(query_count), int(on_device),
                                     int(strategy), ctypes.c_void_p(output.ctypes.data),
                                     dist_ptr))

    def query_batch(self, queries, query_count: int, output,
                    workspace: QueryWorkspace, strategy=QueryStrategy.direct,
                    distances: Optional[np.ndarray] = None) -> np.ndarray:
        """Row-major query_count x dimension host queries; output receives one
        row index per query (a writable uint64 array of query_count entries,
        or None to allocate one). Returns the output array."""
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1)
        if q.size != query_count * self._dimension:
            raise InvalidArgument("query batch dimensions do not match index dimension")
        out = self._output(output, query_count)
        if distances is not None and (distances.dtype != np.float64
                                      or distances.size != query_count):
            raise InvalidArgument("distance output must be float64 of query_count")
        self._run(q.ctypes.data if q.size else 0, query_count, False, out,
                  workspace, strategy, distances)
        return out

    def query_device_batch(self, device_queries: int, query_count: int, output,
                           workspace: QueryWorkspace, strategy=QueryStrategy.direct,
                           distances: Optional[np.ndarray] = None) -> np.ndarray:
        """device_queries is a device pointer (int) to a row-major
        query_count x dimension float matrix on this index's device."""
        out = self._output(output, query_count)
        self._run(int(device_queries), query_count, True, out, workspace, strategy,
                  distances)
        return out

    def query_many(self, queries, query_count: int, batch: int, output,
                   workspace: QueryWorkspace, strategy=QueryStrategy.direct,
                   distances: Optional[np.ndarray] = None,
                   on_device: bool = False) -> np.ndarray:
        """query_count queries answered in consecutive batches of `batch`
        (each batch exactly as one query_batch call), enqueued back to back
        and synchronised once. `queries` is a host array, or a device pointer
        (int) when on_device."""
        if not isinstance(workspace, QueryWorkspace):
            raise InvalidArgument("CUDA workspace belongs to a different index")
        out = self._output(output, query_count)
        if on_device:
            ptr = int(queries)
        else:
            q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1)
            if q.size != query_count * self._dimension:
                raise InvalidArgument("query batch dimensions do not match index dimension")
            ptr = q.ctypes.data if q.size else 0
        dist_ptr = ctypes.c_void_p(distances.ctypes.data) if distances is not None else None
        _check(_abi.load().uha_query_many(self._handle, workspace._handle,
                                          ctypes.c_void_p(ptr), ctypes.c_uint64(query_count),
                                          ctypes.c_uint64(batch), int(on_device),
                                          int(strategy), ctypes.c_void_p(out.ctypes.data),
                                          dist_ptr))
        return out

    def precision_scores(self, queries, query_count: int, workspace: QueryWorkspace,
                         strategy=QueryStrategy.gemm_bf16_rerank):
        """Tensor-core scores of a precision strategy: (scores, norms) with
        scores[q][row] = r~.q~ (FP8: times both scales) and norms[row] =
        ||r~||^2 of the rounded rows."""
        if not isinstance(workspace, QueryWorkspace):
            raise InvalidArgument("CUDA workspace belongs to a different index")
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1)
        if q.size != query_count * self._dimension:
            raise InvalidArgument("query batch dimensions do not match index dimension")
        rows = self.row_count
        scores = np.zeros((query_count, rows), dtype=np.float32)
        norms = np.zeros(rows, dtype=np.float32)
        _check(_abi.load().uha_precision_scores(
            self._handle, workspace._handle, ctypes.c_void_p(q.ctypes.data if q.size else 0),
            ctypes.c_uint64(query_count), int(strategy),
            ctypes.c_void_p(scores.ctypes.data), ctypes.c_void_p(norms.ctypes.data)))
        return scores, norms

    def query(self, query, workspace: QueryWorkspace,
              strategy=QueryStrategy.direct) -> int:
        q = np.ascontiguousarray(query, dtype=np.float32).reshape(-1)
        if q.size != self._dimension:
            raise InvalidArgument("query dimension does not match index dimension")
        return int(self.query_batch(q, 1, None, workspace, strategy)[0])

    @staticmethod
    def _output(output, query_count: int) -> np.ndarray:
        if output is None:
            return np.zeros(query_count, dtype=np.uint64)
        if (not isinstance(output, np.ndarray) or output.dtype != np.uint64
                or output.size != query_count or not output.flags.c_contiguous):
            raise InvalidArgument("CUDA output size does not match query count")
        return output

    def space_usage(self) -> IndexSpaceUsage:
        u = _abi.SpaceUsage()
        _check(_abi.load().uha_index_space_usage(self._handle, ctypes.byref(u)))
        return IndexSpaceUsage(u.index_payload_bytes, u.query_workspace_payload_bytes,
                               u.unique_query_coordinates, u.sampled_multiplicity)

    def device(self) -> int:
        d = ctypes.c_int()
        _check(_abi.load().uha_index_device(self._handle, ctypes.byref(d), None, 0))
        return d.value

    def device_name(self) -> str:
        buf = ctypes.create_string_buffer(256)
        _check(_abi.load().uha_index_device(self._handle, None, buf, 256))
        return buf.value.decode()


class CudaDenseL2ScanIndex(_CudaIndex):
    """include/ultrahigh_ann/core/cuda_dense_l2_scan_index.hpp:27-91."""

    def __init__(self, representatives, device: int = 0):
        rows = _rows_input(representatives)
        handle = ctypes.c_void_p()
        if isinstance(rows, DeviceMatrix):
            _check(_abi.load().uha_exact_index_create_device(
                device, _abi.L2, ctypes.byref(rows._struct()), ctypes.byref(handle)))
        else:
            _check(_abi.load().uha_exact_index_create(device, _abi.L2, _ptr(rows),
                                                      rows.shape[0], rows.shape[1],
                                                      ctypes.byref(handle)))
        self._adopt(handle, rows.shape[1], rows.shape[0])


class CudaExactL2Index(CudaDenseL2ScanIndex):
    """include/ultrahigh_ann/exact/l2/cuda_exact_l2_index.hpp:22-59."""


class CudaDenseL1ScanIndex(_CudaIndex):
    """include/ultrahigh_ann/core/cuda_dense_l1_scan_index.hpp:18-74; the
    weighted form evaluates sum_j w_j |r_j - q_j|."""

    def __init__(self, representatives, coordinate_weights=None, device: int = 0):
        rows = _rows_input(representatives)
        handle = ctypes.c_void_p()
        lib = _abi.load()
        if isinstance(rows, DeviceMatrix):
            if coordinate_weights is not None:
                raise InvalidArgument("coordinate weights need a host representative matrix")
            _check(lib.uha_exact_index_create_device(device, _abi.L1,
                                                     ctypes.byref(rows._struct()),
                                                     ctypes.byref(handle)))
        elif coordinate_weights is None:
            _check(lib.uha_exact_index_create(device, _abi.L1, _ptr(rows),
                                              rows.shape[0], rows.shape[1],
                                              ctypes.byref(handle)))
        else:
            w = np.ascontiguousarray(coordinate_weights, dtype=np.float32).reshape(-1)
            if w.size != rows.shape[1]:
                raise InvalidArgument("coordinate weight dimension does not match")
            _check(lib.uha_weighted_l1_index_create(device, _ptr(rows), rows.shape[0],
                                                    rows.shape[1], _ptr(w),
                                                    ctypes.byref(handle)))
        self._adopt(handle, rows.shape[1], rows.shape[0])

    def query_batch(self, queries, query_count, output, workspace,
                    strategy=QueryStrategy.direct, distances=None):
        return super().query_batch(queries, query_count, output, workspace,
                                   QueryStrategy.direct, distances)


class CudaExactL1Index(CudaDenseL1ScanIndex):
    """include/ultrahigh_ann/exact/l1/cuda_exact_l1_index.hpp:20-54."""

    def __init__(self, representatives, device: int = 0):
        super().__init__(representatives, None, device)


def _resolve_sample(input_rows, probabilities, repetitions,
                    random_engine, coordinate_sample) -> CoordinateSample:
    if coordinate_sample is not None:
        if isinstance(coordinate_sample, CoordinateSample):
            return coordinate_sample
        return CoordinateSample.from_columns(coordinate_sample)
    p = np.ascontiguousarray(probabilities, dtype=np.float64)
    if p.size != input_rows.shape[1]:
        raise InvalidArgument("sampling probability dimension does not match input")
    return build_coordinate_sample(p, repetitions, random_engine)


class _CudaSampledIndex(_CudaIndex):
    _metric = _abi.L2

    def __init__(self, input, probabilities=None, repetitions=None,
                 random_engine=None, device: int = 0, *, coordinate_sample=None):
        rows = _rows_input(input)
        sample = _resolve_sample(rows, probabilities, repetitions, random_engine,
                                 coordinate_sample)
        handle = ctypes.c_void_p()
        sample_args = (_ptr(sample.source_columns), _ptr(sample.multiplicities),
                       _ptr(sample.inverse_probabilities), len(sample),
                       ctypes.byref(handle))
        if isinstance(rows, DeviceMatrix):
            _check(_abi.load().uha_sampled_index_create_device(
                device, self._metric, ctypes.byref(rows._struct()), *sample_args))
        else:
            _check(_abi.load().uha_sampled_index_create(
                device, self._metric, _ptr(rows), rows.shape[0], rows.shape[1],
                *sample_args))
        self._adopt(handle, rows.shape[1], rows.shape[0])
        self.coordinate_sample = sample


class CudaSampledCoordinateL2AnnIndex(_CudaSampledIndex):
    """include/ultrahigh_ann/coordinate_sampling/cuda_sampled_coordinate_l2_ann_index.hpp:23-93."""

    _metric = _abi.L2


class CudaSampledCoordinateL1AnnIndex(_CudaSampledIndex):
    """include/ultrahigh_ann/coordinate_sampling/cuda_sampled_coordinate_l1_ann_index.hpp:20-82."""

    _metric = _abi.L1

    def query_batch(self, queries, query_count, output, workspace,
                    strategy=QueryStrategy.direct, distances=None):
        return super().query_batch(queries, query_count, output, workspace,
                                   QueryStrategy.direct, distances)


def compute_importance_probabilities_host(metric: str, representatives,
                                          threads: int = 0) -> np.ndarray:
    """The reference CPU policies' probabilities on the host cores
    (bit-identical to its sequential loop for any thread count)."""
    import os
    rows = _matrix(representatives)
    out = np.zeros(rows.shape[1], dtype=np.float64)
    _check(_abi.load().uha_importance_probabilities_host(
        _abi.L2 if metric == "l2" else _abi.L1, _ptr(rows), rows.shape[0],
        rows.shape[1], int(threads or os.cpu_count() or 1), _ptr(out)))
    return out


def compute_l2_importance_probabilities(representatives,
                                        execution_policy=ExecutionPolicy.sequential,
                                        device: int = 0) -> np.ndarray:
    """include/ultrahigh_ann/hnsvw25/l2/importance_sampling.hpp:56-58."""
    return _probabilities_for(_abi.L2, _matrix(representatives), execution_policy,
                              device)


def compute_l1_importance_probabilities(representatives,
                                        execution_policy=ExecutionPolicy.sequential,
                                        device: int = 0) -> np.ndarray:
    """include/ultrahigh_ann/hnsvw25/l1/importance_sampling.hpp:52-57."""
    return _probabilities_for(_abi.L1, _matrix(representatives), execution_policy,
                              device)


def _probabilities_for(metric: int, rows: np.ndarray, policy: ExecutionPolicy,
                       device: int) -> np.ndarray:
    if policy in (ExecutionPolicy.gpu_fp32, ExecutionPolicy.gpu_cublas_fp32):
        if metric == _abi.L1 and policy == ExecutionPolicy.gpu_cublas_fp32:
            raise InvalidArgument("gpu_cublas_fp32 is unavailable for L1 probability "
                                  "computation; L1 distance has no "
                                  "matrix-multiplication identity")
        return _probabilities_gpu(metric, rows, device,
                                  gram=policy == ExecutionPolicy.gpu_cublas_fp32
                                  ).probabilities
    threads = 1 if policy == ExecutionPolicy.sequential else 0
    return compute_importance_probabilities_host(
        "l2" if metric == _abi.L2 else "l1", rows, threads)


class CudaFlatL2AnnIndex(CudaSampledCoordinateL2AnnIndex):
    """include/ultrahigh_ann/hnsvw25/l2/flat/cuda_l2_ann_index.hpp:15-60. With
    importance_probabilities=None the probabilities are built on the device
    (the gpu_fp32 default policy)."""

    def __init__(self, input, repetitions: int, random_engine: MT19937_64,
                 device: int = 0,
                 probability_execution_policy: ExecutionPolicy = ExecutionPolicy.gpu_fp32,
                 *, importance_probabilities=None):
        rows = _rows_input(input)
        if importance_probabilities is None:
            importance_probabilities = _probabilities_for(
                _abi.L2, _matrix(rows), probability_execution_policy, device)
        super().__init__(rows, importance_probabilities, repetitions, random_engine,
                         device)


class CudaFlatL1AnnIndex(CudaSampledCoordinateL1AnnIndex):
    """include/ultrahigh_ann/hnsvw25/l1/flat/cuda_l1_ann_index.hpp:15-50. The
    convenience constructor's default probability policy is sequential
    (src/hnsvw25/l1/flat/cuda_l1_ann_index.cpp:39-46)."""

    def __init__(self, input, repetitions: int, random_engine: MT19937_64,
                 device: int = 0,
                 probability_execution_policy: ExecutionPolicy = ExecutionPolicy.sequential,
                 *, importance_probabilities=None):
        rows = _rows_input(input)
        if importance_probabilities is None:
            importance_probabilities = _probabilities_for(
                _abi.L1, _matrix(rows), probability_execution_policy, device)
        super().__init__(rows, importance_probabilities, repetitions, random_engine,
                         device)


class _CudaHierarchicalIndex(_CudaIndex):
    _metric = _abi.L2

    def __init__(self, input, repetitions=None, projection_dimension=None,
                 random_engine=None, device: int = 0,
                 probability_execution_policy: Optional[ExecutionPolicy] = None, *,
                 importance_probabilities=None, coordinate_sample=None,
                 projection: str = "default"):
        rows = _rows_input(input)
        if projection not in self._projections:
            raise InvalidArgument(f"unknown projection {projection!r}")
        if rows.shape[0] == 0:
            raise InvalidArgument(
                "hierarchical index expects at least one representative")
        if projection_dimension is None or int(projection_dimension) <= 0:
            raise InvalidArgument("projection_dimension has to be a positive integer")
        if random_engine is None:
            raise InvalidArgument("a random engine is required")
        if coordinate_sample is not None:
            sample = (coordinate_sample if isinstance(coordinate_sample,
                                                      CoordinateSample)
                      else CoordinateSample.from_columns(coordinate_sample))
        else:
            if importance_probabilities is None:
                policy = probability_execution_policy or self._default_policy
                importance_probabilities = _probabilities_for(self._metric, _matrix(rows),
                                                              policy, device)
            sample = _resolve_sample(rows, importance_probabilities, repetitions,
                                     random_engine, None)
        if len(sample) == 0 and rows.shape[0] > 1:
            raise CudaRuntimeError("importance sampling selected no coordinates")
        p = int(projection_dimension)
        matrix = self._projections[projection](sample, p, random_engine)
        handle = ctypes.c_void_p()
        sample_args = (_ptr(sample.source_columns), _ptr(sample.multiplicities),
                       _ptr(sample.inverse_probabilities), len(sample), _ptr(matrix), p,
                       ctypes.byref(handle))
        if isinstance(rows, DeviceMatrix):
            _check(_abi.load().uha_hierarchical_index_create_device(
                device, self._metric, ctypes.byref(rows._struct()), *sample_args))
        else:
            _check(_abi.load().uha_hierarchical_index_create(
                device, self._metric, _ptr(rows), rows.shape[0], rows.shape[1],
                *sample_args))
        self._adopt(handle, rows.shape[1], rows.shape[0])
        self.coordinate_sample = sample
        self.projection = matrix
        self.projection_kind = projection


class CudaHierarchicalL2AnnIndex(_CudaHierarchicalIndex):
    """include/ultrahigh_ann/hnsvw25/l2/hierarchical/cuda_hierarchical_l2_ann_index.hpp:33-104:
    sampled coordinates, Rademacher-JL projection to p coordinates, squared-L2
    scan of the projected rows. Default probability policy gpu_fp32.

    projection="gaussian" (keyword only; not in the reference) draws a seeded
    Gaussian JL matrix with binary32 entries from the same engine instead of
    the Rademacher one; everything after the matrix is the same path."""

    _metric = _abi.L2
    _default_policy = ExecutionPolicy.gpu_fp32
    _projections = {"default": build_jl_matrix, "rademacher": build_jl_matrix,
                    "gaussian": build_gaussian_jl_matrix}


class CudaHierarchicalL1AnnIndex(_CudaHierarchicalIndex):
    """include/ultrahigh_ann/hnsvw25/l1/hierarchical/cuda_hierarchical_l1_ann_index.hpp:34-108:
    sampled coordinates, Cauchy projection, median-|diff| scan. Default
    probability policy sequential (cuda_hierarchical_l1_ann_index.cpp:221-228)."""

    _metric = _abi.L1
    _default_policy = ExecutionPolicy.sequential
    _projections = {"default": build_cauchy_matrix, "cauchy": build_cauchy_matrix}

    def query_batch(self, queries, query_count, output, workspace,
                    strategy=QueryStrategy.direct, distances=None):
        return super().query_batch(queries, query_count, output, workspace,
                                   QueryStrategy.direct, distances)


class QueryBatch:
    """Many (index, query count, strategy) pairs on one device answered by one
    CUDA graph launch (uha_batch_*): each pair's pipeline is captured on its
    own graph branch; with autotune each pair's scan shape is tuned first.
    With persistent=True (hierarchical indexes, direct strategy) the graph
    holds the three cooperative launches of the persistent batch kernels
    instead, each draining a device work queue of every pair's units
    (uha_batch_create_persistent). Each pair's answers equal a query_batch of
    the same queries."""

    def __init__(self, pairs, autotune: bool = True, persistent: bool = False):
        pairs = list(pairs)
        if not pairs:
            raise InvalidArgument("a batch needs at least one index")
        self._indexes = [p[0] for p in pairs]
        self._counts = [int(p[1]) for p in pairs]
        strategies = [int(p[2]) if len(p) > 2 else int(QueryStrategy.direct) for p in pairs]
        n = len(pairs)
        handles = (ctypes.c_void_p * n)(*[ix._handle for ix in self._indexes])
        counts = (ctypes.c_uint64 * n)(*self._counts)
        strat = (ctypes.c_int * n)(*strategies)
        handle = ctypes.c_void_p()
        if persistent:
            if any(s != int(QueryStrategy.direct) for s in strategies):
                raise InvalidArgument("the persistent batch runs the direct strategy")
            _check(_abi.load().uha_batch_create_persistent(
                handles, counts, ctypes.c_uint64(n), int(bool(autotune)),
                ctypes.byref(handle)))
        else:
            _check(_abi.load().uha_batch_create(handles, counts, strat, ctypes.c_uint64(n),
                                                int(bool(autotune)), ctypes.byref(handle)))
        self.persistent = bool(persistent)
        self._handle = handle
        self.total = sum(self._counts)

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle:
            self._handle = None
            try:
                _abi.load().uha_batch_destroy(handle)
            except Exception:  # interpreter shutdown: the module is gone
                pass

    def query_buffer(self, pair: int) -> int:
        """Device pointer the graph reads pair `pair`'s queries from."""
        return int(_abi.load().uha_batch_query_buffer(self._handle, ctypes.c_uint64(pair)) or 0)

    def run(self, queries=None, on_device: bool = False):
        """queries: None (use the query buffers) or one array (host) / device
        pointer (on_device) per pair. Returns (indices, distances) per pair."""
        n = len(self._counts)
        keep = []
        ptrs = None
        if queries is not None:
            if len(queries) != n:
                raise InvalidArgument("one query set per batch pair")
            arr = []
            for q, ix, c in zip(queries, self._indexes, self._counts):
                if on_device:
                    arr.append(int(q))
                else:
                    a = np.ascontiguousarray(q, dtype=np.float32).reshape(-1)
                    if a.size != c * ix.dimension:
                        raise InvalidArgument("query batch dimensions do not match index dimension")
                    keep.append(a)
                    arr.append(a.ctypes.data)
            ptrs = (ctypes.c_void_p * n)(*arr)
        idx = np.zeros(self.total, np.uint64)
        dist = np.zeros(self.total, np.float64)
        _check(_abi.load().uha_batch_run(self._handle, ptrs, int(on_device),
                                         ctypes.c_void_p(idx.ctypes.data),
                                         ctypes.c_void_p(dist.ctypes.data)))
        out, o = [], 0
        for c in self._counts:
            out.append((idx[o:o + c], dist[o:o + c]))
            o += c
        return out

    def stats(self) -> dict:
        st = _abi.BatchStats()
        _check(_abi.load().uha_batch_stats_get(self._handle, ctypes.byref(st)))
        return {"pairs": st.pairs, "queries": st.queries, "graph_nodes": st.graph_nodes,
                "kernel_launches": st.kernel_launches,
                "replayed_queries": st.replayed_queries, "device_ms": st.device_ms}

    def stage_ms(self) -> list[float]:
        """Stage times (ms) of the last run of a persistent batch: stage s from
        the completion of every unit of the earlier stages to the completion
        of every unit up to s (pairs' stages overlap; the sum is the run's
        kernel time); [] otherwise."""
        out = np.zeros(16, np.float64)
        stages = ctypes.c_uint64(0)
        _check(_abi.load().uha_batch_stage_times(self._handle, out.ctypes.data, 16,
                                                 ctypes.byref(stages)))
        return [round(float(v), 4) for v in out[:stages.value]]

    def tuning(self, pair: int) -> dict:
        r = _abi.TuneReport()
        _check(_abi.load().uha_batch_tuning(self._handle, ctypes.c_uint64(pair),
                                            ctypes.byref(r)))
        return _tune_dict(r)


class Server:
    """Request loop over device-resident indexes on one GPU (uha_server_*):
    per-index queues, continuous batching into up to `slots` in-flight
    batches, workspaces admitted by an HBM budget, latency per request.
    Query memory (host arrays or device pointers with queries_on_device) must
    stay valid until the request has completed; the wrapper keeps the host
    arrays it was given alive until drain()."""

    RESULT_DTYPE = np.dtype([("tag", np.uint64), ("index_id", np.uint32),
                             ("status", np.uint32), ("row", np.uint64),
                             ("distance", np.float64), ("latency_us", np.float64)])

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 8 << 30,
                 max_batch: int = 256, slots: int = 4, queries_on_device: bool = False):
        cfg = _abi.ServerConfig(int(hbm_budget_bytes), int(max_batch), int(slots),
                                int(bool(queries_on_device)))
        handle = ctypes.c_void_p()
        _check(_abi.load().uha_server_create(int(device), ctypes.byref(cfg),
                                             ctypes.byref(handle)))
        self._handle = handle
        self._on_device = bool(queries_on_device)
        self._indexes = []
        self._keep = []

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle:
            self._handle = None
            try:
                _abi.load().uha_server_destroy(handle)
            except Exception:  # interpreter shutdown: the module is gone
                pass

    def add_index(self, index: "_CudaIndex", strategy=QueryStrategy.direct) -> int:
        out = ctypes.c_uint32()
        _check(_abi.load().uha_server_add_index(self._handle, index._handle, int(strategy),
                                                ctypes.byref(out)))
        self._indexes.append(index)
        return out.value

    def reserve(self, index_id: int, count: int) -> int:
        """Pre-creates pooled workspaces of an index (within the budget);
        returns how many it holds."""
        held = ctypes.c_uint32()
        _check(_abi.load().uha_server_reserve(self._handle, ctypes.c_uint32(index_id),
                                              ctypes.c_uint32(count), ctypes.byref(held)))
        return held.value

    def _pointer(self, query) -> int:
        if self._on_device:
            return int(query)
        a = np.ascontiguousarray(query, dtype=np.float32)
        self._keep.append(a)
        return a.ctypes.data

    def submit(self, index_id: int, query, tag: int) -> None:
        _check(_abi.load().uha_server_submit(self._handle, ctypes.c_uint32(index_id),
                                             ctypes.c_void_p(self._pointer(query)),
                                             ctypes.c_uint64(tag)))

    def replay(self, index_ids, queries, arrival_us, tags=None) -> None:
        """Open-loop load: request i arrives arrival_us[i] microseconds after
        the call; queries[i] is a host array or a device pointer."""
        n = len(index_ids)
        ids = np.ascontiguousarray(index_ids, dtype=np.uint32)
        ptrs = np.array([self._pointer(q) for q in queries], dtype=np.uint64)
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        tg = None if tags is None else np.ascontiguousarray(tags, dtype=np.uint64)
        _check(_abi.load().uha_server_replay(
            self._handle, ctypes.c_uint64(n), ctypes.c_void_p(ids.ctypes.data),
            ctypes.c_void_p(ptrs.ctypes.data), ctypes.c_void_p(arr.ctypes.data),
            ctypes.c_void_p(tg.ctypes.data) if tg is not None else None))

    def drain(self) -> None:
        """Waits for every submitted request; their host queries are then
        released by the wrapper."""
        _check(_abi.load().uha_server_drain(self._handle))
        self._keep.clear()

    def poll(self, capacity: int = 1 << 20) -> np.ndarray:
        buf = np.zeros(capacity, dtype=self.RESULT_DTYPE)
        got = ctypes.c_uint64()
        _check(_abi.load().uha_server_poll(self._handle, ctypes.c_void_p(buf.ctypes.data),
                                           ctypes.c_uint64(capacity), ctypes.byref(got)))
        return buf[:got.value]

    def stats(self) -> dict:
        st = _abi.ServerStats()
        _check(_abi.load().uha_server_stats_get(self._handle, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _abi.ServerStats._fields_}

    def reset_stats(self) -> None:
        _check(_abi.load().uha_server_reset_stats(self._handle))
