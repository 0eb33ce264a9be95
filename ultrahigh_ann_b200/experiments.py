"""Experiment setups and reports: the reference's benchmark-setup format v2
(src/benchmarks/benchmark_setup.cpp) and its schema-6 JSON / CSV reports
(src/benchmarks/nearest_neighbor_benchmark.cpp:1302-1620), driven through
this engine's CUDA indexes, so the public experiment files run unchanged.

    python -m ultrahigh_ann_b200.experiments path/to/setup.tsv

Runs with `backend=cuda` execute on the engine (strategies direct, gemm and
the appended precision strategies gemm_bf16_rerank / gemm_fp8_rerank); CPU
runs are reference-library runs and are reported as skipped.
"""
from __future__ import annotations

import csv
import datetime
import json
import os
import sys
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

FORMAT_HEADER = "ultrahigh_ann_benchmark_setup_v2"

DISTANCES = ("l1", "l2")
INDEXES = ("exact", "flat", "uniform", "hierarchical")
BACKENDS = ("cpu", "cuda")
STRATEGIES = ("sequential", "parallel_queries", "parallel_reference_vectors", "automatic",
              "direct", "gemm", "gemm_bf16_rerank", "gemm_fp8_rerank")
POLICIES = ("sequential", "cpu_parallel", "gpu_fp32", "gpu_cublas_fp32", "load")
DIAGNOSTICS = ("none", "selected_distances", "full_distance_table")
KNOWN_DIRECTIVES = {"dataset", "json_output", "csv_output", "reference", "distance",
                    "max_queries", "warmups", "trials", "batch_sizes", "device",
                    "diagnostics", "probability_policy", "probabilities",
                    "reference_vectors_file", "reference_labels_file", "queries_file",
                    "query_labels_file"}
RUN_PARAMETERS = {"backend", "strategy", "batch_sizes", "warmups", "trials",
                  "repetitions", "seed", "projection_dimension"}
PRECISION_STRATEGIES = ("gemm_bf16_rerank", "gemm_fp8_rerank")
SIZE_MAX = (1 << 64) - 1
INT_MAX = (1 << 31) - 1


class SetupError(RuntimeError):
    """A setup file the reference's loader rejects (std::runtime_error)."""


@dataclass
class BenchmarkRun:
    name: str
    index: str
    backend: str = "cpu"
    strategy: str = "sequential"
    repetitions: int = 0
    seed: int = 0
    projection_dimension: int = 0
    batch_sizes: list = field(default_factory=lambda: [1])
    warmups: int = 0
    trials: int = 1


@dataclass
class BenchmarkSetup:
    setup_path: str = ""
    dataset_directory: str = ""
    representatives_path: str = ""
    representative_labels_path: str = ""
    queries_path: str = ""
    query_labels_path: str = ""
    json_output_path: str = ""
    csv_output_path: str = ""
    probabilities_path: Optional[str] = None
    distance: str = "l2"
    probability_policy: str = "sequential"
    diagnostics: str = "selected_distances"
    maximum_queries: int = 0
    warmups: int = 0
    trials: int = 1
    batch_sizes: list = field(default_factory=lambda: [1])
    device: int = 0
    reference_run: str = ""
    runs: list = field(default_factory=list)


# ------------------------------------------------------------------ parser

def _trim(v: str) -> str:
    return v.strip(" \t\r\n")


def _err(path: str, line: int, message: str) -> SetupError:
    return SetupError(f"{path}:{line}: {message}")


def _integer(text: str, path, line, name, allow_zero, signed=False, limit=SIZE_MAX) -> int:
    # as std::from_chars: decimal digits (a leading '-' for signed types), no
    # '+', no whitespace, within the type's range
    body = text[1:] if signed and text.startswith("-") else text
    ok = bool(body) and body.isascii() and body.isdigit()
    value = 0
    if ok:
        value = int(body)
        if text.startswith("-"):
            value = -value
        ok = -limit - 1 <= value <= limit
    if ok and (value < 0 or (not allow_zero and value == 0)):
        ok = False
    if not ok:
        raise _err(path, line, f"{name} must be a "
                   + ("nonnegative integer" if allow_zero else "positive integer"))
    return value


def _batch_sizes(value: str, path, line) -> list:
    out, seen = [], set()
    for f in (_trim(x) for x in value.split(",")):
        b = _integer(f, path, line, "batch_sizes", False)
        if b in seen:
            raise _err(path, line, "batch_sizes must not contain duplicates")
        seen.add(b)
        out.append(b)
    return out


def _resolve(setup_path: str, configured: str) -> str:
    if os.path.isabs(configured):
        return os.path.normpath(configured)
    return os.path.normpath(os.path.join(os.path.dirname(setup_path), configured))


def _valid_name(v: str) -> bool:
    return bool(v) and all(c.isascii() and (c.isalnum() or c in "_-.") for c in v)


def _parse_run(fields, setup: BenchmarkSetup, path, line) -> BenchmarkRun:
    if len(fields) < 3:
        raise _err(path, line, "run requires a name and index kind")
    if not _valid_name(fields[1]):
        raise _err(path, line,
                   "run name may contain only letters, digits, '.', '_', and '-'")
    if fields[2] not in INDEXES:
        raise _err(path, line, "index must be exact, flat, uniform, or hierarchical")
    run = BenchmarkRun(name=fields[1], index=fields[2], batch_sizes=list(setup.batch_sizes),
                       warmups=setup.warmups, trials=setup.trials)
    params = {}
    for f in fields[3:]:
        sep = f.find("=")
        if sep <= 0 or sep + 1 == len(f):
            raise _err(path, line, "run parameters must use key=value syntax")
        key, value = _trim(f[:sep]), _trim(f[sep + 1:])
        if key in params:
            raise _err(path, line, f"duplicate run parameter: {key}")
        params[key] = value
    if "backend" in params:
        if params["backend"] not in BACKENDS:
            raise _err(path, line, "backend must be cpu or cuda")
        run.backend = params["backend"]
    run.strategy = (("direct" if setup.distance == "l1" else "gemm")
                    if run.backend == "cuda" else "sequential")
    if "strategy" in params:
        if params["strategy"] not in STRATEGIES:
            raise _err(path, line, "unknown query strategy")
        run.strategy = params["strategy"]
    if "batch_sizes" in params:
        run.batch_sizes = _batch_sizes(params["batch_sizes"], path, line)
    if "warmups" in params:
        run.warmups = _integer(params["warmups"], path, line, "warmups", True)
    if "trials" in params:
        run.trials = _integer(params["trials"], path, line, "trials", False)
    approximate = run.index != "exact"
    has_rep, has_seed = "repetitions" in params, "seed" in params
    if approximate and not (has_rep and has_seed):
        raise _err(path, line, "approximate runs require repetitions and seed")
    if not approximate and (has_rep or has_seed):
        raise _err(path, line, "exact runs do not accept repetitions or seed")
    if approximate:
        run.repetitions = _integer(params["repetitions"], path, line, "repetitions", False)
        run.seed = _integer(params["seed"], path, line, "seed", True)
    if run.index == "hierarchical":
        if "projection_dimension" not in params:
            raise _err(path, line, "hierarchical runs require projection_dimension")
        run.projection_dimension = _integer(params["projection_dimension"], path, line,
                                            "projection_dimension", False)
    elif "projection_dimension" in params:
        raise _err(path, line, "projection_dimension requires a hierarchical run")
    for key in params:
        if key not in RUN_PARAMETERS:
            raise _err(path, line, f"unsupported run parameter: {key}")
    if run.backend == "cuda":
        if run.strategy not in ("direct", "gemm") + PRECISION_STRATEGIES:
            raise _err(path, line, "CUDA strategy must be direct or gemm")
        if (setup.distance == "l1" and run.index != "hierarchical"
                and run.strategy != "direct"):
            raise _err(path, line,
                       "CUDA L1 exact, flat, and uniform strategies must be direct")
        if run.strategy in PRECISION_STRATEGIES and (
                setup.distance != "l2" or run.index == "hierarchical"):
            raise _err(path, line, "precision strategies serve exact and flat L2 runs")
    else:
        if run.strategy in ("direct", "gemm") + PRECISION_STRATEGIES:
            raise _err(path, line, "CPU runs cannot use direct or gemm strategy")
        if ((setup.distance == "l1" or run.index == "hierarchical")
                and run.strategy != "sequential"):
            raise _err(path, line, "CPU L1 and hierarchical runs require sequential strategy")
    return run


def load_benchmark_setup(input_path) -> BenchmarkSetup:
    """src/benchmarks/benchmark_setup.cpp:478-665, with the same checks in the
    same order and the same messages. Extension: the strategies
    gemm_bf16_rerank / gemm_fp8_rerank on CUDA exact and flat L2 runs."""
    path = os.path.normpath(os.path.abspath(str(input_path)))
    try:
        with open(path, "r", newline="") as f:
            lines = f.read().split("\n")
    except OSError:
        raise SetupError(f"cannot open benchmark setup: {path}") from None
    if lines and lines[-1] == "":
        lines.pop()
    setup = BenchmarkSetup(setup_path=path)
    header_seen = False
    directives: dict = {}
    raw_runs = []
    for number, text in enumerate(lines, start=1):
        line = _trim(text)
        if not line or line.startswith("#"):
            continue
        if not header_seen:
            if line != FORMAT_HEADER:
                raise _err(path, number, f"expected format header {FORMAT_HEADER}")
            header_seen = True
            continue
        fields = [_trim(x) for x in line.split("\t")]
        if fields[0] == "run":
            raw_runs.append((fields, number))
            continue
        if len(fields) != 2 or not fields[1]:
            raise _err(path, number, f"{fields[0]} requires exactly one value")
        if fields[0] in directives:
            raise _err(path, number, f"duplicate directive: {fields[0]}")
        directives[fields[0]] = (fields[1], number)
    if not header_seen:
        raise SetupError(f"benchmark setup is empty: {path}")

    def require(key):
        if key not in directives:
            raise SetupError(f"benchmark setup does not define {key}")
        return directives[key][0]

    setup.dataset_directory = _resolve(path, require("dataset"))
    setup.json_output_path = _resolve(path, require("json_output"))
    setup.csv_output_path = _resolve(path, require("csv_output"))
    setup.reference_run = require("reference")
    if setup.json_output_path == setup.csv_output_path:
        raise SetupError("json_output and csv_output must differ")
    value = {k: v[0] for k, v in directives.items()}
    line_of = {k: v[1] for k, v in directives.items()}
    if "distance" in value:
        if value["distance"] not in DISTANCES:
            raise _err(path, line_of["distance"], "distance must be l1 or l2")
        setup.distance = value["distance"]
    for key, attr, zero in (("max_queries", "maximum_queries", True),
                            ("warmups", "warmups", True), ("trials", "trials", False)):
        if key in value:
            setattr(setup, attr, _integer(value[key], path, line_of[key], key, zero))
    if "batch_sizes" in value:
        setup.batch_sizes = _batch_sizes(value["batch_sizes"], path, line_of["batch_sizes"])
    if "device" in value:
        setup.device = _integer(value["device"], path, line_of["device"], "device", True,
                                signed=True, limit=INT_MAX)
    if "diagnostics" in value:
        if value["diagnostics"] not in DIAGNOSTICS:
            raise _err(path, line_of["diagnostics"],
                       "diagnostics must be none, selected_distances, or full_distance_table")
        setup.diagnostics = value["diagnostics"]
    if "probability_policy" in value:
        if value["probability_policy"] not in POLICIES:
            raise _err(path, line_of["probability_policy"], "unknown probability policy")
        setup.probability_policy = value["probability_policy"]
    if "probabilities" in value:
        setup.probabilities_path = _resolve(path, value["probabilities"])
        if "probability_policy" not in value:
            setup.probability_policy = "load"
    if setup.probability_policy == "load" and setup.probabilities_path is None:
        raise SetupError("probability_policy=load requires probabilities")
    if setup.distance == "l1" and setup.probability_policy == "gpu_cublas_fp32":
        raise _err(path, line_of["probability_policy"],
                   "gpu_cublas_fp32 is unavailable for L1 probability computation")

    def dataset_file(key, default):
        name = value.get(key, default)
        if os.path.isabs(name):
            return os.path.normpath(name)
        return os.path.normpath(os.path.join(setup.dataset_directory, name))

    setup.representatives_path = dataset_file("reference_vectors_file", "reference_vectors.npy")
    setup.representative_labels_path = dataset_file("reference_labels_file",
                                                    "reference_labels.npy")
    setup.queries_path = dataset_file("queries_file", "queries.npy")
    setup.query_labels_path = dataset_file("query_labels_file", "query_labels.npy")
    for key in directives:
        if key not in KNOWN_DIRECTIVES:
            raise _err(path, line_of[key], f"unknown directive: {key}")
    names = set()
    for fields, number in raw_runs:
        run = _parse_run(fields, setup, path, number)
        if run.name in names:
            raise _err(path, number, f"duplicate run name: {run.name}")
        names.add(run.name)
        setup.runs.append(run)
    if not setup.runs:
        raise SetupError("benchmark setup does not define any runs")
    ref = [r for r in setup.runs if r.name == setup.reference_run]
    if not ref:
        raise SetupError("reference does not name a configured run")
    if ref[0].index != "exact":
        raise SetupError("reference run must use the exact index")
    return setup


def setup_summary(setup: BenchmarkSetup) -> dict:
    """The parsed setup as plain data (the fields the reference keeps)."""
    d = {k: getattr(setup, k) for k in (
        "setup_path", "dataset_directory", "representatives_path",
        "representative_labels_path", "queries_path", "query_labels_path",
        "json_output_path", "csv_output_path", "probabilities_path", "distance",
        "probability_policy", "diagnostics", "maximum_queries", "warmups", "trials",
        "batch_sizes", "device", "reference_run")}
    d["runs"] = [dict(r.__dict__) for r in setup.runs]
    return d


# ------------------------------------------------------------------ runner

def _probabilities(setup: BenchmarkSetup, reps: np.ndarray, reps_sha: bytes):
    import ultrahigh_ann_b200 as uha
    from . import io as uio

    t = time.perf_counter()
    out = {"policy": setup.probability_policy, "source_file": None, "source_sha256": None,
           "reference_vectors_sha256": None, "gpu": None, "load_ms": 0.0, "build_ms": 0.0}
    if setup.probability_policy == "load":
        f = uio.load_importance_probabilities(setup.probabilities_path)
        kind = (uio.ImportanceProbabilityKind.l1 if setup.distance == "l1"
                else uio.ImportanceProbabilityKind.l2)
        if not uio.importance_probability_source_matches(f, kind, reps.shape[0], reps.shape[1],
                                                         reps_sha):
            raise RuntimeError("importance-probability file does not match the "
                               "representative matrix")
        probs = f.probabilities
        out.update(source_file=setup.probabilities_path,
                   source_sha256=uio.sha256_hex(uio.sha256_file(setup.probabilities_path)),
                   reference_vectors_sha256=uio.sha256_hex(f.representatives_sha256),
                   load_ms=(time.perf_counter() - t) * 1e3)
    elif setup.probability_policy in ("sequential", "cpu_parallel"):
        probs = uha.compute_importance_probabilities_host(
            setup.distance, reps, threads=1 if setup.probability_policy == "sequential" else 0)
        out["build_ms"] = (time.perf_counter() - t) * 1e3
    else:
        fn = (uha.compute_l1_importance_probabilities_gpu if setup.distance == "l1"
              else uha.compute_l2_importance_probabilities_gpu)
        kwargs = {"device": setup.device}
        if setup.probability_policy == "gpu_cublas_fp32":
            kwargs["distance_backend"] = "gram"
        res = fn(reps, **kwargs)
        probs = res.probabilities
        out["build_ms"] = (time.perf_counter() - t) * 1e3
        out["gpu"] = {"device": setup.device,
                      "distance_backend": ("gram" if setup.probability_policy
                                           == "gpu_cublas_fp32" else "direct"),
                      "arithmetic": "fp64", "total_ms": res.total_ms}
    out["coordinate_count"] = int(probs.size)
    out["sampling_mass"] = float(np.sum(probs))
    return probs, out


def _strategy(name):
    import ultrahigh_ann_b200 as uha
    return {"direct": uha.QueryStrategy.direct, "gemm": uha.QueryStrategy.gemm,
            "gemm_bf16_rerank": uha.QueryStrategy.gemm_bf16_rerank,
            "gemm_fp8_rerank": uha.QueryStrategy.gemm_fp8_rerank}[name]


def _build(run: BenchmarkRun, setup: BenchmarkSetup, reps, probs):
    import ultrahigh_ann_b200 as uha
    l2 = setup.distance == "l2"
    dev = setup.device
    if run.index == "exact":
        return (uha.CudaExactL2Index if l2 else uha.CudaExactL1Index)(reps, device=dev)
    rng = uha.MT19937_64(run.seed)
    if run.index in ("flat", "uniform"):
        p = probs
        if run.index == "uniform":
            # mass-matched uniform probabilities
            # (src/coordinate_sampling/uniform_probabilities.cpp)
            mass = float(np.sum(probs))
            p = np.full(reps.shape[1], mass / reps.shape[1]) if reps.shape[1] else probs
        cls = uha.CudaSampledCoordinateL2AnnIndex if l2 else uha.CudaSampledCoordinateL1AnnIndex
        return cls(reps, p, run.repetitions, rng, device=dev)
    cls = uha.CudaHierarchicalL2AnnIndex if l2 else uha.CudaHierarchicalL1AnnIndex
    return cls(reps, run.repetitions, run.projection_dimension, rng, device=dev,
               importance_probabilities=probs)


def _distances(metric, reps, queries, rows):
    """Binary64 distance of each query to its returned row."""
    diff = queries.astype(np.float64) - reps[rows.astype(np.int64)].astype(np.float64)
    return np.abs(diff).sum(axis=1) if metric == "l1" else (diff * diff).sum(axis=1)


def _approximation(opt, got):
    n = opt.size
    optimal = got <= opt
    non = ~optimal
    zero = opt == 0
    safe = np.where(opt > 0, opt, 1.0)
    ratio = np.where(opt > 0, got / safe, np.where(got > 0, np.inf, 1.0))
    cond = non & (opt > 0)
    excess = (got[cond] - opt[cond]) / opt[cond]
    finite = np.isfinite(ratio)
    return {"distance_optimal_count": int(optimal.sum()),
            "distance_optimal_rate": float(optimal.mean()) if n else 0.0,
            "non_optimal_count": int(non.sum()),
            "non_optimal_rate": float(non.mean()) if n else 0.0,
            "distance_ratio": {"mean": float(np.mean(ratio[finite])) if finite.any() else None,
                               "max": float(np.max(ratio)) if n else None},
            "zero_optimum_query_count": int(zero.sum()),
            "zero_optimum_non_optimal_count": int((zero & non).sum()),
            "non_optimal_ratio_count": int(cond.sum()),
            "non_optimal_distance_ratio_mean": float(np.mean(ratio[cond])) if cond.any() else None,
            "non_optimal_relative_excess_mean": float(np.mean(excess)) if cond.any() else None}


def run_benchmark(setup_or_path) -> dict:
    """Runs every CUDA run of a setup (the exact reference run first); writes
    and returns the schema-6 report and the CSV table."""
    import ultrahigh_ann_b200 as uha  # noqa: F401
    from . import io as uio

    setup = (setup_or_path if isinstance(setup_or_path, BenchmarkSetup)
             else load_benchmark_setup(setup_or_path))
    t = time.perf_counter()
    reps_sha = uio.sha256_file(setup.representatives_path)
    q_sha = uio.sha256_file(setup.queries_path)
    hash_ms = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    reps = uio.load_float_matrix_npy(setup.representatives_path)
    if reps.shape[0] == 0:
        raise RuntimeError("dataset has no reference vectors")
    if reps.shape[1] == 0:
        raise RuntimeError("dataset has no features")
    queries = uio.load_float_matrix_npy(setup.queries_path)
    if queries.shape[1] != reps.shape[1]:
        raise RuntimeError("reference-vector and query dimensions do not match")
    labels = (os.path.isfile(setup.query_labels_path)
              and os.path.isfile(setup.representative_labels_path))
    qlab = uio.load_label_vector_npy(setup.query_labels_path) if labels else None
    rlab = uio.load_label_vector_npy(setup.representative_labels_path) if labels else None
    load_ms = (time.perf_counter() - t) * 1e3
    available = queries.shape[0]
    n = available if setup.maximum_queries == 0 else min(setup.maximum_queries, available)
    queries = np.ascontiguousarray(queries[:n])
    if labels:
        qlab = qlab[:n]
    approximate = any(r.index != "exact" for r in setup.runs if r.backend == "cuda")
    if approximate:
        probs, prob_info = _probabilities(setup, reps, reps_sha)
    else:
        probs = None
        prob_info = {"policy": setup.probability_policy, "gpu": None, "source_file": None,
                     "source_sha256": None, "reference_vectors_sha256": None,
                     "build_ms": 0.0, "load_ms": 0.0, "coordinate_count": 0,
                     "sampling_mass": 0.0}
    order = sorted(setup.runs, key=lambda r: r.name != setup.reference_run)
    ref_choice = opt = None
    executions = {}
    for run in order:
        if run.backend != "cuda":
            executions[run.name] = {"skipped": "CPU runs execute the reference library, "
                                               "not this engine"}
            continue
        t = time.perf_counter()
        index = _build(run, setup, reps, probs)
        build_ms = (time.perf_counter() - t) * 1e3
        u = index.space_usage()
        meas = []
        for b in run.batch_sizes:
            batch = min(b, n)
            ws = index.make_query_workspace(batch)
            out = np.zeros(n, np.uint64)
            dist = np.zeros(n, np.float64)
            strategy = _strategy(run.strategy)
            for _ in range(run.warmups):
                index.query_many(queries, n, batch, out, ws, strategy, dist)
            trials = []
            for _ in range(run.trials):
                t = time.perf_counter()
                index.query_many(queries, n, batch, out, ws, strategy, dist)
                trials.append((time.perf_counter() - t) * 1e3)
            if run.name == setup.reference_run and ref_choice is None:
                ref_choice = out.copy()
                opt = _distances(setup.distance, reps, queries, ref_choice)
            med = float(np.median(trials))
            agree = int(np.sum(out == ref_choice)) if ref_choice is not None else 0
            m = {"batch_size": b, "workspace_payload_bytes": ws.payload_bytes(),
                 "trial_ms": trials, "median_ms": med,
                 "median_microseconds_per_query": med * 1e3 / n,
                 "median_queries_per_second": n * 1e3 / med,
                 "exact_neighbor_agreement_count": agree,
                 "exact_neighbor_agreement": agree / n,
                 "correct": None, "accuracy": None, "label_agreement_with_exact": None,
                 "approximation": None}
            if labels:
                mine = rlab[out.astype(np.int64)]
                correct = int(np.sum(mine == qlab))
                m["correct"] = correct
                m["accuracy"] = correct / n
                m["label_agreement_with_exact"] = float(np.mean(
                    mine == rlab[ref_choice.astype(np.int64)]))
            if setup.diagnostics != "none" and opt is not None:
                m["approximation"] = _approximation(
                    opt, _distances(setup.distance, reps, queries, out))
            meas.append(m)
        executions[run.name] = {
            "build_ms": build_ms,
            "space": {"index_payload_bytes": u.index_payload_bytes,
                      "query_workspace_payload_bytes": u.query_workspace_payload_bytes,
                      "unique_coordinates": u.unique_query_coordinates,
                      "sampled_multiplicity": u.sampled_multiplicity},
            "device": {"index": index.device(), "name": index.device_name()},
            "measurements": meas}
    hexd = uio.sha256_hex
    report = {
        "schema_version": 6,
        "generated_at_utc": datetime.datetime.now(datetime.timezone.utc).strftime(
            "%Y-%m-%dT%H:%M:%SZ"),
        "setup_file": setup.setup_path,
        "engine": "ultrahigh_ann_b200",
        "outputs": {"json": setup.json_output_path, "csv": setup.csv_output_path},
        "dataset": {"directory": setup.dataset_directory,
                    "reference_vectors_file": setup.representatives_path,
                    "reference_labels_file": (setup.representative_labels_path
                                              if labels else None),
                    "queries_file": setup.queries_path,
                    "query_labels_file": setup.query_labels_path if labels else None,
                    "reference_vectors_sha256": hexd(reps_sha),
                    "queries_sha256": hexd(q_sha),
                    "reference_vector_count": int(reps.shape[0]),
                    "query_count_available": int(available),
                    "query_count_run": int(n), "dimension": int(reps.shape[1]),
                    "labels_available": bool(labels), "hash_ms": hash_ms,
                    "load_ms": load_ms},
        "settings": {"distance": setup.distance, "reference_run": setup.reference_run,
                     "max_queries": setup.maximum_queries, "device": setup.device,
                     "diagnostics": setup.diagnostics},
        "sampling_probabilities": dict(prob_info, required=approximate),
        "runs": []}
    for run in setup.runs:
        entry = {"name": run.name, "index": run.index, "backend": run.backend,
                 "strategy": run.strategy, "reference": run.name == setup.reference_run,
                 "repetitions": run.repetitions, "seed": run.seed,
                 "projection_dimension": run.projection_dimension, "warmups": run.warmups,
                 "trials": run.trials}
        entry.update(executions[run.name])
        report["runs"].append(entry)
    for p in (setup.json_output_path, setup.csv_output_path):
        os.makedirs(os.path.dirname(p) or ".", exist_ok=True)
    with open(setup.json_output_path, "w") as f:
        json.dump(report, f, indent=2)
    with open(setup.csv_output_path, "w", newline="") as f:
        w = csv.writer(f, quoting=csv.QUOTE_NONNUMERIC)
        w.writerow(["run", "index", "backend", "strategy", "batch_size", "median_ms",
                    "median_microseconds_per_query", "median_queries_per_second",
                    "exact_neighbor_agreement", "accuracy"])
        for entry in report["runs"]:
            for m in entry.get("measurements", []):
                w.writerow([entry["name"], entry["index"], entry["backend"],
                            entry["strategy"], m["batch_size"], m["median_ms"],
                            m["median_microseconds_per_query"],
                            m["median_queries_per_second"], m["exact_neighbor_agreement"],
                            m["accuracy"] if m["accuracy"] is not None else ""])
    return report


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1:
        print("usage: python -m ultrahigh_ann_b200.experiments SETUP.tsv", file=sys.stderr)
        return 2
    report = run_benchmark(argv[0])
    print(report["outputs"]["json"])
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
