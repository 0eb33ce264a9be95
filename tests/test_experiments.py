"""Experiment setups (benchmark-setup format v2) and the schema-6 report.

The parser is pinned to the reference's own loader
(src/benchmarks/benchmark_setup.cpp, compiled into oracle/_ref): the same
parsed fields for the reference's experiment files and for setups written
here, and the same error messages for malformed ones. The runner is checked
end to end on the GPU with a small dataset directory.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np
import pytest

uha = pytest.importorskip("ultrahigh_ann_b200")
from ultrahigh_ann_b200 import experiments as ex  # noqa: E402

HEADER = "ultrahigh_ann_benchmark_setup_v2"
BASE = [HEADER, "dataset\tdata", "json_output\tout/r.json", "csv_output\tout/r.csv",
        "reference\texact"]


def _ref(oracle_module):
    if not oracle_module.ref_available():
        pytest.skip("reference library not built here")
    return oracle_module


def _write(tmp_path, lines, name="setup.tsv") -> Path:
    p = tmp_path / name
    p.write_text("\n".join(lines) + "\n")
    return p


def _same(oracle_module, path):
    theirs = oracle_module.ref_parse_setup(path)
    ours = json.loads(json.dumps(ex.setup_summary(ex.load_benchmark_setup(path))))
    assert ours == theirs


def test_reference_experiment_files_parse_identically(oracle_module):
    O = _ref(oracle_module)
    tree = O.reference_dir()
    if tree is None or not (tree / "experiments").is_dir():
        pytest.skip("reference experiment files are not present")
    files = sorted((tree / "experiments").rglob("*.tsv"))
    assert files
    for f in files:
        _same(O, f)


VALID = {
    "defaults": ["run\texact\texact"],
    "everything": ["distance\tl1", "max_queries\t17", "warmups\t2", "trials\t3",
                   "batch_sizes\t1, 8 ,64", "device\t0", "diagnostics\tnone",
                   "probability_policy\tcpu_parallel", "queries_file\t/abs/q.npy",
                   "reference_vectors_file\tsub/../rv.npy",
                   "run\texact\texact\tbackend=cuda\tstrategy=direct",
                   "run\tflat.1\tflat\trepetitions=4\tseed=0\tbackend=cuda",
                   "run\tu-2\tuniform\trepetitions=2\tseed=7\tbatch_sizes=3,1",
                   "run\th_3\thierarchical\trepetitions=8\tseed=1\tprojection_dimension=16"
                   "\twarmups=0\ttrials=5\tbackend=cuda\tstrategy=gemm"],
    "load_implied": ["probabilities\t../p.uap", "run\texact\texact\tbackend=cuda"],
    "cpu_strategies": ["run\texact\texact\tstrategy=parallel_queries",
                       "run\tf\tflat\trepetitions=1\tseed=1\tstrategy=automatic",
                       "run\tg\tflat\trepetitions=1\tseed=1"
                       "\tstrategy=parallel_reference_vectors"],
    "comments": ["# a comment", "", "run\texact\texact", "   # indented comment"],
}

INVALID = {
    "header": ["run\texact\texact"],
    "duplicate_directive": ["distance\tl2", "distance\tl1", "run\texact\texact"],
    "one_value": ["warmups\t1\t2", "run\texact\texact"],
    "bad_distance": ["distance\tl3", "run\texact\texact"],
    "zero_trials": ["trials\t0", "run\texact\texact"],
    "plus_sign": ["warmups\t+1", "run\texact\texact"],
    "negative_device": ["device\t-1", "run\texact\texact"],
    "dup_batches": ["batch_sizes\t4,4", "run\texact\texact"],
    "bad_batches": ["batch_sizes\t4,,8", "run\texact\texact"],
    "unknown_directive": ["color\tred", "run\texact\texact"],
    "load_without_file": ["probability_policy\tload", "run\texact\texact"],
    "cublas_l1": ["distance\tl1", "probability_policy\tgpu_cublas_fp32",
                  "run\texact\texact"],
    "no_runs": [],
    "bad_name": ["run\tex act\texact"],
    "bad_index": ["run\texact\tivf"],
    "short_run": ["run\texact"],
    "syntax": ["run\texact\texact\tbackend"],
    "dup_param": ["run\texact\texact\tbackend=cuda\tbackend=cpu"],
    "exact_seed": ["run\texact\texact\tseed=1"],
    "flat_no_seed": ["run\texact\texact", "run\tf\tflat\trepetitions=2"],
    "projection_flat": ["run\texact\texact",
                        "run\tf\tflat\trepetitions=2\tseed=1\tprojection_dimension=4"],
    "hier_no_p": ["run\texact\texact", "run\th\thierarchical\trepetitions=2\tseed=1"],
    "unsupported": ["run\texact\texact\tcolor=red"],
    "cuda_strategy": ["run\texact\texact\tbackend=cuda\tstrategy=sequential"],
    "cpu_direct": ["run\texact\texact\tstrategy=direct"],
    "l1_gemm": ["distance\tl1", "run\texact\texact\tbackend=cuda\tstrategy=gemm"],
    "l1_cpu_parallel": ["distance\tl1", "run\texact\texact\tstrategy=parallel_queries"],
    "dup_run": ["run\texact\texact", "run\texact\texact"],
    "reference_missing": ["run\tother\texact"],
    "reference_not_exact": ["run\tother\texact", "run\texact\tflat\trepetitions=1\tseed=1"],
    "bad_strategy": ["run\texact\texact\tstrategy=fastest"],
}


@pytest.mark.parametrize("name", sorted(VALID))
def test_setups_parse_like_the_reference(tmp_path, oracle_module, name):
    O = _ref(oracle_module)
    _same(O, _write(tmp_path, BASE + VALID[name]))


@pytest.mark.parametrize("name", sorted(INVALID))
def test_malformed_setups_fail_like_the_reference(tmp_path, oracle_module, name):
    O = _ref(oracle_module)
    lines = INVALID[name] if name == "header" else BASE + INVALID[name]
    path = _write(tmp_path, lines)
    with pytest.raises(O.ReferenceError_) as theirs:
        O.ref_parse_setup(path)
    with pytest.raises(ex.SetupError) as ours:
        ex.load_benchmark_setup(path)
    assert str(ours.value) == str(theirs.value).split(": ", 1)[1]


def test_same_output_paths_and_missing_file(tmp_path):
    path = _write(tmp_path, [HEADER, "dataset\td", "json_output\tx", "csv_output\tx",
                             "reference\te", "run\te\texact"])
    with pytest.raises(ex.SetupError, match="must differ"):
        ex.load_benchmark_setup(path)
    with pytest.raises(ex.SetupError, match="cannot open benchmark setup"):
        ex.load_benchmark_setup(tmp_path / "none.tsv")


def test_precision_strategies_are_an_extension(tmp_path):
    ok = ex.load_benchmark_setup(_write(tmp_path, BASE + [
        "run\texact\texact\tbackend=cuda",
        "run\tb\texact\tbackend=cuda\tstrategy=gemm_bf16_rerank"]))
    assert ok.runs[1].strategy == "gemm_bf16_rerank"
    with pytest.raises(ex.SetupError, match="precision strategies"):
        ex.load_benchmark_setup(_write(tmp_path, BASE + [
            "run\texact\texact", "run\th\thierarchical\trepetitions=2\tseed=1"
            "\tprojection_dimension=4\tbackend=cuda\tstrategy=gemm_fp8_rerank"], "b.tsv"))


@pytest.mark.gpu
def test_run_benchmark_end_to_end(tmp_path):
    from ultrahigh_ann_b200 import io as uio
    from ultrahigh_ann_b200 import synthetic
    ds = synthetic.row_dataset(rows=300, classes=6, queries=50, d=1500, seed=5)
    data = tmp_path / "data"
    data.mkdir()
    np.save(data / "reference_vectors.npy", ds.rows)
    np.save(data / "queries.npy", ds.queries)
    np.save(data / "reference_labels.npy", ds.row_class.astype(np.uint16))
    np.save(data / "query_labels.npy", ds.query_class.astype(np.uint16))
    probs = uha.compute_importance_probabilities_host("l2", ds.rows)
    uio.save_importance_probabilities(data / "p.uap", uio.ImportanceProbabilityKind.l2,
                                      300, uio.sha256_file(data / "reference_vectors.npy"),
                                      probs)
    setup = _write(tmp_path, [
        HEADER, "dataset\tdata", "json_output\tout/r.json", "csv_output\tout/r.csv",
        "reference\texact", "probabilities\tdata/p.uap", "batch_sizes\t1,16",
        "trials\t2", "warmups\t1",
        "run\texact\texact\tbackend=cuda\tstrategy=direct",
        "run\texact_gemm\texact\tbackend=cuda",
        "run\tbf16\texact\tbackend=cuda\tstrategy=gemm_bf16_rerank",
        "run\tflat\tflat\trepetitions=16\tseed=3\tbackend=cuda\tstrategy=direct",
        "run\tuniform\tuniform\trepetitions=16\tseed=3\tbackend=cuda\tstrategy=direct",
        "run\thier\thierarchical\trepetitions=16\tseed=3\tprojection_dimension=16"
        "\tbackend=cuda\tstrategy=direct",
        "run\tcpu\texact"])
    report = ex.run_benchmark(setup)
    assert report["schema_version"] == 6
    assert report["dataset"]["labels_available"]
    assert report["sampling_probabilities"]["policy"] == "load"
    runs = {r["name"]: r for r in report["runs"]}
    assert "skipped" in runs["cpu"]
    for name in ("exact", "exact_gemm", "bf16", "flat", "uniform", "hier"):
        assert [m["batch_size"] for m in runs[name]["measurements"]] == [1, 16]
        for m in runs[name]["measurements"]:
            assert len(m["trial_ms"]) == 2 and m["median_queries_per_second"] > 0
    for m in runs["exact"]["measurements"]:
        assert m["exact_neighbor_agreement"] == 1.0
        assert m["approximation"]["distance_optimal_rate"] == 1.0
    assert json.loads((tmp_path / "out" / "r.json").read_text())["runs"][0]["name"] == "exact"
    rows = (tmp_path / "out" / "r.csv").read_text().strip().splitlines()
    assert len(rows) == 1 + 6 * 2
    assert os.path.isabs(report["dataset"]["reference_vectors_file"])
