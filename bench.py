#!/usr/bin/env python
"""Benchmark of the HNSVW query path on B200.

Workload (headline): the exact L2 index over r = 7,028 reference rows in
d = 60,660 coordinates (the row-level TCGA-shaped synthetic workload), 8,192
queries per step answered one query at a time (batch 1). A step is one pass
over the 8,192 queries, as one trial of the reference benchmark's
measure_queries loop. Each answer is the reference CPU's argmin, bit-exact
(certified binary32 scan + binary64 replay of uncertified queries).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs under torchrun as independent replicas: every rank holds a copy of
the index and answers its own 8,192 queries (weak scaling, no collective on the
data path); timing is the max over ranks. `--impl reference` times the
reference's own CPU implementation (its library compiled from source into
oracle/_ref) on the host cores, on rank 0 only.
"""
from __future__ import annotations

import argparse
import functools
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ROWS, DIM, QUERIES = 7028, 60660, 8192
METRIC = "queries/s at r=7028,d=60660 (agreement vs FP64 exact); %HBM peak; p99 latency"
WORKLOAD = "exact_l2_r7028_d60660_b1"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--batch", type=int, default=1)
    p.add_argument("--queries", type=int, default=QUERIES)
    p.add_argument("--no-suite", action="store_true",
                   help="skip the secondary configurations")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--precision-only", action="store_true",
                   help="only the precision-strategy table (one JSON line)")
    p.add_argument("--only", default="",
                   choices=["", "precision", "batched", "serving", "centroids", "wide",
                            "hierarchies", "flat"],
                   help="only this section of the bench (one JSON line)")
    p.add_argument("--full-probabilities", action="store_true",
                   help="with --only hierarchies: each index's importance "
                        "probabilities over all its rows (minutes at 65,536 rows)")
    p.add_argument("--hier-shape", default="",
                   help="ROWS,DIM,QUERIES of the full-size hierarchical batch "
                        "(--only hierarchies; smaller shapes for profiler captures)")
    p.add_argument("--precision-batch", type=int, default=0,
                   help="with --precision-only: one batch size (2048 queries)")
    p.add_argument("--precision-shape", default="",
                   help="with --precision-only: ROWS,DIM of a smaller index "
                        "(profiling captures)")
    return p.parse_args()


def headline_config(batch: int, world: int) -> dict:
    """The workload both arms run: the same dict on the engine and the
    reference line."""
    return {"workload": WORKLOAD, "rows": ROWS, "dimension": DIM, "batch": batch,
            "index": "exact", "metric": "l2", "parallelism": f"replicas x{world}",
            "l2_flush": "inputs larger than L2 (rows 1.71 GB per query pass)"}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return json.loads(path.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.file.flush()
        self.file.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in self.file.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": mx or None, "reasons": sorted(reasons),
                "samples": len(sm)}


def profile_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return None
    entry = json.loads(path.read_text()).get(kernel)
    return None if entry is None else entry.get("dram_bytes_per_launch")


# --------------------------------------------------------------- engine arm
def run_engine(args):
    import torch

    import ultrahigh_ann_b200 as uha
    from ultrahigh_ann_b200 import synthetic

    world, rank, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    device = torch.cuda.current_device()

    # weak scaling: every rank answers its own query set against the same rows
    ds = synthetic.row_dataset(rows=ROWS, classes=33, queries=args.queries, d=DIM,
                               seed=1, query_stream=rank)
    B = args.batch
    n = args.queries
    index = uha.CudaExactL2Index(ds.rows, device=device)
    qdev = torch.from_numpy(ds.queries).to(f"cuda:{device}")
    ws = index.make_query_workspace(B)
    # scan events on every 8th batch: the roofline's launch time is measured
    # over the timed region at an eighth of the events' cost
    ws.set_timing(True, stride=8 if B <= 8 else 1)
    stream = torch.cuda.ExternalStream(ws.stream_handle())
    out = np.zeros(n, np.uint64)

    def one_step(acc=None):
        # one pass over the query set: consecutive batches of B, enqueued back
        # to back by the engine and synchronised once
        index.query_many(qdev.data_ptr(), n, B, out, ws, on_device=True)
        if acc is not None:
            st = ws.last_stats()
            acc["scan_ms"] += st["scan_ms"]
            acc["scan_launches"] += st["timed_scans"]
            acc["launches"] += st["kernel_launches"]
            acc["replayed"] += st["replayed_queries"]

    for _ in range(args.warmup):
        one_step()
    acc = {"scan_ms": 0.0, "scan_launches": 0, "launches": 0, "replayed": 0}
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            one_step(acc)
        stop.record(stream)
        stop.synchronize()
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    from ultrahigh_ann_b200 import replicas
    elapsed_ms = replicas.max_over_ranks(start.elapsed_time(stop),
                                         device=f"cuda:{device}")
    value = replicas.whole_job_rate(n * args.steps, world, elapsed_ms / 1e3)

    # latency of single calls (one batch per uha_query call, host wall clock)
    lat = []
    ws.set_timing(False)
    for s in range(0, min(n, 1024 * B), B):
        t = time.perf_counter()
        index.query_device_batch(qdev.data_ptr() + s * DIM * 4, min(B, n - s),
                                 out[s:s + B], ws)
        lat.append((time.perf_counter() - t) * 1e3)

    # roofline of the dominant kernel (the batch-1 stream scan)
    peaks = measured_peaks()
    scan_avg_ms = acc["scan_ms"] / max(1, acc["scan_launches"])
    alg_bytes = ROWS * DIM * 4 + B * DIM * 4
    achieved = alg_bytes / (scan_avg_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1),
                "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / peaks["hbm_gbs"], 4),
                "traffic": profile_traffic("stream_scan_kernel<1,0>"),
                "kernel": "stream_scan_kernel<1,0>",
                "algorithmic_bytes_per_launch": alg_bytes,
                "avg_launch_ms": round(scan_avg_ms, 5),
                "peak_source": "measured" if not peaks.get("fallback") else "fallback"}

    # end to end through the public API: host queries (pinned), H2D and the
    # result read inside the timed region
    host_q = torch.from_numpy(ds.queries).pin_memory()
    host_np = host_q.numpy()
    e2e_steps = args.steps
    index.query_many(host_np, n, B, out, ws)  # untimed warm-up pass
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        index.query_many(host_np, n, B, out, ws)
    e2e_s = time.perf_counter() - t0
    e2e = {"value": round(n * e2e_steps / e2e_s, 2), "unit": "queries/s",
           "h2d_bytes_per_step": n * DIM * 4,
           "d2h_bytes_per_step": n * 8 + (n // B) * 8,
           "path": "uha_query_many (C ABI) with pinned host queries, "
                   "batch-by-batch H2D inside the call"}

    line = {"metric": METRIC, "value": round(value, 2), "unit": "queries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(elapsed_ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 scan, f64 certification replay", "data": "synthetic",
            "config": headline_config(B, world),
            "queries_per_step": n,
            "implementation": "certified binary32 scan (direct), binary64 replay",
            "roofline": roofline,
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 4),
                           "p99": round(float(np.percentile(lat, 99)), 4),
                           "scope": f"{len(lat)} single uha_query calls of one batch, "
                                    "host wall clock"},
            "replayed_queries": acc["replayed"],
            "agreement_vs_fp64_exact": None,
            "e2e": e2e, "gpu_launches": acc["launches"]}
    line["clocks"] = clocks.summary()

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], agree = cpu_baseline(ds, index, ws, B)
        line["agreement_vs_fp64_exact"] = agree
    if rank == 0 and not args.no_suite and world == 1:
        del qdev
        torch.cuda.empty_cache()
        line["suite"] = suite(ds, index)
        line["centroids_flat"] = centroids_flat()
        line["precision"] = precision(ds, index)
        torch.cuda.empty_cache()
        line["batched"] = batched(ds)
        torch.cuda.empty_cache()
        line["serving"] = serving(ds)
        torch.cuda.empty_cache()
        line["wide"] = wide()
        torch.cuda.empty_cache()
        line["hierarchies_full"] = hierarchies_full()
        # last key of the line: the figures the sections above are quoted by
        line["summary"] = summarize(line)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def summarize(line: dict) -> dict:
    """One short dict of the sections' headline figures (printed last)."""
    out = {"queries_per_s": line["value"], "e2e_queries_per_s": line["e2e"]["value"],
           "roofline_frac": line["roofline"]["frac"]}
    suite_ = line.get("suite") or {}
    eq = [e["equal_to_reference"] for e in suite_.get("lines", [])
          if e.get("equal_to_reference") is not None]
    parity = {"headline_sample": line.get("agreement_vs_fp64_exact"),
              "r7028_exact_flat_min": min(eq) if eq else None,
              "r7028_lines_checked": len(eq),
              "probabilities_bit_identical": suite_.get("probabilities")}
    cent = line.get("centroids_flat") or {}
    parity["r33_flat_t8"] = cent.get("equal_to_reference_cpu_flat")
    hf = line.get("hierarchies_full") or {}
    ref = hf.get("reference") or {}
    parity["hierarchical_16"] = ref.get("equal_to_reference")
    out["equal_to_reference"] = parity
    out["flat_batch1"] = {
        f"{e['metric']}_T{e['T']}": {"queries_per_s": e["queries_per_s"],
                                     "one_read_frac_of_hbm": e.get("one_read_frac_of_hbm")}
        for e in suite_.get("lines", []) if e["index"] == "flat" and e["batch"] == 1}
    prec = [e for e in line.get("precision") or [] if e.get("strategy") != "direct"
            and e["batch"] == 1024]
    out["precision_b1024"] = {f"{e['strategy']}_k{e['k']}": {
        "speedup_vs_direct": e["speedup_vs_direct"],
        "agreement": e["agreement_vs_fp64_exact"]} for e in prec}
    if hf:
        out["hierarchical_16"] = {"device_ms": hf.get("device_ms"),
                                  "kernels_per_run": hf.get("kernels_per_run"),
                                  "persistent": {k: (hf.get("persistent") or {}).get(k)
                                                 for k in ("device_ms", "kernels_per_run",
                                                           "answers_equal_graph")},
                                  "l2_bf16_device_ms":
                                      (hf.get("l2_bf16_rerank") or {}).get("device_ms"),
                                  "autotune": hf.get("autotune")}
    return out


def cpu_baseline(ds, index, ws, batch):
    """The reference's own ExactL2Index (oracle/_ref) on all host cores, on a
    bounded sample of the same queries, at the engine's batch size (query_batch
    calls of `batch` queries with the reference's automatic strategy: split
    over rows for one query). Also checks the engine's answers on that sample
    against it (agreement with the binary64 exact scan)."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    ref = O.RefExactIndex("l2", ds.rows)
    probe = ds.queries[:max(threads, batch)]
    t = time.perf_counter()
    ref.query_in_batches(probe, batch, threads)
    per = (time.perf_counter() - t) / probe.shape[0]
    sample = int(min(ds.queries.shape[0], max(threads, 15.0 / per)))
    step = max(threads, batch)
    sample = max(step, sample // step * step)
    q = ds.queries[:sample]
    t = time.perf_counter()
    expected = ref.query_in_batches(q, batch, threads)
    secs = time.perf_counter() - t
    got = np.zeros(sample, np.uint64)
    for s in range(sample):
        index.query_batch(q[s], 1, got[s:s + 1], ws)
    agree = float(np.mean(got == expected))
    return ({"value": round(sample / secs, 3), "unit": "queries/s", "cores": threads,
             "kind": "reference",
             "sample": f"{sample} of the {ds.queries.shape[0]} queries, "
                       f"ExactL2Index::query_batch in calls of {batch} "
                       f"(automatic strategy), {threads} OpenMP threads "
                       f"({secs:.1f} s)"}, agree)


def suite(ds, exact_index, nq=1024):
    """Secondary configurations of the same data (r = 7,028, d = 60,660): exact
    and flat (importance-sampled, T = 32 and 128) indexes, L1 and L2, at
    batches 1, 64 and 1,024 over the same `nq` queries. Every line states
    `equal_to_reference`: the fraction of answers equal to the reference's own
    CPU index (oracle/_ref: ExactL2Index / ExactL1Index, and the reference's
    SampledCoordinateL{2,1}AnnIndex given the engine's coordinate sample), and
    the flat lines their agreement with the binary64 exact argmin. The flat
    indexes sample from GPU probabilities, which equal the reference CPU's bit
    for bit (checked here on a 512-row subset, and the sample drawn from them
    against the reference sampler)."""
    import torch

    import ultrahigh_ann_b200 as uha
    from oracle import oracle as O

    out = []
    threads = os.cpu_count() or 1
    queries = np.ascontiguousarray(ds.queries[:nq])
    qdev = torch.from_numpy(queries).cuda()
    have_ref = O.ref_available()

    def timeit(index, B, n, emulated=False):
        # One uha_query_many call answers the n device-resident queries in
        # batches of B (each batch as one query_batch call); the first,
        # identical call warms the workspace and its pipeline buffers.
        ws = index.make_query_workspace(B)
        ws.set_replay(emulated)
        res = np.zeros(n, np.uint64)
        index.query_many(qdev.data_ptr(), n, B, res, ws, on_device=True)
        torch.cuda.synchronize()
        t = time.perf_counter()
        index.query_many(qdev.data_ptr(), n, B, res, ws, on_device=True)
        qps = n / (time.perf_counter() - t)
        return res, qps, ws.last_stats()["replayed_queries"]

    def equal(res, ref):
        return None if ref is None else round(float(np.mean(res == ref)), 4)

    exact_ans = {}
    ref_seconds = 0.0
    for metric, index in (("l2", exact_index), ("l1", uha.CudaExactL1Index(ds.rows))):
        ref = None
        if have_ref:
            t = time.perf_counter()
            ref = O.ref_exact(metric, ds.rows, queries, threads)
            ref_seconds += time.perf_counter() - t
        for B in (1, 64, 1024):
            res, qps, repl = timeit(index, B, nq)
            if B == 1024:
                exact_ans[metric] = res
            out.append({"index": "exact", "metric": metric, "batch": B, "queries": nq,
                        "queries_per_s": round(qps, 1), "replayed": repl,
                        "equal_to_reference": equal(res, ref)})
        # the replay of uncertified queries without FP64 instructions
        res, qps, repl = timeit(index, 1, nq, emulated=True)
        out.append({"index": "exact", "metric": metric, "batch": 1, "queries": nq,
                    "replay": "emulated (float-float, emulated binary64)",
                    "queries_per_s": round(qps, 1), "replayed": repl,
                    "equal_to_reference": equal(res, ref)})
    for metric, cls in (("l2", uha.CudaSampledCoordinateL2AnnIndex),
                        ("l1", uha.CudaSampledCoordinateL1AnnIndex)):
        probs = _probabilities(metric, ds.rows)
        for T in (32, 128):
            index = cls(ds.rows, probs, T, uha.MT19937_64(0))
            cs = index.coordinate_sample
            ref = None
            sample_equal = None
            if have_ref:
                t = time.perf_counter()
                cols, mult, invp, _ = O.ref_sample(probs, T, 0)
                sample_equal = bool(np.array_equal(cols, cs.source_columns) and
                                    np.array_equal(mult, cs.multiplicities) and
                                    invp.tobytes() == cs.inverse_probabilities.tobytes())
                ref = O.ref_sampled(metric, ds.rows, cols, mult, invp, queries, threads)
                ref_seconds += time.perf_counter() - t
            for B in (1, 64, 1024):
                res, qps, repl = timeit(index, B, nq)
                entry = {"index": "flat", "metric": metric, "T": T, "k": len(cs),
                         "batch": B, "queries": nq, "queries_per_s": round(qps, 1),
                         "replayed": repl, "equal_to_reference": equal(res, ref),
                         "sample_equal_to_reference_sampler": sample_equal,
                         "agreement_vs_fp64_exact": round(
                             float(np.mean(res == exact_ans[metric])), 4)}
                if B == 1:
                    # the index's rows read once per query at the measured HBM
                    # bandwidth (they also fit the 126 MB L2)
                    row_bytes = ds.rows.shape[0] * (-(-len(cs) // 4) * 4) * 4
                    entry["one_read_frac_of_hbm"] = round(
                        row_bytes * qps / (measured_peaks()["hbm_gbs"] * 1e9), 3)
                out.append(entry)
    return {"lines": out, "probabilities": probability_parity(ds),
            "reference_cpu_seconds": round(ref_seconds, 1)}


def probability_parity(ds, rows=512):
    """GPU importance probabilities (direct pair backend) against the
    reference CPU's (oracle/_ref, cpu_parallel policy) on the first `rows`
    rows at full dimension: bit-identical or not."""
    import ultrahigh_ann_b200 as uha
    from oracle import oracle as O

    if not O.ref_available():
        return None
    sub = np.ascontiguousarray(ds.rows[:rows])
    res = {"rows": rows, "dimension": sub.shape[1]}
    for metric, fn in (("l2", uha.compute_l2_importance_probabilities_gpu),
                       ("l1", uha.compute_l1_importance_probabilities_gpu)):
        got = fn(sub).probabilities
        want = O.ref_probabilities(metric, sub)
        res[f"{metric}_bit_identical"] = got.tobytes() == want.tobytes()
    return res


def precision(ds, exact_index, batches=((1, 256), (64, 2048), (1024, 2048))):
    """Precision strategies on the same data: BF16 and FP8-E4M3 tensor-core
    scores, top-k (k = 8, 32), then a certified re-score of the candidates
    from the original rows -- binary64 terms (`*_rerank`) or binary32 with
    near-ties settled without FP64 instructions (`*_rerank_fp32`). For each batch:
    queries/s against the plain certified path at the same batch, agreement of
    the answers with the binary64 exact argmin (the plain path's answers, which
    are the reference CPU's), the relative distance excess over the exact
    minimum, and the score kernel's tensor throughput."""
    import torch

    import ultrahigh_ann_b200 as uha

    peaks = measured_peaks()
    nq = max(n for _, n in batches)
    qdev = torch.from_numpy(ds.queries[:nq]).cuda()
    rows, dim = ds.rows.shape

    def timed(B, n, strategy, k=None):
        ws = exact_index.make_query_workspace(B)
        if k is not None:
            ws.set_candidates(k)
        ws.set_timing(True)
        res = np.zeros(n, np.uint64)
        dist = np.zeros(n, np.float64)
        # warm-up: the same call (first use builds the low-precision rows and
        # the workspace's pipeline buffers)
        exact_index.query_many(qdev.data_ptr(), n, B, res, ws, strategy, dist,
                               on_device=True)
        torch.cuda.synchronize()
        t = time.perf_counter()
        exact_index.query_many(qdev.data_ptr(), n, B, res, ws, strategy, dist,
                               on_device=True)
        secs = time.perf_counter() - t
        return res, dist, n / secs, ws.last_stats()

    out = []
    for B, n in batches:
        ref, ref_dist, plain_qps, _ = timed(B, n, uha.QueryStrategy.direct)
        out.append({"strategy": "direct", "batch": B, "queries": n,
                    "queries_per_s": round(plain_qps, 1)})
        for strategy, name, elem in (
                (uha.QueryStrategy.gemm_bf16_rerank, "bf16_rerank", 2),
                (uha.QueryStrategy.gemm_fp8_rerank, "fp8_rerank", 1),
                (uha.QueryStrategy.gemm_bf16_rerank_fp32, "bf16_rerank_fp32", 2),
                (uha.QueryStrategy.gemm_fp8_rerank_fp32, "fp8_rerank_fp32", 1)):
            for k in (8, 32):
                res, dist, qps, st = timed(B, n, strategy, k)
                excess = (dist - ref_dist) / np.maximum(ref_dist, 1e-300)
                ms = st["scan_ms"] / max(1, st["timed_scans"])
                pitch = -(-dim // (64 if elem == 2 else 128)) * (64 if elem == 2 else 128)
                tflops = 2.0 * rows * dim * min(B, n) / (ms * 1e-3) / 1e12
                out.append({
                    "strategy": name, "k": k, "batch": B, "queries": n,
                    "queries_per_s": round(qps, 1),
                    "speedup_vs_direct": round(qps / plain_qps, 2),
                    "agreement_vs_fp64_exact": round(float(np.mean(res == ref)), 4),
                    "distance_excess": {"mean": float(np.mean(excess)),
                                        "max": float(np.max(excess))},
                    "replayed": st["replayed_queries"],
                    "score_kernel": {
                        "ms_per_launch": round(ms, 4),
                        "tflops": round(tflops, 1),
                        "frac_of_measured_bf16": round(tflops / peaks["bf16_tflops"], 3),
                        "row_bytes_gbs": round(rows * pitch * elem / (ms * 1e-3) / 1e9, 1)}})
    return out


def centroids_flat(queries=3013):
    """The reference's own CPU-runnable case: 33 class centroids, d = 60,660,
    flat L2 importance-sampling index with T = 8 and seed 0 (probabilities by
    the reference CPU policy's arithmetic), 3,013 queries answered one at a
    time (one launch each: gather, scan and certified argmin fused for small
    indexes). Reported in microseconds per query and kernels per query (the
    index is 33 x |I| floats: launch-latency bound, not a %HBM case), with the
    answers checked against the reference's own CPU flat index (oracle/_ref)
    and the agreement with the binary64 exact argmin."""
    import torch

    import ultrahigh_ann_b200 as uha
    from oracle import oracle as O
    from ultrahigh_ann_b200 import synthetic

    ds = synthetic.centroid_dataset(classes=33, queries=queries, seed=0)
    probs = uha.compute_importance_probabilities_host("l2", ds.rows)
    index = uha.CudaSampledCoordinateL2AnnIndex(ds.rows, probs, 8, uha.MT19937_64(0))
    s = index.coordinate_sample
    ws = index.make_query_workspace(1)
    qdev = torch.from_numpy(ds.queries).cuda()
    out = np.zeros(queries, np.uint64)
    index.query_many(qdev.data_ptr(), 64, 1, out[:64], ws, on_device=True)
    torch.cuda.synchronize()
    t = time.perf_counter()
    index.query_many(qdev.data_ptr(), queries, 1, out, ws, on_device=True)
    dev_s = time.perf_counter() - t
    launches = ws.last_stats()["kernel_launches"]
    host = np.ascontiguousarray(ds.queries)
    out_h = np.zeros(queries, np.uint64)
    t = time.perf_counter()
    index.query_many(host, queries, 1, out_h, ws)
    e2e_s = time.perf_counter() - t
    lat = []
    for i in range(512):
        t = time.perf_counter()
        index.query(host[i], ws)
        lat.append((time.perf_counter() - t) * 1e6)
    entry = {"workload": "flat_l2_centroids_r33_d60660_T8_seed0", "queries": queries,
             "k": len(s), "device_us_per_query": round(dev_s / queries * 1e6, 2),
             "e2e_us_per_query": round(e2e_s / queries * 1e6, 2),
             "single_call_us": {"p50": round(float(np.percentile(lat, 50)), 2),
                                "p99": round(float(np.percentile(lat, 99)), 2)},
             "kernels_per_query": round(launches / queries, 2),
             "answers_equal_host_api": bool(np.array_equal(out, out_h))}
    exact = uha.CudaExactL2Index(ds.rows)
    ex = exact.query_many(host, queries, 1024, None, exact.make_query_workspace(1024))
    entry["agreement_vs_fp64_exact"] = round(float(np.mean(out == ex)), 4)
    if O.ref_available():
        ref = O.ref_sampled("l2", ds.rows, s.source_columns, s.multiplicities,
                            s.inverse_probabilities, ds.queries)
        entry["equal_to_reference_cpu_flat"] = round(float(np.mean(out == ref)), 4)
    return entry


_PROBS: dict = {}


def flat_batch1(ds, nq=2048):
    """The flat indexes (T = 32, L2 and L1) of the r = 7,028, d = 60,660 data
    at batch 1 and 8: one uha_query_many call of `nq` device-resident queries
    per line after an identical warm-up call (the suite's timing, without its
    reference checks; for profiler captures of the fused flat query)."""
    import torch

    import ultrahigh_ann_b200 as uha

    qdev = torch.from_numpy(np.ascontiguousarray(ds.queries[:nq])).cuda()
    out = []
    for metric, cls in (("l2", uha.CudaSampledCoordinateL2AnnIndex),
                        ("l1", uha.CudaSampledCoordinateL1AnnIndex)):
        index = cls(ds.rows, _probabilities(metric, ds.rows), 32, uha.MT19937_64(0))
        for B in (1, 8):
            ws = index.make_query_workspace(B)
            res = np.zeros(nq, np.uint64)
            index.query_many(qdev.data_ptr(), nq, B, res, ws, on_device=True)
            torch.cuda.synchronize()
            t = time.perf_counter()
            index.query_many(qdev.data_ptr(), nq, B, res, ws, on_device=True)
            secs = time.perf_counter() - t
            out.append({"metric": metric, "T": 32, "k": len(index.coordinate_sample),
                        "batch": B, "queries": nq, "queries_per_s": round(nq / secs, 1),
                        "us_per_query": round(secs / nq * 1e6, 3)})
    return out


def _probabilities(metric: str, rows):
    """GPU importance probabilities of the bench rows, computed once per metric."""
    import ultrahigh_ann_b200 as uha

    if metric not in _PROBS:
        fn = (uha.compute_l2_importance_probabilities_gpu if metric == "l2"
              else uha.compute_l1_importance_probabilities_gpu)
        _PROBS[metric] = fn(rows).probabilities
    return _PROBS[metric]


def batched(ds, per_index=4096, reps=3):
    """16 hierarchical indexes of uneven (rows, |I|, p), L2 (JL) and L1
    (Cauchy, median), 4,096 queries each, answered by one captured CUDA graph
    per run with autotuned scan shapes; against the same queries answered
    index by index (uha_query_many, built-in shapes, one stream). The indexes
    take row subsets of the r = 7,028, d = 60,660 data and the probabilities
    of the full matrix."""
    import torch

    import ultrahigh_ann_b200 as uha

    rows_choice = (1024, 2048, 4096, 7028)
    p_choice = (16, 64, 256)
    t_choice = (16, 32, 64)
    specs, indexes = [], []
    for i in range(16):
        metric = "l2" if i % 2 == 0 else "l1"
        r, p, T = rows_choice[i % 4], p_choice[i % 3], t_choice[(i // 3) % 3]
        cls = (uha.CudaHierarchicalL2AnnIndex if metric == "l2"
               else uha.CudaHierarchicalL1AnnIndex)
        ix = cls(ds.rows[:r], T, p, uha.MT19937_64(100 + i),
                 importance_probabilities=_probabilities(metric, ds.rows))
        indexes.append(ix)
        specs.append({"metric": metric, "rows": r, "T": T, "k": len(ix.coordinate_sample),
                      "p": p})
    qdev = torch.from_numpy(ds.queries[:per_index]).cuda()
    t = time.perf_counter()
    batch = uha.QueryBatch([(ix, per_index, uha.QueryStrategy.direct) for ix in indexes],
                           autotune=True)
    setup_s = time.perf_counter() - t
    batch.run([qdev.data_ptr()] * len(indexes), on_device=True)  # queries into its buffers
    ms = []
    for _ in range(reps):
        res = batch.run(None)
        ms.append(batch.stats()["device_ms"])
    st = batch.stats()
    tuned = [batch.tuning(i) for i in range(len(indexes))]
    # the same work index by index
    ws = [ix.make_query_workspace(per_index) for ix in indexes]
    out = np.zeros(per_index, np.uint64)
    for ix, w, i in zip(indexes, ws, range(len(indexes))):
        ix.query_many(batch.query_buffer(i), per_index, per_index, out, w, on_device=True)
    torch.cuda.synchronize()
    t = time.perf_counter()
    agree = []
    for ix, w, i in zip(indexes, ws, range(len(indexes))):
        ix.query_many(batch.query_buffer(i), per_index, per_index, out, w, on_device=True)
        agree.append(bool(np.array_equal(out, res[i][0])))
    seq_s = time.perf_counter() - t
    total = per_index * len(indexes)
    best = min(ms)
    return {"indexes": specs, "queries_per_index": per_index,
            "graph": {"queries_per_s": round(total / (best * 1e-3), 1),
                      "device_ms": round(best, 3), "graph_nodes": st["graph_nodes"],
                      "kernels_per_run": st["kernel_launches"],
                      "replayed": st["replayed_queries"],
                      "setup_s_with_autotune": round(setup_s, 2)},
            "index_by_index": {"queries_per_s": round(total / seq_s, 1),
                               "wall_ms": round(seq_s * 1e3, 3)},
            "answers_equal": all(agree),
            "autotune": {"pairs_changed": sum(1 for t_ in tuned
                                               if t_["candidates"] and t_["best_ms"] < t_["default_ms"]),
                         "default_scan_ms": round(sum(t_["default_ms"] for t_ in tuned), 3),
                         "tuned_scan_ms": round(sum(t_["best_ms"] for t_ in tuned), 3)}}


def _bf16_values(a: np.ndarray) -> np.ndarray:
    """The binary32 values a BF16 store decodes to (round to nearest even)."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32)


@functools.lru_cache(maxsize=1)
def _wide_data(queries=1024, dim=262_144):
    """2,048 rows and `queries` queries at d = dim with BF16-stored values
    (the config-0 generator, 33 latent classes), and the L2 / L1 importance
    probabilities of the first 1,024 rows; built once per run."""
    import ultrahigh_ann_b200 as uha
    from ultrahigh_ann_b200 import synthetic

    t = time.perf_counter()
    ds = synthetic.row_dataset(rows=2048, classes=33, queries=queries, d=dim, seed=3)
    rows = _bf16_values(ds.rows)
    qs = _bf16_values(ds.queries)
    gen_s = time.perf_counter() - t
    t = time.perf_counter()
    p2 = uha.compute_l2_importance_probabilities_gpu(rows[:1024]).probabilities
    p1 = uha.compute_l1_importance_probabilities_gpu(rows[:1024]).probabilities
    return rows, qs, p2, p1, gen_s, time.perf_counter() - t


def wide(per_index=1024, dim=262_144):
    """Hierarchical indexes at d = 262,144 with BF16-stored values (binary32
    values that BF16 represents exactly): L2 (JL) and L1 (Cauchy / median),
    rows 1,024 and 2,048, p = 16 and 64, T = 32, 1,024 queries each, in one
    captured batch; the probabilities are those of the first 1,024 rows."""
    import torch

    import ultrahigh_ann_b200 as uha

    rows, queries, p2, p1, gen_s, prob_s = _wide_data(per_index, dim)
    specs = [("l2", 1024, 16), ("l1", 1024, 64), ("l2", 2048, 64), ("l1", 2048, 16)]
    indexes = []
    t = time.perf_counter()
    for i, (metric, r, p) in enumerate(specs):
        cls = (uha.CudaHierarchicalL2AnnIndex if metric == "l2"
               else uha.CudaHierarchicalL1AnnIndex)
        indexes.append(cls(rows[:r], 32, p, uha.MT19937_64(200 + i),
                           importance_probabilities=p2 if metric == "l2" else p1))
    build_s = time.perf_counter() - t
    qdev = torch.from_numpy(queries).cuda()
    batch = uha.QueryBatch([(ix, per_index, uha.QueryStrategy.direct) for ix in indexes],
                           autotune=True)
    batch.run([qdev.data_ptr()] * len(indexes), on_device=True)
    ms = []
    for _ in range(3):
        res = batch.run(None)
        ms.append(batch.stats()["device_ms"])
    # the same answers index by index
    same = True
    for ix, (got, _) in zip(indexes, res):
        ws = ix.make_query_workspace(per_index)
        want = ix.query_many(qdev.data_ptr(), per_index, per_index, None, ws, on_device=True)
        same = same and bool(np.array_equal(want, got))
    total = per_index * len(indexes)
    return {"dimension": dim, "storage": "bf16 values",
            "indexes": [{"metric": m, "rows": r, "p": p, "T": 32,
                         "k": len(ix.coordinate_sample)} for (m, r, p), ix in
                        zip(specs, indexes)],
            "queries_per_index": per_index,
            "queries_per_s": round(total / (min(ms) * 1e-3), 1),
            "device_ms": round(min(ms), 3), "replayed": batch.stats()["replayed_queries"],
            "answers_equal_index_by_index": same,
            "setup_s": {"generate": round(gen_s, 1), "probabilities": round(prob_s, 1),
                        "build": round(build_s, 1)}}


def _projected_check(ix, metric, sampled64, queries64, got):
    """Binary64 check of a hierarchy's answers on the host: for each query
    (sampled coordinates, binary64) the returned row's projected distance
    (squared L2, or the median |diff| with the mean of the two middle values
    for even p) must equal the minimum over all rows within 1e-9 relative (the
    numpy evaluation order differs from the reference's sequential one)."""
    P = np.asarray(ix.projection, np.float64).reshape(-1, sampled64.shape[1])
    reps = sampled64 @ P.T
    ok = 0
    for q, row in zip(queries64, got):
        diff = reps - q @ P.T
        d = (np.einsum("ij,ij->i", diff, diff) if metric == "l2"
             else np.median(np.abs(diff), axis=1))
        ok += int(d[int(row)] <= d.min() * (1 + 1e-9) + 1e-300)
    return ok


def hierarchies_full(per_index=4096, dim=262_144, rows=65_536, reps=3, checked=16,
                     ref_queries=64, full_probabilities=False):
    """16 hierarchical indexes at the full size of the hierarchical batched
    configuration: rows 1,024 / 7,028 / 65,536 (row subsets of one
    65,536 x 262,144 BF16 matrix generated on the device), T = 32,
    p = 16 / 64 / 256, L2 (JL) and L1 (Cauchy, median), 4,096 queries each,
    in one captured CUDA graph launch with autotuned scan shapes. The indexes
    are built from the device-resident matrix (no host copy of it); the
    importance probabilities are those of the first 1,024 rows (the pair
    computation over all 65,536 rows is ~1e15 operations), or with
    full_probabilities each row count's own probabilities over all its rows
    (direct binary64 pair distances, binary32 column maxima, from the device
    matrix; minutes per metric at 65,536 rows, reported). Checks:
    the same answers index by index, and a binary64 host check of `checked`
    queries per index."""
    import torch

    import ultrahigh_ann_b200 as uha
    from ultrahigh_ann_b200 import synthetic

    t = time.perf_counter()
    data = synthetic.device_row_dataset(rows=rows, classes=33, queries=per_index, d=dim,
                                        seed=4, storage="bfloat16")
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t
    t = time.perf_counter()
    full_report = None
    if full_probabilities:
        # every row count's probabilities over its own rows, from a binary32
        # copy of the device matrix
        probs_by_rows, full_report = {}, {}
        for r in sorted({min(1024, rows), min(7028, rows), rows}):
            x = data.rows[:r].float()
            for metric, fn in (("l2", uha.compute_l2_importance_probabilities_gpu),
                               ("l1", uha.compute_l1_importance_probabilities_gpu)):
                res = fn(x, maxima="binary32", pair_chunks=256)
                probs_by_rows[(metric, r)] = res.probabilities
                full_report[f"{metric}_r{r}"] = {
                    "pair_distance_s": round(res.inverse_distance_ms / 1e3, 2),
                    "column_maxima_s": round(res.coordinate_maximum_ms / 1e3, 2),
                    "total_s": round(res.total_ms / 1e3, 2),
                    "pairs": int(res.pair_count)}
            del x
            torch.cuda.empty_cache()
        probs = None
        # reported at once: the build takes minutes
        print(json.dumps({"full_probability_build": full_report}), file=sys.stderr,
              flush=True)
    else:
        head = data.rows[:1024].float().cpu().numpy()
        probs = {"l2": uha.compute_l2_importance_probabilities_gpu(head).probabilities,
                 "l1": uha.compute_l1_importance_probabilities_gpu(head).probabilities}
    prob_s = time.perf_counter() - t

    def probs_of(metric, r):
        return probs[metric] if probs is not None else probs_by_rows[(metric, r)]
    specs, indexes, seeds = [], [], []
    t = time.perf_counter()
    i = 0
    for r in sorted({min(1024, rows), min(7028, rows), rows}):
        for p in (16, 64, 256):
            for metric in ("l2", "l1"):
                if r == 1024 and p == 256:
                    continue
                cls = (uha.CudaHierarchicalL2AnnIndex if metric == "l2"
                       else uha.CudaHierarchicalL1AnnIndex)
                ix = cls(uha.DeviceMatrix.from_torch(data.rows[:r]), 32, p,
                         uha.MT19937_64(300 + i),
                         importance_probabilities=probs_of(metric, r))
                seeds.append(300 + i)
                indexes.append(ix)
                specs.append({"metric": metric, "rows": r, "T": 32, "p": p,
                              "k": len(ix.coordinate_sample)})
                i += 1
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t
    # host copies of the sampled columns (binary32 holds the BF16 values
    # exactly) for the reference check, then the matrix is released
    sampled = []
    for ix, spec in zip(indexes, specs):
        cols = torch.from_numpy(ix.coordinate_sample.source_columns.astype(np.int64)).cuda()
        sampled.append(data.rows[:spec["rows"]].index_select(1, cols).float().cpu().numpy())
    # the picked queries (reference and binary64 checks) and their binary64
    # exact L2 distances to every row over the full dimension; a Gaussian-JL
    # twin of every L2 hierarchy (same seed, so the same sample) from the same
    # device matrix
    picks = np.random.default_rng(9).choice(per_index, max(checked, ref_queries),
                                            replace=False)
    exact_d2 = exact_l2_distances(data.rows, data.queries, picks[:ref_queries])
    gaussian = []
    for k, spec in enumerate(specs):
        if spec["metric"] == "l2":
            gaussian.append((k, uha.CudaHierarchicalL2AnnIndex(
                uha.DeviceMatrix.from_torch(data.rows[:spec["rows"]]), 32, spec["p"],
                uha.MT19937_64(seeds[k]),
                importance_probabilities=probs_of("l2", spec["rows"]),
                projection="gaussian")))
    data.rows = None
    torch.cuda.empty_cache()
    qdev = data.queries
    t = time.perf_counter()
    batch = uha.QueryBatch([(ix, per_index, uha.QueryStrategy.direct) for ix in indexes],
                           autotune=True)
    setup_s = time.perf_counter() - t
    batch.run([qdev.data_ptr()] * len(indexes), on_device=True)
    ms = []
    torch.cuda.nvtx.range_push("timed_graph")  # the launch list's filter
    for _ in range(reps):
        res = batch.run(None)
        ms.append(batch.stats()["device_ms"])
    torch.cuda.nvtx.range_pop()
    st = batch.stats()
    # the same pairs in one persistent cooperative launch per run
    persistent = None
    try:
        t = time.perf_counter()
        pbatch = uha.QueryBatch([(ix, per_index) for ix in indexes], autotune=True,
                                persistent=True)
        psetup = time.perf_counter() - t
        pbatch.run([qdev.data_ptr()] * len(indexes), on_device=True)
        pms = []
        torch.cuda.nvtx.range_push("timed_persistent")
        for _ in range(reps):
            pres = pbatch.run(None)
            pms.append(pbatch.stats()["device_ms"])
        torch.cuda.nvtx.range_pop()
        pst = pbatch.stats()
        persistent = {
            "queries_per_s": round(per_index * len(indexes) / (min(pms) * 1e-3), 1),
            "device_ms": round(min(pms), 3), "device_ms_runs": [round(m, 3) for m in pms],
            "kernels_per_run": pst["kernel_launches"], "graph_nodes": pst["graph_nodes"],
            "answers_equal_graph": all(bool(np.array_equal(a[0], b[0]))
                                       for a, b in zip(pres, res)),
            "stage_ms_last_run": dict(zip(
                ["clear", "gather", "project", "tile_scan_or_median_sample",
                 "median_count", "argmin_l2_or_median_survivor",
                 "refine_l2_or_argmin_l1", "refine_l1"], pbatch.stage_ms())),
            "setup_s": round(psetup, 1)}
        del pbatch
    except (ValueError, RuntimeError) as e:  # reported, not fatal: the graph batch stands
        persistent = {"error": str(e)}
    same = True
    for k, ix in enumerate(indexes):
        ws = ix.make_query_workspace(per_index)
        ws.set_timing(True)
        want = ix.query_many(qdev.data_ptr(), per_index, per_index, None, ws, on_device=True)
        same = same and bool(np.array_equal(want, res[k][0]))
        ix.query_many(qdev.data_ptr(), per_index, per_index, want, ws, on_device=True)
        ls = ws.last_stats()
        specs[k]["alone_ms"] = round(ls["device_ms"], 3)
        specs[k]["alone_scan_ms"] = round(ls["scan_ms"], 3)
        specs[k]["replayed"] = ls["replayed_queries"]
        tune = batch.tuning(k)
        specs[k]["tuned_scan_ms"] = round(tune["best_ms"], 3)
        specs[k]["tuning"] = {"kernel": tune["kernel"], "candidates": tune["candidates"],
                              "default_ms": round(tune["default_ms"], 3),
                              "changed": bool(tune["candidates"] and
                                              tune["best_ms"] < tune["default_ms"]),
                              "queries_per_pass": tune["queries_per_pass"],
                              "splits": tune["splits"]}
        del ws
    # the same batch with the L2 hierarchies on the BF16 precision strategy
    # (tensor-core projection and scores, 32 candidates, binary64 re-score)
    bf16 = uha.QueryStrategy.gemm_bf16_rerank
    mixed = uha.QueryBatch([(ix, per_index, bf16 if spec["metric"] == "l2"
                             else uha.QueryStrategy.direct)
                            for ix, spec in zip(indexes, specs)], autotune=True)
    mixed.run([qdev.data_ptr()] * len(indexes), on_device=True)
    mixed_ms = []
    torch.cuda.nvtx.range_push("timed_mixed_graph")
    for _ in range(reps):
        mres = mixed.run(None)
        mixed_ms.append(mixed.stats()["device_ms"])
    torch.cuda.nvtx.range_pop()
    precision = []
    for k, spec in enumerate(specs):
        if spec["metric"] != "l2":
            continue
        want_rows, want_dist = res[k]
        got_rows, got_dist = mres[k]
        excess = (got_dist - want_dist) / np.maximum(want_dist, 1e-300)
        precision.append({"rows": spec["rows"], "p": spec["p"],
                          "agreement_vs_direct": round(float(np.mean(got_rows == want_rows)), 4),
                          "distance_excess_mean": float(excess.mean()),
                          "distance_excess_max": float(excess.max())})
    del mixed
    q_host = qdev.index_select(0, torch.from_numpy(picks).cuda()).float().cpu().numpy()
    ok = 0
    for k, (ix, spec) in enumerate(zip(indexes, specs)):
        cols = ix.coordinate_sample.source_columns.astype(np.int64)
        ok += _projected_check(ix, spec["metric"], sampled[k].astype(np.float64),
                               q_host[:checked, cols].astype(np.float64),
                               res[k][0][picks[:checked]])
    reference = hierarchy_reference_parity(indexes, specs, seeds,
                                           [probs_of(sp["metric"], sp["rows"]) for sp in specs],
                                           sampled,
                                           q_host[:ref_queries], picks[:ref_queries],
                                           [r[0] for r in res])
    projections = gaussian_vs_rademacher(gaussian, specs, res, qdev, per_index,
                                         picks[:ref_queries], exact_d2)
    total = per_index * len(indexes)
    best = min(ms)
    return {"workload": f"hierarchical_16_indexes_r{rows}_d{dim}_bf16",
            "indexes": specs, "queries_per_index": per_index,
            "autotune": {"pairs_changed": sum(1 for sp in specs if sp["tuning"]["changed"]),
                         "median_pairs_changed": sum(1 for sp in specs
                                                     if sp["tuning"]["kernel"] == "median"
                                                     and sp["tuning"]["changed"])},
            "queries_per_s": round(total / (best * 1e-3), 1),
            "device_ms": round(best, 3), "device_ms_runs": [round(m, 3) for m in ms],
            "graph_nodes": st["graph_nodes"], "kernels_per_run": st["kernel_launches"],
            "replayed": st["replayed_queries"], "answers_equal_index_by_index": same,
            "persistent": persistent,
            "binary64_checked": {"queries": checked * len(indexes), "distance_optimal": ok},
            "reference": reference,
            "l2_projection_modes": projections,
            "l2_bf16_rerank": {"queries_per_s": round(total / (min(mixed_ms) * 1e-3), 1),
                               "device_ms": round(min(mixed_ms), 3),
                               "strategy": "L2 hierarchies gemm_bf16_rerank (k = 32), "
                                           "L1 hierarchies direct",
                               "indexes": precision},
            "probabilities": ("all rows of each index (direct binary64 pair distances, "
                              "binary32 column maxima)" if full_probabilities
                              else "the first 1,024 rows"),
            "full_probability_build": full_report,
            "setup_s": {"generate_on_device": round(gen_s, 1),
                        "probabilities": round(prob_s, 1), "build": round(build_s, 1),
                        "autotune_and_capture": round(setup_s, 1)}}


def exact_l2_distances(rows_dev, queries_dev, picks, chunk=4096):
    """Binary64 squared L2 distances of the picked queries to every row over
    the full dimension (host array, queries x rows), in row chunks on the
    device: ||x||^2 - 2 x.q + ||q||^2 with binary64 products (relative error
    near 1e-14 here, far below the gaps the agreement figures resolve)."""
    import torch

    q = queries_dev.index_select(0, torch.from_numpy(picks).to(queries_dev.device))
    q = q.double()
    qn = (q * q).sum(1)
    out = []
    for s in range(0, rows_dev.shape[0], chunk):
        x = rows_dev[s:s + chunk].double()
        d = (x * x).sum(1)[None, :] - 2.0 * (q @ x.T) + qn[:, None]
        out.append(d.clamp_min(0.0).cpu().numpy())
        del x, d
    torch.cuda.empty_cache()
    return np.concatenate(out, axis=1)


def gaussian_vs_rademacher(gaussian, specs, res, qdev, per_index, picks, exact_d2):
    """Agreement with the binary64 exact L2 argmin over the full dimension and
    the relative distance excess of the returned row, for each L2 hierarchy
    with the reference's Rademacher projection and with the seeded Gaussian
    one (same sample), on the picked queries; plus the Gaussian twins' device
    time in one captured batch."""
    import ultrahigh_ann_b200 as uha

    if not gaussian:
        return None
    batch = uha.QueryBatch([(ix, per_index, uha.QueryStrategy.direct)
                            for _, ix in gaussian], autotune=True)
    batch.run([qdev.data_ptr()] * len(gaussian), on_device=True)
    ms = []
    for _ in range(3):
        gres = batch.run(None)
        ms.append(batch.stats()["device_ms"])
    rows_out = []
    for (k, _), (got_rows, _) in zip(gaussian, gres):
        r = specs[k]["rows"]
        d2 = exact_d2[:, :r]
        best = d2.min(axis=1)
        exact_rows = d2.argmin(axis=1)

        def stats(answer):
            a = answer[picks].astype(np.int64)
            excess = d2[np.arange(len(picks)), a] / np.maximum(best, 1e-300) - 1.0
            return {"agreement_vs_fp64_exact": round(float(np.mean(a == exact_rows)), 4),
                    "distance_excess_mean": float(excess.mean()),
                    "distance_excess_max": float(excess.max())}
        rows_out.append({"rows": r, "p": specs[k]["p"], "k": specs[k]["k"],
                         "rademacher": stats(res[k][0]), "gaussian": stats(got_rows)})
    return {"queries_per_index": len(picks), "indexes": rows_out,
            "gaussian_batch_device_ms": round(min(ms), 3),
            "exact": "binary64 squared L2 over all 262,144 coordinates"}


def hierarchy_reference_parity(indexes, specs, seeds, spec_probs, sampled, q_host, picks,
                               answers):
    """Each hierarchy's answers on the picked queries against the reference's
    own HierarchicalL{2,1}AnnIndex (oracle/_ref) built over the same sampled
    columns, with the sample renumbered (the same index: it reads only those
    columns). The reference sampler is run on the same probabilities and seed;
    its sample must equal the engine's and its engine state after sampling
    seeds the reference's projection draws."""
    from oracle import oracle as O

    if not O.ref_available():
        return None
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    equal, samples_equal, total = 0, 0, 0
    per_index = []
    for ix, spec, seed, rows_k, want, pr in zip(indexes, specs, seeds, sampled, answers,
                                                spec_probs):
        cols, mult, invp, state = O.ref_sample(pr, spec["T"], seed)
        cs = ix.coordinate_sample
        same_sample = bool(np.array_equal(cols, cs.source_columns) and
                           np.array_equal(mult, cs.multiplicities) and
                           invp.tobytes() == cs.inverse_probabilities.tobytes())
        got = O.ref_hierarchical_sampled(spec["metric"], rows_k, mult, invp, spec["p"],
                                         state, q_host[:, cols.astype(np.int64)], threads)
        e = int(np.sum(got == want[picks]))
        equal += e
        total += len(picks)
        samples_equal += int(same_sample)
        per_index.append(e)
    return {"queries_per_index": len(picks), "queries": total,
            "equal_to_reference": round(equal / max(1, total), 4),
            "equal_per_index": per_index,
            "samples_equal_to_reference_sampler": samples_equal,
            "reference": "HierarchicalL{2,1}AnnIndex::query on the sampled columns, "
                         f"{threads} threads",
            "seconds": round(time.perf_counter() - t, 1)}


def serving(ds, rates=(10_000, 100_000, 1_000_000, 2_000_000), seconds=0.5, pool=2048):
    """Request loop over 8 device-resident indexes (exact, flat and
    hierarchical, L1 and L2; r from 33 to 65,536; six at d = 60,660 and two
    hierarchies at d = 262,144 with BF16-stored values), Poisson arrivals with
    a uniformly chosen index per request, queries from a device-resident pool
    of each dimension. The 65,536-row flat index is built from a BF16 matrix
    generated on the device (same law, 33 latent classes) with the
    probabilities of the 7,028-row matrix. Plain strategies, then BF16 +
    re-score on the exact and flat L2 indexes; agreement of the exact L2
    answers with the binary64 exact argmin."""
    import torch

    import ultrahigh_ann_b200 as uha
    from ultrahigh_ann_b200 import synthetic

    S = uha.QueryStrategy
    pl2, pl1 = _probabilities("l2", ds.rows), _probabilities("l1", ds.rows)
    r33 = ds.rows[:33]

    def flat_65536():
        big = synthetic.device_row_dataset(rows=65_536, classes=33, queries=1,
                                           d=ds.rows.shape[1], seed=5, storage="bfloat16")
        ix = uha.CudaSampledCoordinateL2AnnIndex(uha.DeviceMatrix.from_torch(big.rows), pl2,
                                                 32, uha.MT19937_64(7))
        del big
        torch.cuda.empty_cache()
        return ix

    build = [
        ("flat_l2_r65536_T32", flat_65536, True),
        ("flat_l2_r33_T8", lambda: uha.CudaSampledCoordinateL2AnnIndex(
            r33, pl2, 8, uha.MT19937_64(1)), True),
        ("exact_l2_r7028", lambda: uha.CudaExactL2Index(ds.rows), True),
        ("flat_l2_r7028_T32", lambda: uha.CudaSampledCoordinateL2AnnIndex(
            ds.rows, pl2, 32, uha.MT19937_64(2)), True),
        ("flat_l1_r7028_T32", lambda: uha.CudaSampledCoordinateL1AnnIndex(
            ds.rows, pl1, 32, uha.MT19937_64(3)), False),
        ("hier_l2_r7028_p64", lambda: uha.CudaHierarchicalL2AnnIndex(
            ds.rows, 32, 64, uha.MT19937_64(4), importance_probabilities=pl2), False),
        ("hier_l2_r2048_p64_d262144", lambda: uha.CudaHierarchicalL2AnnIndex(
            wrows, 32, 64, uha.MT19937_64(5), importance_probabilities=wp2), False),
        ("hier_l1_r1024_p16_d262144", lambda: uha.CudaHierarchicalL1AnnIndex(
            wrows[:1024], 32, 16, uha.MT19937_64(6), importance_probabilities=wp1), False),
    ]
    wrows, wqueries, wp2, wp1, _, _ = _wide_data()
    names = [b[0] for b in build]
    indexes = [b[1]() for b in build]
    qdev = torch.from_numpy(ds.queries[:pool]).cuda()
    wdev = torch.from_numpy(wqueries).cuda()
    # per index: the query pool's base pointer, its row stride and its size
    pools = [(qdev.data_ptr(), ds.rows.shape[1] * 4, pool)] * 6 + \
        [(wdev.data_ptr(), wrows.shape[1] * 4, wqueries.shape[0])] * 2
    base_of = np.array([p[0] for p in pools], np.uint64)
    stride_of = np.array([p[1] for p in pools], np.uint64)
    size_of = np.array([p[2] for p in pools], np.int64)

    def pointers(ids, draws):
        # a uniform query of each request's own pool
        qi = (draws * size_of[ids]).astype(np.int64)
        return qi, (base_of[ids] + qi.astype(np.uint64) * stride_of[ids]).tolist()
    # binary64 exact answers of the pool on the exact L2 index
    ws = indexes[2].make_query_workspace(256)
    exact = np.zeros(pool, np.uint64)
    indexes[2].query_many(qdev.data_ptr(), pool, 256, exact, ws, on_device=True)
    rng = np.random.default_rng(7)
    out = {"indexes": names, "pool_queries": pool, "seconds_per_rate": seconds, "modes": []}
    for mode in ("plain", "bf16_rerank"):
        server = uha.Server(hbm_budget_bytes=16 << 30, max_batch=256, slots=8,
                            queries_on_device=True)
        for (name, _, l2_exact_or_flat), ix in zip(build, indexes):
            st = S.gemm_bf16_rerank if (mode == "bf16_rerank" and l2_exact_or_flat) else S.direct
            sid = server.add_index(ix, st)
            # one workspace per slot up front: creating one mid-run would stop
            # the dispatcher for a warm-up batch
            server.reserve(sid, 8)
        # warm-up load, then the measured rates
        n = 2000
        ids = rng.integers(0, 8, n)
        server.replay(ids, pointers(ids, rng.random(n))[1], np.arange(n) * 50.0)
        server.drain()
        server.poll()
        rows = []
        for rate in rates:
            n = int(rate * seconds)
            ids = rng.integers(0, 8, n).astype(np.uint32)
            qi, ptrs = pointers(ids, rng.random(n))
            arrival = np.cumsum(rng.exponential(1e6 / rate, n))
            server.reset_stats()
            t = time.perf_counter()
            server.replay(ids, ptrs, arrival, np.arange(n))
            server.drain()
            wall = time.perf_counter() - t
            res = server.poll(n)
            st = server.stats()
            order = np.argsort(res["tag"])
            res = res[order]
            sel = ids == 2
            agreement = float(np.mean(res["row"][sel] == exact[qi[sel]])) if sel.any() else None
            rows.append({"offered_qps": rate, "requests": n,
                         "throughput_qps": round(st["throughput_qps"], 1),
                         "p50_ms": round(st["p50_us"] / 1e3, 4),
                         "p99_ms": round(st["p99_us"] / 1e3, 4),
                         "mean_batch": round(st["mean_batch"], 2),
                         "failed": st["failed"], "peak_in_flight": st["peak_in_flight"],
                         "peak_workspace_gb": round(st["peak_workspace_bytes"] / 2**30, 3),
                         "exact_l2_agreement_vs_fp64": agreement,
                         "wall_s": round(wall, 2)})
        out["modes"].append({"mode": mode, "rates": rows})
        del server
    return out


# ------------------------------------------------------------ reference arm
def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    from ultrahigh_ann_b200 import synthetic

    if not O.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference library oracle/_ref/libref.so "
                                         "was not built"}))
        return
    threads = os.cpu_count() or 1
    ds = synthetic.row_dataset(rows=ROWS, classes=33, queries=args.queries, d=DIM,
                               seed=1)
    ref = O.RefExactIndex("l2", ds.rows)
    B = args.batch
    probe = ds.queries[:max(threads, B)]
    t = time.perf_counter()
    ref.query_in_batches(probe, B, threads)
    per = (time.perf_counter() - t) / probe.shape[0]
    # each step: a bounded sample sized for ~8 s of host work, answered in
    # query_batch calls of the configured batch (the reference's automatic
    # strategy: for one query, its scan split over the rows across threads)
    step = max(threads, B)
    sample = int(max(step, min(args.queries, 8.0 / per)))
    sample = max(step, sample // step * step)
    for w in range(args.warmup):
        ref.query_in_batches(ds.queries[:step], B, threads)
    t = time.perf_counter()
    for k in range(args.steps):
        s = (k * sample) % max(1, args.queries - sample)
        ref.query_in_batches(ds.queries[s:s + sample], B, threads)
    secs = time.perf_counter() - t
    value = sample * args.steps / secs
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3),
        "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(secs * 1e3 / args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": headline_config(B, world),
        "queries_per_step": sample,
        "implementation": f"reference ExactL2Index::query_batch, calls of {B} queries, "
                          f"automatic strategy, {threads} OpenMP threads",
        "cpu_baseline": {"value": round(value, 3), "unit": "queries/s",
                         "cores": threads, "kind": "reference",
                         "sample": f"{sample} queries per step in query_batch calls of "
                                   f"{B} (automatic strategy), {threads} threads"},
        "e2e": {"value": round(value, 3), "unit": "queries/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.precision_only or args.only == "precision":
        run_precision_only(args)
    elif args.only:
        run_section(args)
    else:
        run_engine(args)


def run_section(args):
    """One section (batched, serving, centroids, wide, hierarchies or flat)
    alone on one GPU."""
    from ultrahigh_ann_b200 import synthetic

    if args.only == "centroids":
        print(json.dumps({"centroids_flat": centroids_flat()}), flush=True)
        return
    if args.only == "wide":
        print(json.dumps({"wide": wide()}), flush=True)
        return
    if args.only == "hierarchies":
        shape = {}
        if args.hier_shape:
            rows, dim, queries = (int(x) for x in args.hier_shape.split(","))
            shape = {"rows": rows, "dim": dim, "per_index": queries}
        shape["full_probabilities"] = args.full_probabilities
        print(json.dumps({"hierarchies_full": hierarchies_full(**shape)}), flush=True)
        return
    ds = synthetic.row_dataset(rows=ROWS, classes=33, queries=4096, d=DIM, seed=1,
                               query_stream=0)
    if args.only == "flat":
        print(json.dumps({"workload": f"flat_t32_r{ROWS}_d{DIM}", "flat": flat_batch1(ds)}),
              flush=True)
        return
    fn = batched if args.only == "batched" else serving
    print(json.dumps({"workload": f"{args.only}_r{ROWS}_d{DIM}", args.only: fn(ds)}),
          flush=True)


def run_precision_only(args):
    """The precision table alone on one GPU (development runs)."""
    import ultrahigh_ann_b200 as uha
    from ultrahigh_ann_b200 import synthetic

    rows, dim = ROWS, DIM
    if args.precision_shape:
        rows, dim = (int(x) for x in args.precision_shape.split(","))
    ds = synthetic.row_dataset(rows=rows, classes=33, queries=2048, d=dim, seed=1,
                               query_stream=0)
    index = uha.CudaExactL2Index(ds.rows)
    batches = ((args.precision_batch, 2048),) if args.precision_batch else None
    table = precision(ds, index, batches) if batches else precision(ds, index)
    print(json.dumps({"workload": f"exact_l2_r{rows}_d{dim}", "precision": table}),
          flush=True)


if __name__ == "__main__":
    main()
