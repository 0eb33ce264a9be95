"""Generates the golden fixtures in tests/golden/ by running the REFERENCE
itself (its CPU library compiled from its own sources into oracle/_ref by
oracle/Makefile) on small seeded inputs.

    python tests/golden/make_golden.py

inputs.npz holds the shared rows and queries; every other .npz holds the
parameters and the reference outputs of one case. Inputs are
seeded synthetic log-expression data (ultrahigh_ann_b200.synthetic) plus a
few planted near-ties (duplicate rows, rows one ulp apart, equal-distance
rows) so that the argmin's lowest-index rule is exercised.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from ultrahigh_ann_b200 import synthetic  # noqa: E402

OUT = Path(__file__).resolve().parent


def planted(rows: np.ndarray, queries: np.ndarray, rng: np.random.Generator):
    """Adds near-tie structure: a duplicate of row 3 at the end, a copy of row 5
    one ulp away in one coordinate, and queries equal to a row midpoint."""
    rows = rows.copy()
    dup = rows[3].copy()
    ulp = rows[5].copy()
    j = int(np.argmax(ulp))
    ulp[j] = np.nextafter(ulp[j], np.float32(np.inf))
    rows = np.vstack([rows, dup[None], ulp[None]])
    q = queries.copy()
    q[0] = rows[3]                      # exact hit on a duplicated row
    q[1] = 0.5 * (rows[5] + rows[-1])   # between a row and its ulp copy
    q[2] = rows[-1]
    return rows.astype(np.float32), q.astype(np.float32)


def main() -> None:
    if not O.ref_available():
        O.build()
    rng = np.random.default_rng(20251203)
    ds = synthetic.centroid_dataset(classes=46, queries=96, d=777, seed=17)
    rows, queries = planted(ds.rows, ds.queries, rng)
    r, d = rows.shape

    cases = {"inputs": dict(rows=rows, queries=queries)}
    # exact scans
    for metric in ("l2", "l1"):
        cases[f"exact_{metric}"] = dict(
            indices=O.ref_exact(metric, rows, queries, threads=1))
    # importance probabilities (reference sequential policy)
    probs = {m: O.ref_probabilities(m, rows, parallel=False) for m in ("l2", "l1")}
    for metric in ("l2", "l1"):
        cases[f"probabilities_{metric}"] = dict(probabilities=probs[metric])
    # flat (sampled-coordinate) indexes
    for metric, reps, seed in (("l2", 8, 7), ("l1", 8, 9), ("l2", 32, 5)):
        cols, mult, inv, state = O.ref_sample(probs[metric], reps, seed)
        cases[f"flat_{metric}_t{reps}"] = dict(
            probabilities=probs[metric],
            repetitions=np.uint64(reps), seed=np.uint64(seed), columns=cols,
            multiplicities=mult, inverse_probabilities=inv,
            engine_state=np.frombuffer(state.encode(), dtype=np.uint8),
            indices=O.ref_sampled(metric, rows, cols, mult, inv, queries))
    # hierarchical indexes (odd and even projection dimension)
    for metric, p, seed in (("l2", 16, 11), ("l2", 15, 12), ("l1", 16, 13),
                            ("l1", 15, 14)):
        cols, mult, inv, state = O.ref_sample(probs[metric], 8, seed)
        matrix, reps_ = O.ref_projection(metric, rows, cols, mult, inv, p, state)
        idx, state_after = O.ref_hierarchical(metric, rows, probs[metric], 8, p, seed,
                                              queries)
        cases[f"hier_{metric}_p{p}"] = dict(
            probabilities=probs[metric],
            repetitions=np.uint64(8), projection_dimension=np.uint64(p),
            seed=np.uint64(seed), columns=cols, multiplicities=mult,
            inverse_probabilities=inv, projection=matrix, projected_rows=reps_,
            engine_state_after=np.frombuffer(state_after.encode(), dtype=np.uint8),
            indices=idx)
    for name, arrays in cases.items():
        np.savez_compressed(OUT / f"{name}.npz", **arrays)
        print(name, {k: v.shape for k, v in arrays.items() if hasattr(v, "shape")})


if __name__ == "__main__":
    main()
