"""Seeded synthetic stand-ins for the TCGA Pan-Cancer shapes the reference is
measured on (d = 60,660 expression coordinates; 33 class centroids or 7,028
individual rows; held-out queries). The TCGA data itself is not available, so
values follow a log-expression-like law:

    x ~ Gamma(shape=0.5, scale=200), value = log2(1 + x),

with one fixed mask that zeroes 40% of the coordinates in every reference row.
A query (and, for row-level indexes, a reference row) is a class centroid plus
N(0, sigma^2) noise clipped at 0.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

TCGA_DIMENSION = 60660


@dataclass
class Dataset:
    rows: np.ndarray       # r x d float32 reference rows
    queries: np.ndarray    # n x d float32 queries
    query_class: np.ndarray  # latent class of each query
    row_class: np.ndarray    # latent class of each row


def _centroids(rng: np.random.Generator, classes: int, d: int,
               zero_fraction: float) -> tuple[np.ndarray, np.ndarray]:
    x = rng.gamma(0.5, 200.0, size=(classes, d))
    cent = np.log2(1.0 + x).astype(np.float32)
    mask = rng.random(d) < zero_fraction
    cent[:, mask] = 0.0
    return cent, mask


def _noisy(rng: np.random.Generator, base: np.ndarray, labels: np.ndarray,
           sigma: float, chunk: int = 512) -> np.ndarray:
    out = np.empty((labels.size, base.shape[1]), dtype=np.float32)
    for s in range(0, labels.size, chunk):
        e = min(labels.size, s + chunk)
        noise = rng.standard_normal((e - s, base.shape[1]), dtype=np.float32)
        block = base[labels[s:e]] + np.float32(sigma) * noise
        np.maximum(block, 0.0, out=block)
        out[s:e] = block
    return out


def centroid_dataset(classes: int = 33, queries: int = 3013,
                     d: int = TCGA_DIMENSION, sigma: float = 0.8,
                     zero_fraction: float = 0.4, seed: int = 0) -> Dataset:
    """The 33-centroid workload: reference rows are the class centroids."""
    rng = np.random.default_rng(seed)
    cent, _ = _centroids(rng, classes, d, zero_fraction)
    labels = rng.integers(0, classes, size=queries)
    q = _noisy(rng, cent, labels, sigma)
    return Dataset(cent, q, labels, np.arange(classes))


def row_dataset(rows: int = 7028, classes: int = 33, queries: int = 8192,
                d: int = TCGA_DIMENSION, sigma: float = 0.8,
                zero_fraction: float = 0.4, seed: int = 1,
                query_stream: int = 0) -> Dataset:
    """The row-level workload: every reference row is a latent class centroid
    plus noise; the masked coordinates stay zero in every row. Queries come
    from their own random stream, so `query_stream` selects an independent
    query set over the same rows (one per replica in a multi-GPU run)."""
    rng = np.random.default_rng([seed, 0])
    cent, mask = _centroids(rng, classes, d, zero_fraction)
    row_labels = rng.integers(0, classes, size=rows)
    r = _noisy(rng, cent, row_labels, sigma)
    r[:, mask] = 0.0
    qrng = np.random.default_rng([seed, 1, query_stream])
    q_labels = qrng.integers(0, classes, size=queries)
    q = _noisy(qrng, cent, q_labels, sigma)
    return Dataset(r, q, q_labels, row_labels)


@dataclass
class DeviceDataset:
    rows: "object"          # r x d torch tensor on the device (float32 or bfloat16)
    queries: "object"       # n x d float32 torch tensor on the device
    query_class: np.ndarray
    row_class: np.ndarray


def device_row_dataset(rows: int, classes: int = 33, queries: int = 4096,
                       d: int = TCGA_DIMENSION, sigma: float = 0.8,
                       zero_fraction: float = 0.4, seed: int = 1,
                       storage: str = "bfloat16", device: int = 0,
                       chunk: int = 1024) -> DeviceDataset:
    """The row-level workload generated on the device, for sizes whose host
    matrix would not fit host memory (65,536 x 262,144 values): the same law
    as row_dataset (class centroids drawn on the host with numpy, per-value
    N(0, sigma^2) noise from torch's device generator, clipped at 0, masked
    columns zero in the rows). Rows are stored as `storage` (BF16 rounds to nearest
    even); queries hold the binary32 values of the same storage type, so
    queries and rows share one value grid. Different random streams than
    row_dataset: the values are not the same as a host dataset's."""
    import torch

    rng = np.random.default_rng([seed, 0])
    cent, mask = _centroids(rng, classes, d, zero_fraction)
    row_labels = rng.integers(0, classes, size=rows)
    q_labels = np.random.default_rng([seed, 1]).integers(0, classes, size=queries)
    dev = torch.device("cuda", device)
    cent_t = torch.from_numpy(cent).to(dev)
    keep = torch.from_numpy(~mask).to(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    dtype = torch.bfloat16 if storage == "bfloat16" else torch.float32

    def fill(out, labels, store_dtype, masked):
        for s in range(0, labels.size, chunk):
            e = min(labels.size, s + chunk)
            lab = torch.from_numpy(labels[s:e]).to(dev)
            block = torch.randn((e - s, d), generator=gen, device=dev)
            block.mul_(sigma).add_(cent_t[lab]).clamp_(min=0.0)
            if masked:
                block.mul_(keep)
            out[s:e] = block.to(store_dtype).to(out.dtype)
        return out

    r = fill(torch.empty((rows, d), dtype=dtype, device=dev), row_labels, dtype, True)
    q = fill(torch.empty((queries, d), dtype=torch.float32, device=dev), q_labels, dtype,
             False)
    return DeviceDataset(r, q, q_labels, row_labels)
