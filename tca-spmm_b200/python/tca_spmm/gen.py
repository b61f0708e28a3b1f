"""Seeded synthetic CSR inputs for the benchmark shapes.

The reference ships one pattern-only .smtx fixture; the matrices its name
points to are not available, so seeded synthetic matrices with the stated
shapes, sparsities and value distributions stand in for them. All generators
use numpy's PCG64 (default_rng) and return host numpy arrays:
row_ptr/col_idx int32, vals float16, B float16, columns sorted in each row.
"""
from __future__ import annotations

import numpy as np


def _csr_from_row_nnz(rng, row_nnz: np.ndarray, K: int):
    """Distinct uniform columns per row (without replacement), sorted."""
    M = row_nnz.size
    row_nnz = np.asarray(row_nnz, dtype=np.int64)
    keys = rng.random((M, K), dtype=np.float32)
    order = np.argsort(keys, axis=1, kind="stable")
    rank = np.empty_like(order)
    np.put_along_axis(rank, order, np.broadcast_to(np.arange(K), (M, K)), axis=1)
    mask = rank < row_nnz[:, None]
    rows, cols = np.nonzero(mask)
    row_ptr = np.zeros(M + 1, dtype=np.int32)
    np.cumsum(row_nnz, out=row_ptr[1:])
    return row_ptr, cols.astype(np.int32)


def zipf_row_nnz(rng, M: int, K: int, total: int, a: float = 1.2) -> np.ndarray:
    """Row lengths proportional to Zipf(a) draws, clipped to [1, K], rescaled
    to exactly `total`: bisection on the scale c of clip(rint(w c), 1, K), then
    +-1 corrections on the rows with the largest draws that still have room."""
    total = int(min(max(total, M), M * K))
    w = rng.zipf(a, size=M).astype(np.float64)
    lo, hi = 0.0, float(K)
    while np.clip(np.rint(w * hi), 1, K).sum() < total:
        hi *= 2.0
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if np.clip(np.rint(w * mid), 1, K).sum() < total:
            lo = mid
        else:
            hi = mid
    n = np.clip(np.rint(w * hi), 1, K).astype(np.int64)
    diff = total - int(n.sum())
    order = np.argsort(-w, kind="stable")
    i = 0
    while diff != 0:
        r = order[i % M]
        if diff > 0 and n[r] < K:
            n[r] += 1
            diff -= 1
        elif diff < 0 and n[r] > 1:
            n[r] -= 1
            diff += 1
        i += 1
    return n


def random_csr(rng, M, K, row_nnz, val_std):
    row_ptr, col = _csr_from_row_nnz(rng, row_nnz, K)
    vals = (rng.standard_normal(col.size) * val_std).astype(np.float16)
    return row_ptr, col, vals


def uniform_b(rng, K, N):
    return rng.uniform(-1.0, 1.0, size=(K, N)).astype(np.float16)


def cfg1(seed: int = 0):
    """2048 x 512 at 80% sparsity, row nnz ~ Binomial(512, 0.2), values
    N(0, 1/sqrt(512)), B 512 x 256 U(-1, 1)."""
    rng = np.random.default_rng(seed)
    M, K, N = 2048, 512, 256
    row_nnz = rng.binomial(K, 0.2, size=M)
    row_ptr, col, vals = random_csr(rng, M, K, row_nnz, 1.0 / np.sqrt(512.0))
    return dict(name="cfg1", M=M, K=K, N=N, row_ptr=row_ptr, col=col, vals=vals, B=uniform_b(rng, K, N))


def sweep(sparsity: float, N: int = 256, seed: int | None = None, M: int = 4096, K: int = 1024):
    """4096 x 1024, Zipf(1.2) row lengths at the given sparsity, values
    N(0, 0.03), B K x N U(-1, 1)."""
    pct = int(round(sparsity * 100))
    rng = np.random.default_rng(1000 + pct if seed is None else seed)
    total = int(round((1.0 - sparsity) * M * K))
    row_nnz = zipf_row_nnz(rng, M, K, total)
    row_ptr, col, vals = random_csr(rng, M, K, row_nnz, 0.03)
    return dict(name=f"sweep{pct}_N{N}", M=M, K=K, N=N, row_ptr=row_ptr, col=col, vals=vals,
                B=uniform_b(rng, K, N))


def diff(seed: int = 3, N: int = 4096):
    """2048 x 512 at 90% sparsity with uniform row lengths (51 or 52 nnz),
    values N(0, 0.044); B 512 x N and dY 2048 x N, both N(0, 1)."""
    rng = np.random.default_rng(seed)
    M, K = 2048, 512
    total = int(round(0.1 * M * K))
    row_nnz = np.full(M, total // M, dtype=np.int64)
    row_nnz[: total - row_nnz.sum()] += 1
    row_ptr, col, vals = random_csr(rng, M, K, row_nnz, 0.044)
    B = rng.standard_normal((K, N)).astype(np.float16)
    dY = rng.standard_normal((M, N)).astype(np.float16)
    return dict(name="diff", M=M, K=K, N=N, row_ptr=row_ptr, col=col, vals=vals, B=B, dY=dY)


def precision(seed: int = 4, N: int = 1024):
    """4096 x 4096 at ~90% sparsity, row lengths ~ Poisson(410) clipped to
    [0, 4096], values N(0, 0.016); B 4096 x N N(0, 1)."""
    rng = np.random.default_rng(seed)
    M = K = 4096
    row_nnz = np.clip(rng.poisson(410, size=M), 0, K)
    row_ptr, col, vals = random_csr(rng, M, K, row_nnz, 0.016)
    B = rng.standard_normal((K, N)).astype(np.float16)
    return dict(name="precision", M=M, K=K, N=N, row_ptr=row_ptr, col=col, vals=vals, B=B)


def batch_layers(seed: int = 5):
    """24 layers: six each of 512x2048, 2048x512, 512x512, 1024x4096; sparsity
    U[0.5, 0.98]; Binomial row lengths; values N(0, 1/sqrt(cols)); per-layer
    N from {64, 128, 256, 512, 1024}; B U(-1, 1)."""
    rng = np.random.default_rng(seed)
    shapes = [(512, 2048)] * 6 + [(2048, 512)] * 6 + [(512, 512)] * 6 + [(1024, 4096)] * 6
    layers = []
    for li, (M, K) in enumerate(shapes):
        s = rng.uniform(0.5, 0.98)
        N = int(rng.choice([64, 128, 256, 512, 1024]))
        row_nnz = rng.binomial(K, 1.0 - s, size=M)
        row_ptr, col, vals = random_csr(rng, M, K, row_nnz, 1.0 / np.sqrt(K))
        layers.append(dict(name=f"layer{li}", M=M, K=K, N=N, sparsity=s, row_ptr=row_ptr, col=col,
                           vals=vals, B=uniform_b(rng, K, N)))
    return layers


def small(rng, M, K, N, density, val_std=0.5, empty_rows=0.0):
    """A small random case for parity tests; `empty_rows` is the fraction of
    rows forced empty."""
    row_nnz = rng.binomial(K, density, size=M)
    if empty_rows > 0:
        row_nnz[rng.random(M) < empty_rows] = 0
    row_ptr, col, vals = random_csr(rng, M, K, row_nnz, val_std)
    return dict(M=M, K=K, N=N, row_ptr=row_ptr, col=col, vals=vals, B=uniform_b(rng, K, N))
