"""Sharding of the SpMM over the ranks of a torch.distributed group.

Row sharding: the forward Y = A B shards by rows with no exchange: rank k
owns a contiguous range of A's rows (balanced by nonzeros), B is replicated,
and it computes Y[rows_k] with its own plan. Gathering Y on every rank is
optional (gather_rows). The backward is local for dA (SDDMM on the rank's
rows); dB = A^T dY is a sum over the row shards (reduce_grad_b: one
all-reduce of K x N).

Column sharding: A (one plan) is replicated, B and Y are cut into column
ranges; the forward has no exchange (gather_cols optionally assembles Y),
dB = A^T dY is local to the columns, and dA, a sum over the column ranges of
SDDMM(dY_k, B_k), is one all-reduce of nnz values (reduce_grad_a).

Batches of layers: independent replicas, layers dealt to the ranks by
longest-processing-time first (assign_layers_lpt), no communication.

The reference has no multi-GPU code; this is the rebuild's sharding layer.
Plumbing (partitioning, slicing, the collectives) is plain numpy and
torch.distributed, so it runs with any backend; the compute is the CUDA
library through tca_spmm.Plan.
"""
from __future__ import annotations

import numpy as np


def partition_rows(row_ptr, n_shards: int) -> np.ndarray:
    """Boundaries b[0] = 0 <= b[1] <= ... <= b[n_shards] = M of contiguous row
    ranges whose nonzero counts are as equal as a split at row boundaries
    allows: b[k] is the first row at which the running nonzero count reaches
    k / n_shards of the total (rows are cut by count, not by work estimate).
    A matrix with no nonzeros is cut by rows."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    M = rp.size - 1
    if n_shards < 1:
        raise ValueError("n_shards must be >= 1")
    nnz = int(rp[-1]) if M >= 0 else 0
    b = np.zeros(n_shards + 1, dtype=np.int64)
    b[-1] = M
    for k in range(1, n_shards):
        if nnz == 0:
            b[k] = (M * k) // n_shards
        else:
            target = (nnz * k + n_shards - 1) // n_shards  # ceil(k * nnz / n)
            b[k] = int(np.searchsorted(rp, target, side="left"))
        b[k] = min(max(b[k], b[k - 1]), M)
    return b


def slice_csr(row_ptr, col_idx, vals, r0: int, r1: int):
    """Rows [r0, r1) of a CSR as a CSR of their own (row offsets rebased to 0)."""
    rp = np.asarray(row_ptr)
    j0, j1 = int(rp[r0]), int(rp[r1])
    return ((rp[r0:r1 + 1] - j0).astype(np.int32), np.ascontiguousarray(np.asarray(col_idx)[j0:j1]),
            np.ascontiguousarray(np.asarray(vals)[j0:j1]))


def gather_rows(local, bounds, group=None):
    """Every rank's row block (rank k: rows bounds[k]..bounds[k+1] of the
    result) concatenated in rank order, on every rank: one all_gather of
    blocks padded to the largest shard."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    sizes = [int(bounds[k + 1] - bounds[k]) for k in range(world)]
    width = local.shape[1]
    pad = max(sizes) if sizes else 0
    buf = torch.zeros((pad, width), dtype=local.dtype, device=local.device)
    buf[: local.shape[0]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([p[:n] for p, n in zip(parts, sizes)], dim=0)


def reduce_grad_b(partial, group=None):
    """dB = sum over the row shards of A_k^T dY_k: one in-place all-reduce."""
    import torch.distributed as dist
    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial


class RowShardedSpMM:
    """This rank's share of a row-sharded SpMM: the rows bounds[rank] ..
    bounds[rank + 1] of A (host CSR in), as a tca_spmm.Plan on `device`."""

    def __init__(self, row_ptr, col_idx, vals, K: int, device, group=None, **plan_opts):
        import torch
        import torch.distributed as dist
        from . import Plan
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.bounds = partition_rows(row_ptr, self.world)
        r0, r1 = int(self.bounds[self.rank]), int(self.bounds[self.rank + 1])
        rp, ci, v = slice_csr(row_ptr, col_idx, vals, r0, r1)
        self.rows = (r0, r1)
        self.plan = Plan(torch.from_numpy(rp).to(device), torch.from_numpy(ci).to(device),
                         torch.from_numpy(np.asarray(v, dtype=np.float16)).to(device), K, **plan_opts)

    def forward(self, B, out_dtype=None, gather=False):
        """Y[rows] = A[rows] B on this rank; with gather=True the full Y on every rank."""
        y = self.plan.spmm(B, out_dtype=out_dtype)
        return gather_rows(y, self.bounds, self.group) if gather and self.world > 1 else y

    def backward(self, dY_local, B):
        """(dA of this rank's nonzeros, dB summed over all ranks)."""
        dA = self.plan.sddmm(dY_local, B)
        dB = self.plan.spmm_t(dY_local)
        if self.world > 1:
            reduce_grad_b(dB, self.group)
        return dA, dB


def partition_cols(N: int, n_shards: int, align: int = 8) -> np.ndarray:
    """Boundaries c[0] = 0 <= ... <= c[n_shards] = N of contiguous column
    ranges of B and Y, as equal as multiples of `align` allow (a column
    range of an FP16 B at a multiple of 8 keeps its rows 16-byte aligned)."""
    if n_shards < 1:
        raise ValueError("n_shards must be >= 1")
    units = -(-N // align)
    c = np.array([min(N, (units * k // n_shards) * align) for k in range(n_shards + 1)], dtype=np.int64)
    c[-1] = N
    return c


def gather_cols(local, bounds, group=None):
    """Every rank's column block (rank k: columns bounds[k]..bounds[k+1] of
    the result) side by side in rank order, on every rank: one all_gather of
    blocks padded to the widest shard."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    widths = [int(bounds[k + 1] - bounds[k]) for k in range(world)]
    pad = max(widths) if widths else 0
    buf = torch.zeros((local.shape[0], pad), dtype=local.dtype, device=local.device)
    buf[:, : local.shape[1]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([p[:, :w] for p, w in zip(parts, widths)], dim=1)


def reduce_grad_a(partial, group=None):
    """dA (values on A's pattern) = sum over the column shards of
    SDDMM(dY_k, B_k): one in-place all-reduce of nnz values."""
    import torch.distributed as dist
    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial


class ColumnShardedSpMM:
    """This rank's share of a column-sharded SpMM: all of A (host CSR in) as
    a tca_spmm.Plan on `device`; the rank works on columns
    bounds[rank] .. bounds[rank + 1] of B, Y and dY."""

    def __init__(self, row_ptr, col_idx, vals, K: int, N: int, device, group=None, **plan_opts):
        import torch
        import torch.distributed as dist
        from . import Plan
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.bounds = partition_cols(N, self.world)
        self.cols = (int(self.bounds[self.rank]), int(self.bounds[self.rank + 1]))
        self.plan = Plan(torch.from_numpy(np.asarray(row_ptr, np.int32)).to(device),
                         torch.from_numpy(np.asarray(col_idx, np.int32)).to(device),
                         torch.from_numpy(np.asarray(vals, dtype=np.float16)).to(device), K, **plan_opts)

    def forward(self, B_local, out_dtype=None, gather=False):
        """Y[:, cols] = A B[:, cols] on this rank; with gather=True the full Y on every rank."""
        y = self.plan.spmm(B_local, out_dtype=out_dtype)
        return gather_cols(y, self.bounds, self.group) if gather and self.world > 1 else y

    def backward(self, dY_local, B_local):
        """(dA summed over all ranks, dB of this rank's columns)."""
        import torch
        dA = self.plan.sddmm(dY_local, B_local, out_dtype=torch.float32)
        if self.world > 1:
            reduce_grad_a(dA, self.group)
        dB = self.plan.spmm_t(dY_local)
        return dA, dB


def assign_layers_lpt(costs, n_ranks: int):
    """Layers (costs[i] >= 0, e.g. 2 nnz N) dealt to n_ranks replicas by
    longest processing time first: in decreasing cost (ties by index), each
    layer goes to the rank with the least total so far (ties to the lowest
    rank). Returns, per rank, its layer indices in increasing order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    load = np.zeros(n_ranks)
    out = [[] for _ in range(n_ranks)]
    for i in sorted(range(costs.size), key=lambda j: (-costs[j], j)):
        r = int(np.argmin(load))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]
