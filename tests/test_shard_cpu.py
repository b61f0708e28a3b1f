"""Row sharding (tca_spmm.shard) on the CPU: partition balance and coverage,
CSR slicing, and the two collectives of the sharded SpMM -- gathering the row
blocks of Y and summing the partial dB = A_k^T dY_k -- run by two `gloo` ranks
in separate processes, each computing its shard with the FP64 oracle.
Bit-for-bit equality with the unsharded FP64 result is expected for the
gather (a copy) and 1e-12 relative for the sum (two FP64 addends)."""
import os
import socket

import numpy as np
import pytest

from oracle import oracle
from tca_spmm import gen, shard

torch = pytest.importorskip("torch")


def test_partition_balances_nonzeros_and_covers_every_row():
    rng = np.random.default_rng(0)
    for M, n in [(1000, 2), (1000, 7), (5, 8), (1, 3)]:
        c = gen.small(rng, M, 64, 8, 0.2, empty_rows=0.2)
        b = shard.partition_rows(c["row_ptr"], n)
        assert b[0] == 0 and b[-1] == M and (np.diff(b) >= 0).all()
        nnz = np.diff(c["row_ptr"][b])
        if M >= 100:  # each shard within one row of the ideal share
            assert nnz.max() - nnz.sum() / n <= np.diff(c["row_ptr"]).max()
    z = shard.partition_rows(np.zeros(11, np.int32), 4)  # no nonzeros: cut by rows
    np.testing.assert_array_equal(z, [0, 2, 5, 7, 10])
    one = shard.partition_rows(np.array([0, 0, 100, 100], np.int32), 2)  # all nonzeros in one row
    assert one[0] == 0 and one[-1] == 3


def test_slice_csr_round_trips():
    rng = np.random.default_rng(1)
    c = gen.small(rng, 300, 50, 8, 0.1, empty_rows=0.1)
    b = shard.partition_rows(c["row_ptr"], 3)
    parts = [shard.slice_csr(c["row_ptr"], c["col"], c["vals"], b[k], b[k + 1]) for k in range(3)]
    np.testing.assert_array_equal(np.concatenate([p[1] for p in parts]), c["col"])
    np.testing.assert_array_equal(np.concatenate([p[2] for p in parts]), c["vals"])
    rp = np.concatenate([parts[0][0]] + [p[0][1:] + sum(q[0][-1] for q in parts[:k + 1])
                                         for k, p in enumerate(parts[1:])])
    np.testing.assert_array_equal(rp, c["row_ptr"])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, seed):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(seed)
        c = gen.small(rng, 257, 96, 24, 0.15, empty_rows=0.1)
        dY = rng.standard_normal((c["M"], 24))
        b = shard.partition_rows(c["row_ptr"], world)
        r0, r1 = int(b[rank]), int(b[rank + 1])
        rp, ci, v = shard.slice_csr(c["row_ptr"], c["col"], c["vals"], r0, r1)
        y_local = torch.from_numpy(oracle.spmm_f64(rp, ci, v, c["B"]))
        y = shard.gather_rows(y_local, b).numpy()
        np.testing.assert_array_equal(y, oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], c["B"]))
        # partial dB = A_k^T dY_k, summed over the ranks
        rows = np.repeat(np.arange(r1 - r0), np.diff(rp))
        part = np.zeros((c["K"], 24))
        np.add.at(part, ci, v.astype(np.float64)[:, None] * dY[r0:r1][rows])
        dB = shard.reduce_grad_b(torch.from_numpy(part)).numpy()
        rows_all = np.repeat(np.arange(c["M"]), np.diff(c["row_ptr"]))
        full = np.zeros((c["K"], 24))
        np.add.at(full, c["col"], c["vals"].astype(np.float64)[:, None] * dY[rows_all])
        assert np.linalg.norm(dB - full) <= 1e-12 * np.linalg.norm(full)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_rows_and_sum_grad_b():
    import torch.multiprocessing as mp
    mp.spawn(_rank, args=(2, _free_port(), 123), nprocs=2, join=True)


def test_partition_cols_covers_and_aligns():
    for N, n in [(256, 2), (264, 4), (8, 3), (100, 3), (1, 2)]:
        c = shard.partition_cols(N, n)
        assert c[0] == 0 and c[-1] == N and (np.diff(c) >= 0).all()
        assert all(x % 8 == 0 for x in c[:-1])
        w = np.diff(c)
        assert w.max() - w.min() <= 8 or N < 8 * n


def test_assign_layers_lpt():
    costs = [7, 3, 9, 1, 4, 4, 8]
    out = shard.assign_layers_lpt(costs, 3)
    assert sorted(i for r in out for i in r) == list(range(len(costs)))
    # 9 -> r0, 8 -> r1, 7 -> r2, 4 (#4) -> r2, 4 (#5) -> r1, 3 -> r0, 1 -> r2
    assert out == [[1, 2], [5, 6], [0, 3, 4]]
    assert [sum(costs[i] for i in r) for r in out] == [12, 12, 12]
    assert shard.assign_layers_lpt([5, 5], 4) == [[0], [1], [], []]
    assert shard.assign_layers_lpt([], 2) == [[], []]
    # the batching config's 24 layers over 8 replicas: LPT within 4/3 of the optimum bound
    ls = gen.batch_layers()
    cost = [2.0 * c["col"].size * c["N"] for c in ls]
    per = shard.assign_layers_lpt(cost, 8)
    loads = [sum(cost[i] for i in r) for r in per]
    assert max(loads) <= 4.0 / 3.0 * max(sum(cost) / 8, max(cost)) + 1e-9


def _rank_cols(rank, world, port, seed):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(seed)
        N = 40
        c = gen.small(rng, 131, 77, N, 0.15, empty_rows=0.1)
        dY = rng.standard_normal((c["M"], N))
        b = shard.partition_cols(N, world)
        c0, c1 = int(b[rank]), int(b[rank + 1])
        Bk = c["B"][:, c0:c1]
        y_local = torch.from_numpy(oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], Bk))
        y = shard.gather_cols(y_local, b).numpy()
        np.testing.assert_array_equal(y, oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], c["B"]))
        # partial dA = SDDMM(dY_k, B_k) on A's pattern, summed over the ranks
        rows = np.repeat(np.arange(c["M"]), np.diff(c["row_ptr"]))
        B64 = c["B"].astype(np.float64)
        part = np.einsum("ij,ij->i", dY[rows][:, c0:c1], B64[c["col"]][:, c0:c1])
        dA = shard.reduce_grad_a(torch.from_numpy(part)).numpy()
        full = np.einsum("ij,ij->i", dY[rows], B64[c["col"]])
        assert np.linalg.norm(dA - full) <= 1e-12 * np.linalg.norm(full)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_cols_and_sum_grad_a():
    import torch.multiprocessing as mp
    mp.spawn(_rank_cols, args=(2, _free_port(), 321), nprocs=2, join=True)
