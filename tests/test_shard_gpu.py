"""Sharding on one GPU: the row shards' plans, run one after another, give
the unsharded forward's rows (FP32 output, relative Frobenius <= 1e-6 -- the
same FP32 sums, possibly in another tensor-core / CUDA-core split); the
column shards give its columns, dB's columns and, summed, dA; one-rank
RowShardedSpMM and ColumnShardedSpMM equal the plain plan in forward and
backward."""
import numpy as np
import pytest

from tca_spmm import gen, shard

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402


def rel(x, y):
    x, y = x.double().cpu(), y.double().cpu()
    return float((x - y).norm() / max(float(y.norm()), 1e-300))


@pytest.mark.parametrize("n_shards", [1, 2, 3, 8])
def test_shards_reassemble_the_forward(cuda, n_shards):
    c = gen.sweep(0.90, N=128, seed=17)
    B = torch.from_numpy(c["B"]).to(cuda)
    full = tca_spmm.Plan(*(torch.from_numpy(x.copy()).to(cuda) for x in (c["row_ptr"], c["col"], c["vals"])),
                         c["K"]).spmm(B, out_dtype=torch.float32)
    b = shard.partition_rows(c["row_ptr"], n_shards)
    parts = []
    for k in range(n_shards):
        rp, ci, v = shard.slice_csr(c["row_ptr"], c["col"], c["vals"], b[k], b[k + 1])
        p = tca_spmm.Plan(torch.from_numpy(rp).to(cuda), torch.from_numpy(ci).to(cuda),
                          torch.from_numpy(v).to(cuda), c["K"])
        parts.append(p.spmm(B, out_dtype=torch.float32))
    torch.cuda.synchronize()
    assert rel(torch.cat(parts), full) <= 1e-6


def test_one_rank_sharded_equals_plan(cuda):
    c = gen.small(np.random.default_rng(4), 600, 200, 64, 0.1)
    B = torch.from_numpy(c["B"]).to(cuda)
    dY = torch.from_numpy(np.random.default_rng(5).standard_normal((600, 64)).astype(np.float16)).to(cuda)
    sh = shard.RowShardedSpMM(c["row_ptr"], c["col"], c["vals"], c["K"], cuda)
    p = tca_spmm.Plan(*(torch.from_numpy(x.copy()).to(cuda) for x in (c["row_ptr"], c["col"], c["vals"])), c["K"])
    assert rel(sh.forward(B, out_dtype=torch.float32), p.spmm(B, out_dtype=torch.float32)) <= 1e-6
    dA, dB = sh.backward(dY, B)
    assert rel(dA, p.sddmm(dY, B)) <= 1e-6 and rel(dB, p.spmm_t(dY)) <= 1e-6


@pytest.mark.parametrize("n_shards", [2, 3])
def test_column_shards_reassemble_forward_and_backward(cuda, n_shards):
    """Column sharding run shard by shard on one GPU: the column blocks of Y
    and dB are the full ones' columns, and dA summed over the blocks is the
    full SDDMM (FP32 outputs, relative Frobenius <= 1e-5: sums of the same
    products in a different grouping)."""
    c = gen.sweep(0.90, N=256, seed=19)
    N = c["N"]
    B = torch.from_numpy(c["B"]).to(cuda)
    dY = torch.from_numpy(np.random.default_rng(6).standard_normal((c["M"], N)).astype(np.float16)).to(cuda)
    p = tca_spmm.Plan(*(torch.from_numpy(x.copy()).to(cuda) for x in (c["row_ptr"], c["col"], c["vals"])), c["K"])
    y_full, dA_full, dB_full = p.spmm(B, out_dtype=torch.float32), p.sddmm(dY, B), p.spmm_t(dY)
    b = shard.partition_cols(N, n_shards)
    ys, dBs, dA = [], [], torch.zeros_like(dA_full)
    for k in range(n_shards):
        Bk, dYk = B[:, b[k]:b[k + 1]], dY[:, b[k]:b[k + 1]]
        ys.append(p.spmm(Bk, out_dtype=torch.float32))
        dBs.append(p.spmm_t(dYk))
        dA += p.sddmm(dYk, Bk)
    torch.cuda.synchronize()
    assert rel(torch.cat(ys, dim=1), y_full) <= 1e-5
    assert rel(torch.cat(dBs, dim=1), dB_full) <= 1e-5
    assert rel(dA, dA_full) <= 1e-5


def test_one_rank_column_sharded_equals_plan(cuda):
    c = gen.small(np.random.default_rng(7), 500, 300, 72, 0.1)
    B = torch.from_numpy(c["B"]).to(cuda)
    dY = torch.from_numpy(np.random.default_rng(8).standard_normal((500, 72)).astype(np.float16)).to(cuda)
    sh = shard.ColumnShardedSpMM(c["row_ptr"], c["col"], c["vals"], c["K"], 72, cuda)
    assert sh.cols == (0, 72)
    p = tca_spmm.Plan(*(torch.from_numpy(x.copy()).to(cuda) for x in (c["row_ptr"], c["col"], c["vals"])), c["K"])
    assert rel(sh.forward(B, out_dtype=torch.float32), p.spmm(B, out_dtype=torch.float32)) <= 1e-6
    dA, dB = sh.backward(dY, B)
    assert rel(dA, p.sddmm(dY, B)) <= 1e-6 and rel(dB, p.spmm_t(dY)) <= 1e-6
