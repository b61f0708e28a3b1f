"""Row sharding on one GPU: the shards' plans, run one after another, give
the unsharded forward's rows (FP32 output, relative Frobenius <= 1e-6 -- the
same FP32 sums, possibly in another tensor-core / CUDA-core split), and a
one-rank RowShardedSpMM equals the plain plan in forward and backward."""
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
