"""The FP16 tensor-core item kernel of the CUDA-core rows (cc_cols =
CC_COLS_MMA) against the FP64 oracle, with the tolerances of
test_spmm_gpu.assert_close: every N class (multiples of 8, slices of 64
columns with a ragged last slice), FP16 and FP32 output, rows of 0 to 1000
nonzeros (an item longer than 32 nonzeros is walked in pieces), alpha/beta
and kept empty rows, strided operands, and a mixed tensor-core/CUDA-core
plan in a batch."""
import numpy as np
import pytest

from tca_spmm import gen
from test_spmm_gpu import assert_close, dev

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402

MMA = tca_spmm.CC_COLS_MMA


def run(plan, B, C, **kw):
    tca_spmm.spmm_batched([plan], [B], [C], cc_cols=MMA, **kw)
    torch.cuda.synchronize()
    plan.status()
    return C


@pytest.mark.parametrize("N", [8, 16, 40, 64, 72, 128, 200, 256, 512])
@pytest.mark.parametrize("out_dtype", ["f16", "f32"])
def test_cuda_core_plan(cuda, N, out_dtype):
    rng = np.random.default_rng(700 + N)
    c = gen.small(rng, 700, 520, N, 0.08, empty_rows=0.1)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], path="cuda_core")
    dt = torch.float16 if out_dtype == "f16" else torch.float32
    C = torch.full((c["M"], N), 3.0, dtype=dt, device=cuda)
    assert_close(run(plan, B, C), c)


def test_edge_rows(cuda):
    rng = np.random.default_rng(34)
    K, N = 1000, 96
    lengths = [0, 1, 63, 64, 65, 1000, 0, 2, 999, 500, 31, 32, 33, 17, 16] * 9 + [7]
    rp, col, vals = gen.random_csr(rng, len(lengths), K, np.array(lengths), 0.2)
    c = dict(M=len(lengths), K=K, N=N, row_ptr=rp, col=col, vals=vals, B=gen.uniform_b(rng, K, N))
    d = dev(c, cuda)
    for sort_rows in (True, False):
        plan = tca_spmm.Plan(*d[:3], K, path="cuda_core", sort_rows=sort_rows)
        C = torch.zeros((c["M"], N), dtype=torch.float32, device=cuda)
        assert_close(run(plan, d[3], C), c)


def test_short_rows_many_per_item(cuda):
    """Items of up to 31 rows of 0-2 nonzeros (both 16-row groups in use)."""
    rng = np.random.default_rng(35)
    M, K, N = 2000, 300, 64
    lengths = rng.integers(0, 3, size=M)
    rp, col, vals = gen.random_csr(rng, M, K, lengths, 0.5)
    c = dict(M=M, K=K, N=N, row_ptr=rp, col=col, vals=vals, B=gen.uniform_b(rng, K, N))
    d = dev(c, cuda)
    plan = tca_spmm.Plan(*d[:3], K, path="cuda_core")
    for dt in (torch.float16, torch.float32):
        C = torch.zeros((M, N), dtype=dt, device=cuda)
        assert_close(run(plan, d[3], C), c)


def test_alpha_beta_keep_empty(cuda):
    rng = np.random.default_rng(36)
    c = gen.small(rng, 400, 256, 128, 0.05, empty_rows=0.3)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], path="cuda_core")
    C0 = rng.standard_normal((400, 128)).astype(np.float32)
    for keep in (False, True):
        C = torch.from_numpy(C0.copy()).to(cuda)
        run(plan, B, C, alpha=-1.5, beta=0.25, keep_empty_rows=keep)
        assert_close(C, c, keep_empty=keep, C0=C0, alpha=-1.5, beta=0.25)


def test_strided_operands(cuda):
    """B and C as column slices of wider tensors (ldb, ldc > N, 16-byte rows)."""
    rng = np.random.default_rng(37)
    c = gen.small(rng, 500, 384, 72, 0.06, empty_rows=0.05)
    rp, ci, v, B = dev(c, cuda)
    Bw = torch.zeros((c["K"], 136), dtype=torch.float16, device=cuda)
    Bw[:, 8:80] = B
    Cw = torch.full((c["M"], 104), 5.0, dtype=torch.float32, device=cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], path="cuda_core")
    run(plan, Bw[:, 8:80], Cw[:, 16:88])
    assert_close(Cw[:, 16:88], c)
    assert (Cw[:, :16] == 5.0).all() and (Cw[:, 88:] == 5.0).all()


@pytest.mark.parametrize("cfg", ["sweep80", "sweep98"])
def test_mixed_plan_batch(cuda, cfg):
    c = {"sweep80": lambda: gen.sweep(0.80), "sweep98": lambda: gen.sweep(0.98)}[cfg]()
    rp, ci, v, B = dev(c, cuda)
    plans = [tca_spmm.Plan(rp, ci, v, c["K"]) for _ in range(2)]
    outs = [torch.zeros((c["M"], c["N"]), dtype=torch.float16, device=cuda) for _ in range(2)]
    tca_spmm.spmm_batched(plans, [B, B], outs, cc_cols=MMA)
    torch.cuda.synchronize()
    for C in outs:
        assert_close(C, c)
    want = plans[0].spmm(B)
    torch.cuda.synchronize()
    rel = float((outs[0].float() - want.float()).norm() / want.float().norm())
    assert rel <= 1e-3
