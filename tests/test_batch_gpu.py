"""Batching: 24 layers of mixed shapes, sparsity and N (gen.batch_layers) as
one batch -- eager, captured in a CUDA graph and replayed, autotuned -- each
layer against the FP64 oracle (relative Frobenius error <= 1e-3 with FP16
output; E4M3 against its dequantized operands, <= 1e-3)."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle
from tca_spmm import gen

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402


def f64(c):
    A = sp.csr_matrix((c["vals"].astype(np.float64), c["col"], c["row_ptr"]), shape=(c["M"], c["K"]))
    return np.asarray(A @ c["B"].astype(np.float64))


def rel(x, y):
    return float(np.linalg.norm(np.asarray(x, np.float64) - y) / max(np.linalg.norm(y), 1e-300))


@pytest.fixture(scope="module")
def layers(cuda):
    ls = gen.batch_layers()
    plans, Bs, outs = [], [], []
    for c in ls:
        rp, ci, v = (torch.from_numpy(x.copy()).to(cuda) for x in (c["row_ptr"], c["col"], c["vals"]))
        plans.append(tca_spmm.Plan(rp, ci, v, c["K"]))
        Bs.append(torch.from_numpy(c["B"].copy()).to(cuda))
        outs.append(torch.zeros((c["M"], c["N"]), dtype=torch.float16, device=cuda))
    return ls, plans, Bs, outs


def check(ls, outs, ref_fn=f64, tol=1e-3):
    for c, C in zip(ls, outs):
        err = rel(C.float().cpu().numpy(), ref_fn(c))
        assert err <= tol, (c["name"], c["M"], c["K"], c["N"], err)


def test_eager_batch(layers):
    ls, plans, Bs, outs = layers
    for C in outs:
        C.zero_()
    tca_spmm.spmm_batched(plans, Bs, outs)
    torch.cuda.synchronize()
    check(ls, outs)


def test_graph_replay(layers):
    ls, plans, Bs, outs = layers
    g = tca_spmm.BatchGraph(plans, Bs, outs)
    for C in outs:
        C.fill_(7.0)
    torch.cuda.synchronize()
    g.launch()
    g.launch()
    torch.cuda.synchronize()
    check(ls, outs)
    # new B values are picked up by a replay (the graph holds pointers, not data)
    Bs[0].mul_(-1)
    g.launch()
    torch.cuda.synchronize()
    neg = dict(ls[0], B=(-ls[0]["B"].astype(np.float32)).astype(np.float16))
    assert rel(outs[0].float().cpu().numpy(), f64(neg)) <= 1e-3
    Bs[0].mul_(-1)
    g.close()


def test_autotuned_graph(layers):
    ls, plans, Bs, outs = layers
    tuned = tca_spmm.autotune(plans, Bs, outs, reps=3)
    assert len(tuned) == len(plans)
    for (nt, w), c in zip(tuned, ls):
        assert nt in (64, 128, 256) and w in (2, 4, 8, tca_spmm.CC_COLS_MMA)
    g = tca_spmm.BatchGraph(plans, Bs, outs, n_tiles=[t[0] for t in tuned], cc_cols=[t[1] for t in tuned])
    for C in outs:
        C.zero_()
    g.launch()
    torch.cuda.synchronize()
    check(ls, outs)
    g.close()


def test_fp8_graph(layers):
    ls, plans, Bs, outs = layers
    g = tca_spmm.BatchGraph(plans, Bs, outs, precision="e4m3")
    for C in outs:
        C.zero_()
    g.launch()
    torch.cuda.synchronize()
    check(ls, outs, ref_fn=lambda c: oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"]))
    g.close()
