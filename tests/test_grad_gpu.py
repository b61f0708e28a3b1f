"""Adjoints of Y = A B against FP64 references: the dense-masked gradient
(dA = (dY B^T) on A's pattern, dB = A^T dY in FP64) and central finite
differences of L = sum(Y * dY) evaluated in FP64 on 64 random nonzeros and
64 random B entries. Tolerance: relative error <= 1e-2 (FP32 accumulation of
FP16 inputs; the FD values are exact up to FP64 rounding since L is linear)."""
import numpy as np
import pytest

from tca_spmm import gen

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402
from tca_spmm.autograd import spmm as spmm_ad  # noqa: E402


def dev(x, d):
    return torch.from_numpy(np.ascontiguousarray(x)).to(d)


def f64_grads(c, dY):
    """(dA in CSR order, dB) in FP64."""
    rp, col = c["row_ptr"], c["col"]
    rows = np.repeat(np.arange(c["M"]), np.diff(rp))
    B = c["B"].astype(np.float64)
    Y = dY.astype(np.float64)
    dA = np.einsum("jn,jn->j", Y[rows], B[col])
    dB = np.zeros_like(B)
    np.add.at(dB, col, c["vals"].astype(np.float64)[:, None] * Y[rows])
    return dA, dB


def rel(x, y):
    return float(np.linalg.norm(np.asarray(x, np.float64) - y) / max(np.linalg.norm(y), 1e-300))


@pytest.mark.parametrize("N", [8, 40, 64, 256, 1000])
@pytest.mark.parametrize("path", ["auto", "cuda_core"])
def test_sddmm_and_transpose_small(cuda, N, path):
    rng = np.random.default_rng(N)
    c = gen.small(rng, 300, 190, N, 0.08, empty_rows=0.1)
    dY = rng.standard_normal((300, N)).astype(np.float16)
    plan = tca_spmm.Plan(dev(c["row_ptr"], cuda), dev(c["col"], cuda), dev(c["vals"], cuda), c["K"], path=path)
    dA = plan.sddmm(dev(dY, cuda), dev(c["B"], cuda)).cpu().numpy()
    dB = plan.spmm_t(dev(dY, cuda)).cpu().numpy()
    rA, rB = f64_grads(c, dY)
    assert rel(dA, rA) < 1e-5 and rel(dB, rB) < 1e-5
    np.testing.assert_allclose(dA, rA, rtol=1e-4, atol=1e-4 * np.abs(rA).max())
    plan.status()


@pytest.mark.parametrize("M,K,N,d,path,out", [
    (640, 4096, 256, 0.05, "auto", "f32"),        # 64 direct chunks a window: 8 chunk groups, n cut in parts
    (400, 1024, 96, 0.3, "auto", "f16"),          # FP16 out; N not a multiple of 64 (zero-filled tail)
    (1300, 20000, 64, 0.004, "tensor_core", "f32"),  # condensed chunks (gathered B rows), 11 windows
    (2048, 512, 4096, 0.1, "auto", "f32"),        # the differentiation config's shape
])
def test_sddmm_tensor_core_windows(cuda, M, K, N, d, path, out):
    """The tcgen05 SDDMM over tensor-core windows (and the CUDA-core rows
    beside them) against the FP64 product, elementwise."""
    rng = np.random.default_rng(M + K)
    c = gen.small(rng, M, K, N, d, empty_rows=0.02)
    dY = rng.standard_normal((M, N)).astype(np.float16)
    plan = tca_spmm.Plan(dev(c["row_ptr"], cuda), dev(c["col"], cuda), dev(c["vals"], cuda), c["K"], path=path)
    assert plan.info()["n_tc_windows"] > 0
    dt = torch.float16 if out == "f16" else torch.float32
    dA = plan.sddmm(dev(dY, cuda), dev(c["B"], cuda), out_dtype=dt).float().cpu().numpy()
    dA2 = plan.sddmm(dev(dY, cuda), dev(c["B"], cuda), out_dtype=dt).float().cpu().numpy()
    torch.cuda.synchronize()
    plan.status()
    rA = f64_grads(c, dY)[0]
    # FP32 accumulation over N products of FP16 inputs; FP16 out adds half an ulp
    scale = np.sqrt(N) * np.abs(rA).mean() + np.abs(rA)
    tol = (1e-3 * np.abs(rA) if out == "f16" else 0) + 1e-5 * scale
    assert np.all(np.abs(dA - rA) <= tol), np.abs(dA - rA).max()
    assert np.array_equal(dA, dA2)  # the parts are added in a fixed order


def test_sddmm_unaligned_rows_take_the_cuda_core_kernels(cuda):
    rng = np.random.default_rng(5)
    c = gen.small(rng, 300, 256, 100, 0.2)
    wide = rng.standard_normal((300, 101)).astype(np.float16)
    dY = dev(wide, cuda)[:, :100]  # row stride 101: not 16-byte aligned rows
    plan = tca_spmm.Plan(dev(c["row_ptr"], cuda), dev(c["col"], cuda), dev(c["vals"], cuda), c["K"])
    assert plan.info()["n_tc_windows"] > 0
    dA = plan.sddmm(dY, dev(c["B"], cuda)).cpu().numpy()
    assert rel(dA, f64_grads(c, wide[:, :100])[0]) < 1e-5


def test_transpose_follows_value_updates(cuda):
    rng = np.random.default_rng(7)
    c = gen.small(rng, 200, 150, 64, 0.1)
    dY = rng.standard_normal((200, 64)).astype(np.float16)
    plan = tca_spmm.Plan(dev(c["row_ptr"], cuda), dev(c["col"], cuda), dev(c["vals"], cuda), c["K"])
    plan.spmm_t(dev(dY, cuda))  # builds the transpose with the old values
    c2 = dict(c, vals=(rng.standard_normal(c["col"].size) * 0.5).astype(np.float16))
    plan.update_values(dev(c2["vals"], cuda))
    dB = plan.spmm_t(dev(dY, cuda)).cpu().numpy()
    assert rel(dB, f64_grads(c2, dY)[1]) < 1e-5


def test_differentiation_config_vs_fp64_and_finite_differences(cuda):
    """2048 x 512 at 90% (uniform 51-52 nnz per row), B 512 x 4096, dY 2048 x 4096."""
    c = gen.diff()
    dY = c["dY"]
    rp, col = c["row_ptr"], c["col"]
    plan = tca_spmm.Plan(dev(rp, cuda), dev(col, cuda), dev(c["vals"], cuda), c["K"])
    vals = dev(c["vals"], cuda).float().requires_grad_(True)
    B = dev(c["B"], cuda).float().requires_grad_(True)
    Y = spmm_ad(plan, vals, B)
    (Y * dev(dY, cuda).float()).sum().backward()
    gA, gB = vals.grad.cpu().numpy(), B.grad.cpu().numpy()
    rA, rB = f64_grads(c, dY)
    assert rel(gA, rA) < 1e-2 and rel(gB, rB) < 1e-2
    # central finite differences of L = sum(Y * dY) in FP64 (only the touched row /
    # column of Y changes, so L is evaluated on that row / column)
    rng = np.random.default_rng(11)
    v64, B64, Y64 = c["vals"].astype(np.float64), c["B"].astype(np.float64), dY.astype(np.float64)
    rows = np.repeat(np.arange(c["M"]), np.diff(rp))
    h = 1e-3

    def L_row(r, v):
        j0, j1 = rp[r], rp[r + 1]
        return float((v[j0:j1] @ B64[col[j0:j1]]) @ Y64[r])

    def L_col(n, Bm):
        y = np.zeros(c["M"])
        np.add.at(y, rows, v64 * Bm[col, n])
        return float(y @ Y64[:, n])

    for j in rng.choice(col.size, 64, replace=False):
        vp, vm = v64.copy(), v64.copy()
        vp[j] += h
        vm[j] -= h
        fd = (L_row(rows[j], vp) - L_row(rows[j], vm)) / (2 * h)
        assert abs(gA[j] - fd) <= 1e-2 * max(abs(fd), np.abs(rA).mean())
    for k, n in zip(rng.integers(0, c["K"], 64), rng.integers(0, c["N"], 64)):
        Bp, Bm = B64.copy(), B64.copy()
        Bp[k, n] += h
        Bm[k, n] -= h
        fd = (L_col(n, Bp) - L_col(n, Bm)) / (2 * h)
        assert abs(gB[k, n] - fd) <= 1e-2 * max(abs(fd), np.abs(rB).mean())
    plan.status()


def test_autograd_matches_torch_dense(cuda):
    rng = np.random.default_rng(21)
    c = gen.small(rng, 160, 96, 48, 0.2)
    plan = tca_spmm.Plan(dev(c["row_ptr"], cuda), dev(c["col"], cuda), dev(c["vals"], cuda), c["K"])
    vals = dev(c["vals"], cuda).float().requires_grad_(True)
    B = dev(c["B"], cuda).float().requires_grad_(True)
    Y = spmm_ad(plan, vals, B)
    W = torch.randn_like(Y)
    (Y * W).sum().backward()
    rows = np.repeat(np.arange(c["M"]), np.diff(c["row_ptr"]))
    A = torch.zeros((c["M"], c["K"]), dtype=torch.float64)
    v64 = torch.from_numpy(c["vals"].astype(np.float64)).requires_grad_(True)
    A = A.index_put((torch.from_numpy(rows), torch.from_numpy(c["col"].astype(np.int64))), v64)
    B64 = torch.from_numpy(c["B"].astype(np.float64)).requires_grad_(True)
    Yr = A @ B64
    (Yr * W.cpu().double()).sum().backward()
    assert torch.allclose(Y.detach().cpu().double(), Yr.detach(), rtol=1e-3, atol=1e-3)
    assert rel(vals.grad.cpu().numpy(), v64.grad.numpy()) < 2e-3
    assert rel(B.grad.cpu().numpy(), B64.grad.numpy()) < 2e-3
