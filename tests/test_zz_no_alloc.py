"""tca_spmm_fp8_static, the E4M3 forward that allocates nothing.

It exists for callers that may not allocate device memory themselves -- their
memory belongs to another allocator or budget, or a cudaMalloc / cudaFree
(which may synchronise the device) is not allowed where they call from -- so
it quantizes B into one fixed scratch array that comes with the library.

Checked through the C ABI on two calls in a row with different B, alpha and
beta, since every call reuses the same scratch: against tca_spmm_fp8 (the
allocating entry point) and against the oracle's FP64 product of the
dequantized operands, relative Frobenius difference <= 2e-5 (the bound the
other E4M3 tests use). Between the first call (which looks up the scratch's
address) and the end, neither the library's memory pool (reserved bytes, and
no transient use above the current), torch's caching allocator nor the
device's free memory may change. Also: oversized B and a plan without its
E4M3 form are rejected with a clear error, and K == 0 writes beta * C. This
file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from tca_spmm import gen

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402

TCA_OK, TCA_ERR_INVALID_ARG = 0, 1  # tca_status_t in include/tca_spmm.h


def dev(c, device):
    return (torch.from_numpy(c["row_ptr"]).to(device), torch.from_numpy(c["col"]).to(device),
            torch.from_numpy(c["vals"].copy()).to(device))


def call_static(plan, B, C, alpha=1.0, beta=0.0):
    L = tca_spmm.lib()
    rc = L.tca_spmm_fp8_static(plan.handle, B.data_ptr(), B.stride(0), B.shape[1], C.data_ptr(), C.stride(0),
                               tca_spmm.DTYPE_F32 if C.dtype == torch.float32 else tca_spmm.DTYPE_F16,
                               ctypes.c_float(alpha), ctypes.c_float(beta), 0,
                               torch.cuda.current_stream().cuda_stream)
    return rc


def rel(x, y):
    x, y = x.double().cpu().numpy(), y.double().cpu().numpy()
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


def memory_snapshot():
    torch.cuda.synchronize()
    pool = tca_spmm.pool_stats()
    return {"pool_reserved": pool["reserved"], "pool_used": pool["used"], "pool_high": pool["used_high"],
            "torch_reserved": torch.cuda.memory_reserved(), "device_free": torch.cuda.mem_get_info()[0]}


@pytest.mark.parametrize("case", ["sweep80", "ragged"])
def test_static_matches_allocating_entry_point_twice(cuda, case):
    if case == "sweep80":
        c = gen.sweep(0.80, N=256, seed=7000)
    else:
        c = gen.small(np.random.default_rng(31), 700, 333, 136, 0.08, empty_rows=0.1)
    rp, ci, v = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    plan.quantize_fp8()
    N = c["B"].shape[1]
    rng = np.random.default_rng(5)
    C0 = torch.from_numpy(rng.standard_normal((c["M"], N)).astype(np.float32)).to(cuda)
    calls = []
    for call, (alpha, beta) in enumerate([(1.0, 0.0), (0.5, -1.5)]):
        Bh = (c["B"].astype(np.float32) * (1 + call)).astype(np.float16)
        if call == 1:  # a different B: nothing of the first call's scratch may leak in
            Bh = rng.uniform(-3, 3, (c["K"], N)).astype(np.float16)
        B = torch.from_numpy(Bh).to(cuda)
        want = plan.spmm_fp8(B, out=C0.clone(), alpha=alpha, beta=beta)  # allocating path, before the snapshot
        ref = alpha * oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], Bh) + beta * C0.double().cpu().numpy()
        calls.append((alpha, beta, B, want, ref, C0.clone()))
    # the first static call on this device looks up the scratch's address
    warm = C0.clone()
    assert call_static(plan, calls[0][2], warm) == TCA_OK, tca_spmm.lib().tca_last_error_string()
    tca_spmm.pool_stats(reset_high=True)
    before = memory_snapshot()
    for call, (alpha, beta, B, want, ref, got) in enumerate(calls):
        assert call_static(plan, B, got, alpha, beta) == TCA_OK, tca_spmm.lib().tca_last_error_string()
    after = memory_snapshot()
    assert after == before, (before, after)
    assert after["pool_high"] == after["pool_used"], after  # no transient pool use during the calls
    plan.status()
    for call, (alpha, beta, B, want, ref, got) in enumerate(calls):
        assert rel(got, want) <= 2e-5, (case, call, rel(got, want))
        err = float(np.linalg.norm(got.double().cpu().numpy() - ref) / np.linalg.norm(ref))
        assert err <= 2e-5, (case, call, err)


def test_static_k0_writes_beta_c(cuda):
    L = tca_spmm.lib()
    M, N = 300, 64
    plan = tca_spmm.Plan(torch.zeros(M + 1, dtype=torch.int32, device=cuda),
                         torch.zeros(0, dtype=torch.int32, device=cuda),
                         torch.zeros(0, dtype=torch.float16, device=cuda), 0)
    B = torch.zeros((1, N), dtype=torch.float16, device=cuda)
    C0 = torch.randn((M, N), dtype=torch.float32, device=cuda)
    C = C0.clone()
    assert call_static(plan, B, C, 1.0, 0.25) == TCA_OK, L.tca_last_error_string()
    torch.cuda.synchronize()
    assert torch.equal(C, 0.25 * C0)


def test_static_rejects_what_does_not_fit(cuda):
    L = tca_spmm.lib()
    c = gen.small(np.random.default_rng(2), 256, 128, 64, 0.1)
    rp, ci, v = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    B = torch.from_numpy(c["B"]).to(cuda)
    C = torch.empty((256, 64), dtype=torch.float32, device=cuda)
    # no E4M3 form yet: the entry point may not build it (that allocates)
    assert call_static(plan, B, C) == TCA_ERR_INVALID_ARG
    assert b"tca_plan_quantize_fp8" in L.tca_last_error_string()
    # B beyond the fixed scratch: K = 16384, N = 1024 needs 16 MiB + 4 KiB
    K, N = 16384, 1024
    rng = np.random.default_rng(3)
    cols = np.sort(rng.choice(K, 64, replace=False)).astype(np.int32)
    big = tca_spmm.Plan(torch.tensor([0, 64], dtype=torch.int32, device=cuda), torch.from_numpy(cols).to(cuda),
                        torch.ones(64, dtype=torch.float16, device=cuda), K)
    big.quantize_fp8()
    Bb = torch.zeros((K, N), dtype=torch.float16, device=cuda)
    Cb = torch.empty((1, N), dtype=torch.float32, device=cuda)
    assert call_static(big, Bb, Cb) == TCA_ERR_INVALID_ARG
    assert b"static scratch" in L.tca_last_error_string()
