"""The FP8-E4M3 forward against the oracle.

Bit-exact: the quantized operands (per-row scales and E4M3 values of A in
every form the kernels read -- sorted values, tile entries, swizzled tile
images -- and per-column B) against oracle.quant_rows / quant_cols.

Forward: against the FP64 product of the dequantized operands
(oracle.spmm_fp8_f64). The products q_a q_b are exact in FP32, so the only
differences are FP32 accumulation and the final scaling: relative Frobenius
error <= 2e-5 with FP32 output, <= 1e-3 with FP16 output.

Precision config (4096 x 4096, 90 %, N = 1024): relative Frobenius error of
the E4M3 forward against the FP64 product of the original FP16 operands,
reported next to the FP16 forward's. E4M3 keeps 3 mantissa bits, so per-row /
per-column scaling leaves ~3.7e-2 (the quantization error of both operands);
the test bounds it by 5e-2 and the FP16 forward by 1e-3.
"""
import numpy as np
import pytest

from oracle import oracle
from tca_spmm import gen

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402


def dev(c, device):
    return (torch.from_numpy(c["row_ptr"]).to(device), torch.from_numpy(c["col"]).to(device),
            torch.from_numpy(c["vals"].copy()).to(device), torch.from_numpy(c["B"].copy()).to(device))


def rel(x, y):
    x = np.asarray(x, np.float64)
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


def swz64(r, c):
    return r * 64 + (((c >> 4) ^ ((r >> 1) & 3)) << 4) + (c & 15)


CASES = {
    "ragged": lambda: gen.small(np.random.default_rng(1), 700, 333, 256, 0.08, empty_rows=0.1),
    "cfg1": lambda: gen.cfg1(),
    "zipf95": lambda: gen.sweep(0.95, N=256, seed=11),
}


@pytest.mark.parametrize("case", list(CASES))
def test_quantized_operands_bit_exact(cuda, case):
    c = CASES[case]()
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    plan.quantize_fp8()
    torch.cuda.synchronize()
    prp = plan.export(tca_spmm.ARR_P_ROW_PTR)
    pval = plan.export(tca_spmm.ARR_P_VAL).view(np.float16)
    sa, qa = oracle.quant_rows(prp, pval)
    np.testing.assert_array_equal(plan.export(tca_spmm.ARR_ROW_SCALE).view(np.uint32), sa.view(np.uint32))
    np.testing.assert_array_equal(plan.export(tca_spmm.ARR_P_VAL_F8), qa)
    ent = plan.export(tca_spmm.ARR_TILE_ENTRIES)
    src = plan.export(tca_spmm.ARR_TILE_SRC)
    ent8 = plan.export(tca_spmm.ARR_TILE_ENTRIES_F8)
    np.testing.assert_array_equal(ent8, (ent & 0xFFFF0000) | qa[src].astype(np.uint32))
    # images: dense 128 x 64 E4M3 tiles in the 64-byte swizzled K-major layout
    img_idx = plan.export(tca_spmm.ARR_TILE_IMAGE_IDX)
    tptr = plan.export(tca_spmm.ARR_TILE_PTR)
    imgs = plan.export(tca_spmm.ARR_TILE_IMAGES_F8).reshape(-1, 8192) if img_idx.size else np.zeros((0, 8192))
    want = np.zeros_like(imgs)
    for chunk in np.nonzero(img_idx >= 0)[0]:
        e = ent8[tptr[chunk]:tptr[chunk + 1]].astype(np.int64)
        want[img_idx[chunk], swz64(e >> 22, (e >> 16) & 63)] = e & 0xFF
    np.testing.assert_array_equal(imgs, want)
    # B per column
    Bq, sb = tca_spmm.quantize_b_fp8(B)
    qb, sb_ref = oracle.quant_cols(c["B"], ldq=Bq.shape[1])
    np.testing.assert_array_equal(sb.cpu().numpy().view(np.uint32), sb_ref.view(np.uint32))
    np.testing.assert_array_equal(Bq.cpu().numpy()[:, :c["B"].shape[1]], qb[:, :c["B"].shape[1]])


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("path", ["auto", "cuda_core", "tensor_core"])
@pytest.mark.parametrize("N", [64, 128, 256, 320])
@pytest.mark.parametrize("out_dtype", ["f16", "f32"])
def test_fp8_forward_vs_dequantized_f64(cuda, case, path, N, out_dtype):
    c = CASES[case]()
    c["B"] = np.ascontiguousarray(c["B"][:, :N]) if c["B"].shape[1] >= N else \
        np.random.default_rng(N).uniform(-1, 1, (c["K"], N)).astype(np.float16)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], path=path)
    dt = torch.float16 if out_dtype == "f16" else torch.float32
    C = plan.spmm_fp8(B, out_dtype=dt)
    torch.cuda.synchronize()
    plan.status()
    ref = oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
    err = rel(C.float().cpu().numpy(), ref)
    assert err <= (2e-5 if out_dtype == "f32" else 1e-3), err


@pytest.mark.parametrize("K,N", [(300, 2048), (257, 2047), (64, 9472), (1024, 1184), (2000, 1300), (8192, 1200)])
def test_b_quantization_one_launch_bit_exact(cuda, K, N):
    """Wide B (enough column strips for the one-launch quantization, several
    strip widths, a ragged last strip; strips held in shared memory, and --
    K = 8192 -- strips too tall for it, read twice) against the oracle, bit
    for bit."""
    rng = np.random.default_rng(K + N)
    B = (rng.standard_normal((K, N)) * rng.choice([1e-3, 1.0, 50.0], N)).astype(np.float16)
    B[:, 3] = 0  # an all-zero column: scale 1
    Bq, sb = tca_spmm.quantize_b_fp8(torch.from_numpy(B).to(cuda))
    qb, sb_ref = oracle.quant_cols(B, ldq=Bq.shape[1])
    np.testing.assert_array_equal(sb.cpu().numpy().view(np.uint32), sb_ref.view(np.uint32))
    np.testing.assert_array_equal(Bq.cpu().numpy()[:, :N], qb[:, :N])


def test_fp8_alpha_beta_and_empty_rows(cuda):
    c = gen.small(np.random.default_rng(3), 500, 300, 64, 0.1, empty_rows=0.2)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    C0 = np.random.default_rng(4).standard_normal((500, 64)).astype(np.float32)
    C = torch.from_numpy(C0.copy()).to(cuda)
    plan.spmm_fp8(B, out=C, alpha=0.5, beta=-2.0, keep_empty_rows=True)
    torch.cuda.synchronize()
    ref = 0.5 * oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"]) - 2.0 * C0
    empty = np.diff(c["row_ptr"]) == 0
    ref[empty] = C0[empty]
    got = C.cpu().numpy()
    assert rel(got, ref) <= 2e-5
    np.testing.assert_array_equal(got[empty], C0[empty])


def test_fp8_follows_value_updates(cuda):
    rng = np.random.default_rng(9)
    c = gen.small(rng, 400, 256, 128, 0.2)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    plan.spmm_fp8(B)
    c2 = dict(c, vals=(rng.standard_normal(c["col"].size) * 0.3).astype(np.float16))
    plan.update_values(torch.from_numpy(c2["vals"]).to(cuda))
    C = plan.spmm_fp8(B, out_dtype=torch.float32)
    torch.cuda.synchronize()
    assert rel(C.cpu().numpy(), oracle.spmm_fp8_f64(c2["row_ptr"], c2["col"], c2["vals"], c2["B"])) <= 2e-5


def test_fp8_batched_matches_single(cuda):
    plans, Bs, outs, cs = [], [], [], []
    for i, (M, K, N, d) in enumerate([(300, 200, 64, 0.1), (1024, 512, 256, 0.3), (257, 129, 128, 0.05),
                                      (2048, 512, 256, 0.2)]):
        c = gen.small(np.random.default_rng(100 + i), M, K, N, d, empty_rows=0.05)
        rp, ci, v, B = dev(c, cuda)
        plans.append(tca_spmm.Plan(rp, ci, v, K))
        Bs.append(B)
        outs.append(torch.empty((M, N), dtype=torch.float32, device=cuda))
        cs.append(c)
    tca_spmm.spmm_fp8_batched(plans, Bs, outs)
    torch.cuda.synchronize()
    for p, B, C, c in zip(plans, Bs, outs, cs):
        single = p.spmm_fp8(B, out_dtype=torch.float32)
        torch.cuda.synchronize()
        ref = oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
        assert rel(C.cpu().numpy(), ref) <= 2e-5
        assert rel(single.cpu().numpy(), ref) <= 2e-5


def test_fp8_rejects_what_it_cannot_run(cuda):
    c = gen.small(np.random.default_rng(5), 100, 64, 12, 0.1)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    with pytest.raises(tca_spmm.TcaError):
        plan.spmm_fp8(B)  # N % 8 != 0
    c = gen.small(np.random.default_rng(6), 100, 64, 16, 0.1)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    out = torch.empty((100, 16), dtype=torch.float16, device=cuda)
    with pytest.raises(tca_spmm.TcaError):
        tca_spmm.spmm_fp8_batched([plan, plan], [B, B], [out, out])  # one plan twice


def test_precision_config_error_report(cuda, capsys):
    c = gen.precision()
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    C8 = plan.spmm_fp8(B, out_dtype=torch.float16)
    C16 = plan.spmm(B, out_dtype=torch.float16)
    torch.cuda.synchronize()
    plan.status()
    ref = oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
    e8 = rel(C8.float().cpu().numpy(), ref)
    e16 = rel(C16.float().cpu().numpy(), ref)
    e8q = rel(C8.float().cpu().numpy(), oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"]))
    with capsys.disabled():
        print(f"\nprecision config: rel. Frobenius error vs FP64 -- E4M3 {e8:.3e}, FP16 {e16:.3e}; "
              f"E4M3 forward vs its own dequantized operands {e8q:.3e}")
    assert e16 <= 1e-3
    assert e8 <= 5e-2
    assert e8q <= 1e-3
