"""GPU parity of the forward paths against the oracle (FP64 CSR x dense on the
CPU), and of the GPU-built tile format against the host build, bit for bit.

Tolerances (written per element, C64 the FP64 oracle, S = |A| x |B| the FP64
product of absolute values, i.e. the scale of the FP32 rounding error):
  FP32 output: |C - C64| <= 1e-5 * S
  FP16 output: |C - C64| <= 1e-3 * |C64| + 1e-5 * S + 2**-24
"""
import pathlib

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


def assert_close(C, c, keep_empty=False, C0=None, alpha=1.0, beta=0.0):
    got = C.float().cpu().numpy().astype(np.float64)
    ref = oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
    S = oracle.spmm_f64(c["row_ptr"], c["col"], np.abs(c["vals"].astype(np.float32)).astype(np.float16),
                        np.abs(c["B"].astype(np.float32)).astype(np.float16))
    if C0 is not None:
        c0 = C0.astype(np.float64)
        ref = alpha * ref + beta * c0
        S = abs(alpha) * S + abs(beta) * np.abs(c0)
    else:
        ref = alpha * ref
        S = abs(alpha) * S
    if keep_empty:
        empty = np.diff(c["row_ptr"]) == 0
        ref[empty] = C0[empty] if C0 is not None else 0.0
    if C.dtype == torch.float32:
        tol = 1e-5 * S + 1e-30
    else:
        tol = 1e-3 * np.abs(ref) + 1e-5 * S + 2.0 ** -24
    err = np.abs(got - ref)
    bad = err > tol
    assert not bad.any(), f"{bad.sum()} of {bad.size} elements off; worst {err.max():.3e}"
    return float(np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300))


# ------------------------------------------------------------------ plan-free
@pytest.mark.parametrize("N", [8, 16, 40, 64, 72, 128, 256, 320, 512])
@pytest.mark.parametrize("out_dtype", ["f16", "f32"])
def test_csr_cuda_core(cuda, N, out_dtype):
    rng = np.random.default_rng(N)
    c = gen.small(rng, 333, 257, N, 0.06, empty_rows=0.1)
    rp, ci, v, B = dev(c, cuda)
    dt = torch.float16 if out_dtype == "f16" else torch.float32
    C = tca_spmm.spmm_csr(rp, ci, v, B, out_dtype=dt)
    torch.cuda.synchronize()
    assert_close(C, c)


def test_csr_scalar_path_any_n_and_ld(cuda):
    rng = np.random.default_rng(11)
    c = gen.small(rng, 100, 90, 13, 0.2)
    rp, ci, v, _ = dev(c, cuda)
    wide = torch.zeros((90, 16), dtype=torch.float16, device=cuda)
    wide[:, :13] = torch.from_numpy(c["B"]).to(cuda)
    B = wide[:, :13]  # ldb = 16, N = 13
    C = tca_spmm.spmm_csr(rp, ci, v, B, out_dtype=torch.float32)
    assert_close(C, c)


def test_csr_alpha_beta_keep_empty(cuda):
    rng = np.random.default_rng(12)
    c = gen.small(rng, 200, 100, 64, 0.05, empty_rows=0.3)
    rp, ci, v, B = dev(c, cuda)
    C0 = rng.standard_normal((200, 64)).astype(np.float32)
    C = torch.from_numpy(C0.copy()).to(cuda)
    tca_spmm.spmm_csr(rp, ci, v, B, out=C, alpha=0.5, beta=2.0, keep_empty_rows=True)
    assert_close(C, c, keep_empty=True, C0=C0, alpha=0.5, beta=2.0)


# ------------------------------------------------------------------ plans
PLAN_KEYS = {
    "perm": tca_spmm.ARR_ROW_PERM, "p_row_ptr": tca_spmm.ARR_P_ROW_PTR, "p_col": tca_spmm.ARR_P_COL,
    "p_val": tca_spmm.ARR_P_VAL, "src": tca_spmm.ARR_SRC, "tc_windows": tca_spmm.ARR_TC_WINDOWS,
    "cc_windows": tca_spmm.ARR_CC_WINDOWS, "tile_first": tca_spmm.ARR_TILE_FIRST,
    "win_cols": tca_spmm.ARR_WIN_COLS, "tile_ptr": tca_spmm.ARR_TILE_PTR,
    "tile_entries": tca_spmm.ARR_TILE_ENTRIES, "tile_src": tca_spmm.ARR_TILE_SRC,
    "tile_image_idx": tca_spmm.ARR_TILE_IMAGE_IDX, "tile_images": tca_spmm.ARR_TILE_IMAGES,
    "cc_items": tca_spmm.ARR_CC_ITEMS, "all_items": tca_spmm.ARR_ALL_ITEMS, "tc_pairs": tca_spmm.ARR_TC_PAIRS,
}


def plan_cases():
    rng = np.random.default_rng(5)
    yield "ragged", gen.small(rng, 1000, 700, 64, 0.04, empty_rows=0.15)
    yield "cfg1", gen.cfg1()
    yield "zipf95", gen.sweep(0.95, N=64, M=1024, K=1024)
    yield "zipf70", gen.sweep(0.70, N=64, M=512, K=1024)  # dense chunks -> tile images


@pytest.mark.parametrize("path", [0, 1, 2])
@pytest.mark.parametrize("sort_rows", [True, False])
def test_plan_bitexact_vs_host_build(cuda, path, sort_rows):
    for name, c in plan_cases():
        rp, ci, v, _ = dev(c, cuda)
        plan = tca_spmm.Plan(rp, ci, v, c["K"], sort_rows=sort_rows, path=list(tca_spmm.PATHS)[path])
        host = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], c["K"], sort_rows=sort_rows, path=path)
        info = plan.info()
        assert info["n_tc_windows"] == host["n_tc"] and info["n_cc_windows"] == host["n_cc"], name
        assert info["n_tc_chunks"] == host["n_tc_chunks"] and info["tc_nnz"] == host["tc_nnz"], name
        assert info["n_images"] == host["n_images"], name
        for key, which in PLAN_KEYS.items():
            got = plan.export(which)
            assert np.array_equal(got, host[key]), f"{name}: {key} differs"


@pytest.mark.parametrize("M", [8191, 8192, 8193, 20000])
@pytest.mark.parametrize("sort_rows", [True, False])
def test_plan_row_order_both_builders(cuda, M, sort_rows):
    """Up to 8192 rows the row order (sort, offsets, flags) is built by one
    block; above, by device-wide sort and scan passes. Both against the host
    build, bit for bit, with row lengths from 0 to 700 (ties everywhere)."""
    rng = np.random.default_rng(M)
    c = gen.small(rng, M, 700, 16, 0.03, empty_rows=0.1)
    rp, ci, v, _ = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], sort_rows=sort_rows)
    host = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], c["K"], sort_rows=sort_rows, path=0)
    assert plan.info()["n_tc_windows"] == host["n_tc"]
    for key, which in PLAN_KEYS.items():
        assert np.array_equal(plan.export(which), host[key]), key


@pytest.mark.parametrize("path", ["auto", "tensor_core", "cuda_core"])
@pytest.mark.parametrize("N", [16, 64, 128, 200, 256, 512])
@pytest.mark.parametrize("out_dtype", ["f16", "f32"])
def test_plan_forward_paths(cuda, path, N, out_dtype):
    rng = np.random.default_rng(100 + N)
    c = gen.small(rng, 700, 520, N, 0.08, empty_rows=0.1)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], path=path)
    if path == "tensor_core":
        assert plan.info()["n_tc_windows"] > 0
    dt = torch.float16 if out_dtype == "f16" else torch.float32
    C = plan.spmm(B, out_dtype=dt)
    torch.cuda.synchronize()
    plan.status()
    assert_close(C, c)


def test_plan_alpha_beta_keep_empty_tc(cuda):
    rng = np.random.default_rng(21)
    c = gen.small(rng, 300, 256, 128, 0.1, empty_rows=0.25)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], path="tensor_core")
    C0 = rng.standard_normal((300, 128)).astype(np.float32)
    C = torch.from_numpy(C0.copy()).to(cuda)
    plan.spmm(B, out=C, alpha=-1.5, beta=0.25, keep_empty_rows=True)
    assert_close(C, c, keep_empty=True, C0=C0, alpha=-1.5, beta=0.25)


def test_edge_rows(cuda):
    """Rows with 0, 1, 63, 64, 65, 1000 nonzeros; K not a multiple of 8; a
    partial last window."""
    rng = np.random.default_rng(33)
    K, N = 1000, 96
    lengths = [0, 1, 63, 64, 65, 1000, 0, 2, 999, 500] * 13 + [7]
    row_nnz = np.array(lengths)
    rp, col, vals = gen.random_csr(rng, len(lengths), K, row_nnz, 0.2)
    c = dict(M=len(lengths), K=K, N=N, row_ptr=rp, col=col, vals=vals, B=gen.uniform_b(rng, K, N))
    d = dev(c, cuda)
    for path in ("auto", "tensor_core", "cuda_core"):
        plan = tca_spmm.Plan(*d[:3], K, path=path)
        assert_close(plan.spmm(d[3], out_dtype=torch.float32), c)
    assert_close(tca_spmm.spmm_csr(*d, out_dtype=torch.float32), c)


def test_unaligned_operands_fall_back_to_cuda_cores(cuda):
    rng = np.random.default_rng(34)
    c = gen.small(rng, 260, 300, 24, 0.2)
    rp, ci, v, _ = dev(c, cuda)
    wide = torch.zeros((300, 27), dtype=torch.float16, device=cuda)
    wide[:, :24] = torch.from_numpy(c["B"]).to(cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], path="tensor_core")
    assert_close(plan.spmm(wide[:, :24], out_dtype=torch.float32), c)


@pytest.mark.parametrize("density", [0.1, 0.7])
def test_update_values(cuda, density):
    rng = np.random.default_rng(35)
    c = gen.small(rng, 400, 300, 64, density)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    c2 = dict(c, vals=(rng.standard_normal(c["col"].size) * 0.3).astype(np.float16))
    plan.update_values(torch.from_numpy(c2["vals"]).to(cuda))
    assert_close(plan.spmm(B, out_dtype=torch.float32), c2)
    host = oracle.build_plan(c2["row_ptr"], c2["col"], c2["vals"], c2["K"])
    assert np.array_equal(plan.export(tca_spmm.ARR_TILE_ENTRIES), host["tile_entries"])
    assert np.array_equal(plan.export(tca_spmm.ARR_TILE_IMAGES), host["tile_images"])
    if density > 0.5:
        assert plan.info()["n_images"] > 0


@pytest.mark.parametrize("out_dtype", ["f16", "f32"])
def test_batched_matches_per_plan(cuda, out_dtype):
    """Layers of different shapes, sparsities and N in one batched call give
    the oracle's results (tensor-core and CUDA-core parts, several N-slice
    widths, more items than one launch carries)."""
    dt = torch.float16 if out_dtype == "f16" else torch.float32
    rng = np.random.default_rng(50)
    cases, plans, Bs, Cs = [], [], [], []
    for i in range(40):
        M, K = [(300, 200), (130, 520), (64, 64), (512, 256)][i % 4]
        N = [16, 64, 96, 128, 256, 512][i % 6]
        c = gen.small(rng, M, K, N, [0.02, 0.1, 0.4, 0.8][i % 4], empty_rows=0.1)
        rp, ci, v, B = dev(c, cuda)
        cases.append(c)
        plans.append(tca_spmm.Plan(rp, ci, v, K))
        Bs.append(B)
        Cs.append(torch.empty((M, N), dtype=dt, device=cuda))
    tca_spmm.spmm_batched(plans, Bs, Cs)
    torch.cuda.synchronize()
    for c, C, p in zip(cases, Cs, plans):
        p.status()
        assert_close(C, c)


def test_malformed_csr_is_rejected(cuda):
    rp = torch.tensor([0, 2, 1], dtype=torch.int32, device=cuda)
    ci = torch.tensor([0, 1], dtype=torch.int32, device=cuda)
    v = torch.ones(2, dtype=torch.float16, device=cuda)
    with pytest.raises(tca_spmm.TcaError, match="FORMAT"):
        tca_spmm.Plan(rp, ci, v, 4)
    rp = torch.tensor([0, 2], dtype=torch.int32, device=cuda)
    ci = torch.tensor([0, 7], dtype=torch.int32, device=cuda)
    with pytest.raises(tca_spmm.TcaError, match="FORMAT"):
        tca_spmm.Plan(rp, ci, v, 4)


# ------------------------------------------------------------------ full sizes
@pytest.mark.parametrize("cfg", ["cfg1", "sweep80", "sweep95", "sweep98", "sweep70_512", "sweep90_64",
                                 "sweep80_128", "sweep95_128"])
def test_full_size_configs(cuda, cfg):
    if cfg == "cfg1":
        c = gen.cfg1()
    else:
        s, _, n = cfg[5:].partition("_")
        c = gen.sweep(int(s) / 100, N=int(n) if n else 256)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    C = plan.spmm(B, out_dtype=torch.float16)
    rel = assert_close(C, c)
    assert rel < 1e-2
    plan.status()


@pytest.mark.parametrize("M,K,N,d", [(256, 8192, 64, 0.3), (1000, 4096, 136, 0.2), (300, 2048, 512, 0.5)])
def test_long_windows(cuda, M, K, N, d):
    """Few windows with many chunks each (long items on few CTAs, wide K,
    N beyond one slice): FP32 and FP16 outputs within the tolerances above,
    E4M3 within 2e-5 of the FP64 product of its dequantized operands, and two
    launches identical bit for bit."""
    c = gen.small(np.random.default_rng(M + K), M, K, N, d, empty_rows=0.05)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    assert plan.info()["n_tc_windows"] > 0
    C1 = plan.spmm(B, out_dtype=torch.float32)
    C2 = plan.spmm(B, out_dtype=torch.float32)
    torch.cuda.synchronize()
    plan.status()
    assert torch.equal(C1, C2)
    assert_close(C1, c)
    assert_close(plan.spmm(B, out_dtype=torch.float16), c)
    C8 = plan.spmm_fp8(B, out_dtype=torch.float32).double().cpu().numpy()
    ref8 = oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
    assert np.linalg.norm(C8 - ref8) <= 2e-5 * np.linalg.norm(ref8)
    plan.status()


def test_host_api_reference_semantics(cuda):
    rng = np.random.default_rng(40)
    c = gen.small(rng, 500, 256, 64, 0.05, empty_rows=0.3)
    C0 = rng.standard_normal((500, 64)).astype(np.float32)
    out, ms = tca_spmm.spmm_host(c["row_ptr"], c["col"], c["vals"], c["K"], c["B"], C=C0.copy(), n_iter=3)
    assert ms > 0
    assert_close(torch.from_numpy(out), c, keep_empty=True, C0=C0)


# ------------------------------------------------------------------ reference kernels
def fixture_case():
    """The reference's own data fixture (pattern only: every value 1.0), with
    B as its harness makes it (src/test.cu:56: nonzero with probability 0.9,
    value U(0, 1)), seeded, N = 256."""
    path = pathlib.Path(__file__).resolve().parent / "golden" / "body_decoder_layer_2_ffn_conv1.smtx"
    M, K, nnz, rp, ci = oracle.smtx_parse(path.read_bytes())
    rng = np.random.default_rng(56)
    B = np.where(rng.random((K, 256)) > 0.1, rng.random((K, 256)), 0.0).astype(np.float16)
    return {"M": M, "K": K, "row_ptr": rp, "col": ci, "vals": np.ones(nnz, np.float16), "B": B}


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("cfg", ["cfg1", "sweep80", "sweep95", "sweep98", "fixture"])
def test_matches_reference_tca_and_cusparse(cuda, cfg):
    """Our forward vs the reference's own our_spmm_balanced and its cuSPARSE
    comparator on the same inputs: within 1e-2 relative (compare_mat rule and
    relative Frobenius)."""
    if cfg == "fixture":
        c = fixture_case()
    else:
        c = gen.cfg1() if cfg == "cfg1" else gen.sweep(int(cfg[5:]) / 100, N=256)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    ours = plan.spmm(B, out_dtype=torch.float32).cpu().numpy()
    with oracle.quiet_stdout():
        ref_tca, _ = oracle.ref_our_spmm_balanced(c["row_ptr"], c["col"], c["vals"], c["K"], c["B"])
        A = oracle.csr_to_dense(c["M"], c["K"], c["row_ptr"], c["col"], c["vals"])
        ref_sp, _ = oracle.ref_cusparse_spmm(A, c["B"])
    c64 = oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], c["B"])

    def rel(x, y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    # cuSPARSE agrees with the FP64 oracle, and so must we
    assert rel(ref_sp, c64) < 1e-3
    assert rel(ours, ref_sp) < 1e-2 and oracle.compare_mat(ref_sp, ours, 1e-2) == 0
    # The reference TCA kernel: where it is itself within 1e-2 of the FP64
    # product we must match it to 1e-2; where it is not (its long-row path,
    # rows > 64 nnz, src/our_spmm.cu:197-258, reuses its shared B and A
    # staging across nnz chunks without a barrier after the MMAs read them),
    # we must be strictly closer to the FP64 product than it is.
    ref_err, our_err = rel(ref_tca, c64), rel(ours, c64)
    short = np.diff(c["row_ptr"]) <= 64  # rows the reference handles in multirow_per_tb
    bad_short = oracle.compare_mat(ref_tca[short], ours[short], 1e-2)
    bad_long = oracle.compare_mat(ref_tca[~short], ours[~short], 1e-2)
    print(f"{cfg}: reference TCA rel err {ref_err:.3e} (compare_mat flags: rows<=64 nnz {bad_short}, "
          f"rows>64 nnz {bad_long}), ours {our_err:.3e}, cuSPARSE {rel(ref_sp, c64):.3e}")
    assert bad_short == 0  # its short-row path agrees with ours element by element
    if ref_err < 1e-2:
        assert rel(ours, ref_tca) < 1e-2
    assert our_err < ref_err or our_err < 1e-6


@pytest.mark.parametrize("precision", ["f16", "e4m3"])
def test_batch_of_32_full_size_problems(cuda, precision):
    """32 sweep problems in one launch (352 tensor-core items on 148
    persistent CTAs, a third round on 56 of them): the problems of every
    round against FP64 (E4M3: against the FP64 product of its own quantized
    operands)."""
    distinct = [gen.sweep(0.8, N=256, seed=7200 + i) for i in range(4)]
    plans, Bs, Cs = [], [], []
    for g in range(32):
        c = distinct[g % 4]
        rp, ci, v, B = dev(c, cuda)
        plans.append(tca_spmm.Plan(rp, ci, v, c["K"]))
        Bs.append(B)
        Cs.append(torch.empty((c["M"], 256), dtype=torch.float32, device=cuda))
    if precision == "f16":
        tca_spmm.spmm_batched(plans, Bs, Cs)
    else:
        tca_spmm.spmm_fp8_batched(plans, Bs, Cs)
    torch.cuda.synchronize()
    for p in plans:
        p.status()
    if precision == "f16":
        for g in (0, 27, 29, 30, 31):
            assert_close(Cs[g], distinct[g % 4])
    else:
        refs = [oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"]) for c in distinct]
        for g in range(32):
            got = Cs[g].double().cpu().numpy()
            ref = refs[g % 4]
            assert np.linalg.norm(got - ref) <= 2e-5 * np.linalg.norm(ref), g
