"""The oracle against the golden fixtures made by the reference's own CPU
functions (tests/golden/make_golden.py), and against the reference tree
itself when it is present."""
import pathlib

import numpy as np
import pytest

from conftest import REFERENCE_TREE, ROOT
from oracle import oracle

GOLD_DIR = ROOT / "tests" / "golden"


def test_half_conversions_match_ieee():
    L = oracle.lib()
    allh = np.arange(65536, dtype=np.uint32).astype(np.uint16)
    f_np = allh.view(np.float16).astype(np.float32)
    f_or = np.array([L.orc_h2f(int(h)) for h in allh[::7]], np.float32)
    ref = f_np[::7]
    same = (f_or == ref) | (np.isnan(f_or) & np.isnan(ref))
    assert same.all()
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.standard_normal(4000).astype(np.float32) * 10 ** rng.uniform(-9, 5, 4000).astype(np.float32),
                         np.array([65504, 65519.99, 65520, 6.1e-5, 5.96e-8, 2.98e-8, 2.99e-8, -0.0], np.float32)])
    got = np.array([L.orc_f2h(float(x)) for x in xs], np.uint16)
    want = xs.astype(np.float16).view(np.uint16)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("i", [0, 1, 2])
def test_smtx_parse_matches_reference(golden, i):
    text = (GOLD_DIR / f"smtx_{i}.smtx").read_bytes()
    M, K, nnz, rp, ci = oracle.smtx_parse(text)
    shape = golden[f"smtx_{i}_shape"]
    assert (M, K, nnz) == tuple(int(x) for x in shape)
    A = oracle.pattern_to_dense(M, K, rp, ci)
    r, c = np.nonzero(A.view(np.uint16))
    assert np.array_equal(np.stack([r, c]).astype(np.int32), golden[f"smtx_{i}_coords"])
    assert np.all(A[r, c] == 1.0)


@pytest.mark.parametrize("i", [0, 1, 2])
def test_dense_csr_roundtrip_matches_reference(golden, i):
    A = golden[f"d2c_{i}_A"]
    rp, ci, v = oracle.dense_to_csr(A)
    assert np.array_equal(rp, golden[f"d2c_{i}_row_ptr"])
    assert np.array_equal(ci, golden[f"d2c_{i}_col"])
    assert np.array_equal(v.view(np.uint16), golden[f"d2c_{i}_val"].view(np.uint16))
    D = oracle.csr_to_dense(A.shape[0], A.shape[1], rp, ci, v)
    assert np.array_equal(D.view(np.uint16), golden[f"c2d_{i}_dense"].view(np.uint16))


@pytest.mark.parametrize("i", [0, 1, 2])
def test_fp32_spmm_is_bitwise_reference_naive_gemm(golden, i):
    """CSR-order FP32 accumulation == the reference's dense naive_gemm."""
    A, B, C = golden[f"gemm_{i}_A"], golden[f"gemm_{i}_B"], golden[f"gemm_{i}_C"]
    rp, ci, v = oracle.dense_to_csr(A)
    got = oracle.spmm_f32(rp, ci, v, B)
    assert np.array_equal(got.view(np.uint32), C.view(np.uint32))
    assert np.array_equal(oracle.gemm_f32(A, B).view(np.uint32), C.view(np.uint32))
    c64 = oracle.spmm_f64(rp, ci, v, B)
    assert np.allclose(c64, C, rtol=1e-5, atol=1e-5)


def test_compare_mat_semantics():
    gold = np.array([1.0, 100.0, 1e-5, 0.0, 2.0], np.float32)
    x = np.array([1.0005, 100.5, 2e-5, 0.01, 2.0], np.float32)
    # rel>=tol and abs>=tol both needed: only index 1 (abs .5, rel .005) and 3 (abs .01, rel inf)
    assert oracle.compare_mat(gold, x, 1e-3) == 2


def test_smtx_rejects_malformed():
    with pytest.raises(ValueError):
        oracle.smtx_parse(b"4, 4, 2\n0 1 2 2\n0 1\n")       # row_ptr too short
    with pytest.raises(ValueError):
        oracle.smtx_parse(b"2, 4, 2\n0 1 2\n0 9\n")         # column out of range
    with pytest.raises(ValueError):
        oracle.smtx_parse(b"2, 4, 3\n0 1 2\n0 1\n")         # nnz mismatch


def test_reference_warp_demand_bins():
    rp = np.cumsum([0, 0, 1, 8, 9, 16, 17, 32, 33, 64, 65, 200, 1000]).astype(np.int32)
    d = oracle.ref_warp_demand(rp, N=256)
    assert list(d) == [0, 1, 1, 2, 2, 4, 4, 8, 8, 8 * 2, 8 * 4, 8 * 4]


def test_reference_fixture_parse(golden):
    """The reference's own data file (copied into tests/golden/ by
    make_golden.py), parsed by the oracle, against the reference's
    smtx_input_to_Dense output recorded beside it."""
    path = ROOT / "tests" / "golden" / "body_decoder_layer_2_ffn_conv1.smtx"
    M, K, nnz, rp, ci = oracle.smtx_parse(path.read_bytes())
    assert (M, K, nnz) == tuple(golden["fixture_shape"])
    r, c = golden["fixture_coords"]
    assert np.array_equal(np.repeat(np.arange(M), np.diff(rp)), r)
    assert np.array_equal(ci, c)
    assert (np.diff(rp) > 64).any()  # exercises the reference's long-row path


@pytest.mark.skipif(REFERENCE_TREE is None or not (REFERENCE_TREE / "data").exists(),
                    reason="TCA_REFERENCE_ROOT not set")
def test_reference_fixture_parse_live():
    """The reference's own data file, parsed by the oracle and by the
    reference's smtx_input_to_Dense (oracle/_ref), must agree exactly."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    path = next((REFERENCE_TREE / "data").glob("*.smtx"))
    M, K, nnz, rp, ci = oracle.smtx_parse(path.read_bytes())
    A_ref, nnz_ref = oracle.ref_smtx_to_dense(path)
    assert (M, K, nnz) == (A_ref.shape[0], A_ref.shape[1], nnz_ref)
    A = oracle.pattern_to_dense(M, K, rp, ci)
    assert np.array_equal(A.view(np.uint16), A_ref.view(np.uint16))
    assert (np.diff(rp) > 64).any()  # exercises the reference's long-row path
