"""The host build of the tile format (oracle) against its own definition:
it must be a lossless re-encoding of the CSR. The GPU build is compared with
it bit for bit in test_spmm_gpu.py."""
import numpy as np
import pytest

from oracle import oracle
from tca_spmm import gen


def reconstruct_from_tiles(p, M, K):
    """Dense A rebuilt only from tensor-core tiles + CUDA-core windows."""
    A = np.zeros((M, K), np.float64)
    perm = p["perm"]
    for t, w in enumerate(p["tc_windows"]):
        for c in range(p["tile_first"][t], p["tile_first"][t + 1]):
            cols = p["win_cols"][c * 64:(c + 1) * 64]
            for e in p["tile_entries"][p["tile_ptr"][c]:p["tile_ptr"][c + 1]]:
                lr, lc, bits = int(e) >> 22, (int(e) >> 16) & 63, np.uint16(int(e) & 0xffff)
                r = perm[w * 128 + lr]
                assert cols[lc] >= 0
                A[r, cols[lc]] += float(bits.view(np.float16))
    for w in p["cc_windows"]:
        for i in range(w * 128, min(M, w * 128 + 128)):
            for j in range(p["p_row_ptr"][i], p["p_row_ptr"][i + 1]):
                A[perm[i], p["p_col"][j]] += float(p["p_val"][j].view(np.float16))
    return A


@pytest.mark.parametrize("sort_rows", [True, False])
@pytest.mark.parametrize("path", [0, 1, 2])
def test_plan_reencodes_csr(sort_rows, path):
    rng = np.random.default_rng(7)
    c = gen.small(rng, 300, 200, 16, 0.1, empty_rows=0.2)
    p = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], c["K"], sort_rows=sort_rows, path=path)
    M, K = c["M"], c["K"]
    perm = p["perm"]
    assert sorted(perm) == list(range(M))
    nnz = np.diff(c["row_ptr"])
    if sort_rows:
        keys = list(zip(-nnz[perm], perm))
        assert keys == sorted(keys)
    else:
        assert np.array_equal(perm, np.arange(M))
    assert p["n_tc"] + p["n_cc"] == p["n_windows"] == (M + 127) // 128
    if path == 1:
        assert p["n_tc"] == 0
    if path == 2:  # only windows without nonzeros stay off the tensor cores
        for w in p["cc_windows"]:
            lo, hi = w * 128, min(M, w * 128 + 128)
            assert p["p_row_ptr"][hi] == p["p_row_ptr"][lo]
    dense = np.zeros((M, K), np.float64)
    for r in range(M):
        for j in range(c["row_ptr"][r], c["row_ptr"][r + 1]):
            dense[r, c["col"][j]] = float(c["vals"][j])
    assert np.array_equal(reconstruct_from_tiles(p, M, K), dense)
    # src maps every sorted entry back to the caller's value
    assert np.array_equal(p["p_val"], c["vals"].view(np.uint16)[p["src"]])
    assert np.array_equal(p["tile_entries"] & 0xffff, p["p_val"][p["tile_src"]])
    check_images(p)


def unswizzle(img):
    """128 x 64 tile from its 128-byte swizzled K-major image."""
    t = np.zeros((128, 64), np.uint16)
    for r in range(128):
        for c in range(64):
            byte = r * 128 + (((c >> 3) ^ (r & 7)) << 4) + ((c & 7) << 1)
            t[r, c] = img[byte // 2]
    return t


def check_images(p):
    """Every chunk with >= 512 entries (1/16 of the tile) has an image equal to its entries."""
    ptr = p["tile_ptr"]
    n_img = 0
    for ch in range(p["n_tc_chunks"]):
        cnt = ptr[ch + 1] - ptr[ch]
        idx = p["tile_image_idx"][ch]
        assert (idx >= 0) == (cnt >= 512)
        if idx < 0:
            continue
        assert idx == n_img
        n_img += 1
        t = unswizzle(p["tile_images"][idx * 8192:(idx + 1) * 8192])
        want = np.zeros((128, 64), np.uint16)
        for e in p["tile_entries"][ptr[ch]:ptr[ch + 1]]:
            want[int(e) >> 22, (int(e) >> 16) & 63] = int(e) & 0xffff
        assert np.array_equal(t, want)
    assert n_img == p["n_images"]


@pytest.mark.parametrize("path", [0, 1])
def test_cuda_core_items_cover_rows(path):
    rng = np.random.default_rng(8)
    c = gen.sweep(0.9, N=64, M=700, K=512)
    p = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], c["K"], path=path)
    M = c["M"]
    rp = p["p_row_ptr"]
    for key, wins in (("cc_items", p["cc_windows"]), ("all_items", np.arange(p["n_windows"]))):
        items = p[key].reshape(-1, 2)
        rows = np.concatenate([np.arange(a, b) for a, b in items]) if len(items) else np.zeros(0, int)
        want = np.concatenate([np.arange(w * 128, min(M, w * 128 + 128)) for w in wins]) if len(wins) else rows
        assert np.array_equal(rows, want)
        for a, b in items:
            assert 1 <= b - a <= 31
            assert b - a == 1 or rp[b] - rp[a] <= 32


def test_dense_chunks_get_images():
    rng = np.random.default_rng(4)
    c = gen.small(rng, 256, 128, 8, 0.8)
    p = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], c["K"])
    assert p["n_images"] >= 2
    check_images(p)


def test_window_columns_are_sorted_distinct():
    rng = np.random.default_rng(9)
    c = gen.small(rng, 256, 500, 8, 0.05)
    p = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], c["K"], path=2)
    for t in range(p["n_tc"]):
        cols = p["win_cols"][p["tile_first"][t] * 64:p["tile_first"][t + 1] * 64]
        real = cols[cols >= 0]
        assert np.all(np.diff(real) > 0)
        assert np.all(cols[len(real):] == -1) and len(cols) - len(real) < 64


def test_unsorted_rows_go_to_cuda_cores():
    row_ptr = np.array([0, 3, 5], np.int32)
    col = np.array([5, 1, 3, 2, 2], np.int32)  # row 0 unsorted, row 1 duplicate
    vals = np.ones(5, np.float16)
    p = oracle.build_plan(row_ptr, col, vals, 8, path=2)
    assert p["n_tc"] == 0 and p["n_cc"] == 1


def test_density_threshold_decides_path():
    rng = np.random.default_rng(3)
    c = gen.small(rng, 128, 64, 8, 0.5)  # one window, one chunk, density ~0.5
    hi = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], 64, tc_min_density=0.9)
    lo = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], 64, tc_min_density=0.1)
    assert hi["n_tc"] == 0 and lo["n_tc"] == 1


def test_default_density_split_of_the_sweep_problem():
    """The default threshold (0.01) on the 4096 x 1024, 80 % Zipf problem:
    windows whose rows hold 10 or more nonzeros (16 direct chunks, density
    >= 0.0126) take the tensor cores, the windows of rows with at most 10 stay
    on the CUDA cores, among them the windows of one-nonzero
    rows (128 nonzeros in 2 condensed chunks, density 0.0078)."""
    c = gen.sweep(0.8, N=256, seed=7000)
    p = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], c["K"])
    assert p["n_tc"] == 13 and p["n_cc"] == 19
    prp = p["p_row_ptr"]
    for w in p["cc_windows"]:
        lens = np.diff(prp[w * 128:w * 128 + 129])
        assert lens.max() <= 10
    singles = [w for w in p["cc_windows"] if np.all(np.diff(prp[w * 128:w * 128 + 129]) == 1)]
    assert len(singles) == 12
    old = oracle.build_plan(c["row_ptr"], c["col"], c["vals"], c["K"], tc_min_density=0.02)
    assert old["n_tc"] == 11 and set(old["tc_windows"]) < set(p["tc_windows"])


def test_malformed_csr_rejected():
    with pytest.raises(ValueError):
        oracle.build_plan(np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32), np.ones(2, np.float16), 4)
    with pytest.raises(ValueError):
        oracle.build_plan(np.array([0, 1], np.int32), np.array([9], np.int32), np.ones(1, np.float16), 4)
