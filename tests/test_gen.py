"""Seeded synthetic inputs have the stated shapes, counts and orderings."""
import numpy as np

from tca_spmm import gen


def _check_csr(c):
    rp, col = c["row_ptr"], c["col"]
    assert rp[0] == 0 and rp[-1] == col.size and np.all(np.diff(rp) >= 0)
    assert col.min() >= 0 and col.max() < c["K"]
    for r in range(0, c["M"], max(1, c["M"] // 64)):
        seg = col[rp[r]:rp[r + 1]]
        assert np.all(np.diff(seg) > 0)
    assert c["vals"].dtype == np.float16 and c["B"].dtype == np.float16


def test_cfg1_shape_and_sparsity():
    c = gen.cfg1()
    _check_csr(c)
    assert (c["M"], c["K"], c["N"]) == (2048, 512, 256) and c["B"].shape == (512, 256)
    assert abs(c["col"].size - 209715) < 3000
    again = gen.cfg1()
    assert np.array_equal(again["col"], c["col"]) and np.array_equal(again["B"], c["B"])


def test_sweep_exact_nnz_and_zipf_clipping():
    for s in (0.8, 0.98):
        c = gen.sweep(s, N=64)
        _check_csr(c)
        assert c["col"].size == int(round((1 - s) * 4096 * 1024))
        nnz = np.diff(c["row_ptr"])
        assert nnz.min() >= 1 and nnz.max() <= 1024
        assert nnz.max() > 10 * np.median(nnz)  # heavy tail


def test_zipf_rescale_hits_target():
    rng = np.random.default_rng(0)
    for total in (5000, 50000, 300000):
        n = gen.zipf_row_nnz(rng, 1000, 512, total)
        assert n.sum() == total and n.min() >= 1 and n.max() <= 512
