"""The FP64 mode (tca_spmm_csr_f64) against an FP64 product computed on the
CPU (scipy): relative Frobenius error <= 1e-13 (only the summation order
differs), alpha / beta, rows without nonzeros kept, any N and strides."""
import numpy as np
import pytest
import scipy.sparse as sp

from tca_spmm import gen

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402


@pytest.mark.parametrize("M,K,N,d", [(300, 200, 64, 0.1), (1000, 700, 33, 0.02), (64, 4096, 300, 0.5), (5, 3, 1, 0.9)])
def test_f64_forward(cuda, M, K, N, d):
    rng = np.random.default_rng(M + N)
    c = gen.small(rng, M, K, 8, d, empty_rows=0.1)
    vals = rng.standard_normal(c["col"].size)
    B = rng.standard_normal((K, N))
    C0 = rng.standard_normal((M, N))
    A = sp.csr_matrix((vals, c["col"], c["row_ptr"]), shape=(M, K))
    ref = 0.5 * (A @ B) - 2.0 * C0
    empty = np.diff(c["row_ptr"]) == 0
    ref[empty] = C0[empty]
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(cuda)
    C = t(C0)
    tca_spmm.spmm_csr_f64(t(c["row_ptr"]), t(c["col"]), t(vals), t(B), K=K, out=C, alpha=0.5, beta=-2.0,
                          keep_empty_rows=True)
    got = C.cpu().numpy()
    assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref)
    np.testing.assert_array_equal(got[empty], C0[empty])
