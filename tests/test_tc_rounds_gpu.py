"""The tensor-core kernel over batches whose work items (window x N-slice)
fill the persistent grid in different ways: a partial last round, a single
partial round, several full rounds, at N-slice widths 64, 128 and 256, with
dense windows (tile images, 64 contiguous B rows per chunk: tiled TMA) and
sparse ones (scattered entries, condensed B rows: gather4). FP16 against the
FP64 oracle (tolerances of test_spmm_gpu.assert_close); E4M3 against the
FP64 product of the dequantized operands (relative Frobenius error <= 2e-5,
FP32 output)."""
import numpy as np
import pytest

from oracle import oracle
from tca_spmm import gen
from test_spmm_gpu import assert_close, dev

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402

GRID = 148  # persistent tensor-core CTAs (one per SM)
WINDOWS = 40  # 128-row windows per matrix, all on the tensor cores


def cases(n, N, seed):
    """Dense windows (tile images, 64 contiguous B rows per chunk: tiled TMA)
    alternating with sparse ones (scattered entries, condensed B rows:
    gather4)."""
    return [gen.small(np.random.default_rng(seed + i), 128 * WINDOWS, 256, N, 0.3 if i % 2 == 0 else 0.02,
                      empty_rows=0.02)
            for i in range(n)]


def plans_of(cs, cuda):
    out = []
    for c in cs:
        rp, ci, v, B = dev(c, cuda)
        p = tca_spmm.Plan(rp, ci, v, c["K"], path="tensor_core")
        assert p.info()["n_tc_windows"] >= WINDOWS - 2
        out.append((p, B))
    return out


# (matrices, N, n_tile): items = tensor-core windows (~WINDOWS per matrix) x ceil(N / n_tile)
SHAPES = [
    (4, 256, 256),   # ~160 items: one round + ~12
    (4, 256, 128),   # ~320 items: two rounds + ~24
    (2, 256, 256),   # ~80 items: a single partial round
    (1, 256, 256),   # 40 items
    (1, 200, 256),   # the slice partly beyond N
    (1, 256, 128),   # 80 items
    (4, 256, 64),    # ~640 items: four rounds + ~48
]


@pytest.mark.parametrize("shape", SHAPES, ids=[f"{m}x{n}_nt{t}" for m, n, t in SHAPES])
@pytest.mark.parametrize("out_dtype", ["f16", "f32"])
def test_f16_rounds(cuda, shape, out_dtype):
    m, N, nt = shape
    cs = cases(m, N, 500 + N + nt)
    pb = plans_of(cs, cuda)
    dt = torch.float16 if out_dtype == "f16" else torch.float32
    outs = [torch.full((c["M"], N), 9.0, dtype=dt, device=cuda) for c in cs]
    tca_spmm.spmm_batched([p for p, _ in pb], [B for _, B in pb], outs, n_tile=nt)
    torch.cuda.synchronize()
    for (p, _), C, c in zip(pb, outs, cs):
        p.status()
        assert_close(C, c)


@pytest.mark.parametrize("shape", [(4, 256, 256), (1, 256, 256), (2, 256, 256), (4, 256, 128)],
                         ids=["4x256_nt256", "1x256_nt256", "2x256_nt256", "4x256_nt128"])
def test_e4m3_rounds(cuda, shape):
    m, N, nt = shape
    cs = cases(m, N, 900 + nt)
    pb = plans_of(cs, cuda)
    outs = [torch.empty((c["M"], N), dtype=torch.float32, device=cuda) for c in cs]
    tca_spmm.spmm_fp8_batched([p for p, _ in pb], [B for _, B in pb], outs, n_tile=nt)
    torch.cuda.synchronize()
    for (p, _), C, c in zip(pb, outs, cs):
        p.status()
        ref = oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
        got = C.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 2e-5
