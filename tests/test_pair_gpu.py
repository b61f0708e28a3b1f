"""The tensor-core pair kernel (two windows with identical chunk columns on a
CTA pair, tcgen05 cta_group::2) against the single-window kernel on the same
plans and against the FP64 oracle.

Pairs are formed by the plan builder: consecutive tensor-core windows that
are direct and touch every 64-column block of K. The pair kernel runs for
N-slices of 256 (batched forwards, or single forwards with enough windows);
The pair kernel is opt-in (`pair_windows=True`; measured slower than the
single-window kernel on the sweep problems); `pair_windows=False`, the
default, keeps the same plan on the single-window kernel.

Tolerances: FP32 output |C - C64| <= 1e-5 * (|A| |B|) elementwise (the FP32
rounding scale); pair vs single kernel: relative Frobenius <= 1e-6 (the same
products in the same chunk order)."""
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


def check_f64(C, c):
    got = C.double().cpu().numpy()
    ref = oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
    S = oracle.spmm_f64(c["row_ptr"], c["col"], np.abs(c["vals"].astype(np.float32)).astype(np.float16),
                        np.abs(c["B"].astype(np.float32)).astype(np.float16))
    bad = np.abs(got - ref) > 1e-5 * S + 1e-30
    assert not bad.any(), f"{bad.sum()} elements off"


def rel(a, b):
    a, b = a.double().cpu().numpy(), b.double().cpu().numpy()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def cases():
    rng = np.random.default_rng(71)
    # every window dense and direct over all of K: all pairs, odd count -> one alone
    yield "dense_odd", gen.small(rng, 128 * 7 - 5, 520, 256, 0.08)
    # N not a multiple of 256: the second slice is partly (second half: wholly) outside N
    yield "n320", gen.small(rng, 128 * 6, 256, 320, 0.1)
    # the sweep problem itself (13 tensor-core windows, 6 pairs + 1 alone)
    yield "sweep80", gen.sweep(0.8, N=256, seed=7000)


@pytest.mark.parametrize("name,c", list(cases()), ids=lambda x: x if isinstance(x, str) else "")
def test_pair_kernel_matches_single_window_kernel(cuda, name, c):
    rp, ci, v, B = dev(c, cuda)
    paired = tca_spmm.Plan(rp, ci, v, c["K"], pair_windows=True)
    single = tca_spmm.Plan(rp, ci, v, c["K"], pair_windows=False)
    pairs = paired.export(tca_spmm.ARR_TC_PAIRS).reshape(-1, 2)
    n_tc = paired.info()["n_tc_windows"]
    assert n_tc > 0 and (pairs[:, 1] >= 0).sum() * 3 >= n_tc, pairs  # the pair kernel takes the plan
    # batched forwards take 256-wide N-slices, hence the pair kernel
    outs = []
    for plan in (paired, single):
        C = torch.empty((c["M"], c["N"]), dtype=torch.float32, device=cuda)
        tca_spmm.spmm_batched([plan], [B], [C])
        torch.cuda.synchronize()
        plan.status()
        outs.append(C)
    check_f64(outs[0], c)
    assert rel(outs[0], outs[1]) <= 1e-6


def test_pair_kernel_e4m3_and_fp16_out(cuda):
    c = gen.sweep(0.8, N=256, seed=7001)
    rp, ci, v, B = dev(c, cuda)
    paired = tca_spmm.Plan(rp, ci, v, c["K"], pair_windows=True)
    single = tca_spmm.Plan(rp, ci, v, c["K"], pair_windows=False)
    res = {}
    for name, plan in (("paired", paired), ("single", single)):
        C8 = torch.empty((c["M"], c["N"]), dtype=torch.float32, device=cuda)
        tca_spmm.spmm_fp8_batched([plan], [B], [C8])
        C16 = torch.empty((c["M"], c["N"]), dtype=torch.float16, device=cuda)
        tca_spmm.spmm_batched([plan], [B], [C16])
        torch.cuda.synchronize()
        plan.status()
        res[name] = (C8, C16)
    ref8 = oracle.spmm_fp8_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
    got8 = res["paired"][0].double().cpu().numpy()
    assert np.linalg.norm(got8 - ref8) <= 2e-5 * np.linalg.norm(ref8)
    assert rel(res["paired"][0], res["single"][0]) <= 1e-6
    assert torch.equal(res["paired"][1], res["single"][1]) or rel(res["paired"][1], res["single"][1]) <= 1e-3


def test_pair_kernel_batch_of_many_plans(cuda):
    """32 problems in one launch: pair items of all jobs over the persistent
    CTA pairs, against the single-window kernel."""
    distinct = [gen.sweep(0.8, N=256, seed=7100 + i) for i in range(4)]
    plans_p, plans_s, Bs, Cp, Cs = [], [], [], [], []
    for g in range(32):
        c = distinct[g % 4]
        rp, ci, v, B = dev(c, cuda)
        plans_p.append(tca_spmm.Plan(rp, ci, v, c["K"], pair_windows=True))
        plans_s.append(tca_spmm.Plan(rp, ci, v, c["K"], pair_windows=False))
        Bs.append(B)
        Cp.append(torch.empty((c["M"], 256), dtype=torch.float32, device=cuda))
        Cs.append(torch.empty((c["M"], 256), dtype=torch.float32, device=cuda))
    tca_spmm.spmm_batched(plans_p, Bs, Cp)
    tca_spmm.spmm_batched(plans_s, Bs, Cs)
    torch.cuda.synchronize()
    for g in range(32):
        plans_p[g].status()
        assert rel(Cp[g], Cs[g]) <= 1e-6, g
    check_f64(Cp[0], distinct[0])


def test_unpairable_plan_stays_on_single_window_kernel(cuda):
    """Windows that do not touch every block of K (condensed or partial
    direct) are alone; with fewer than two thirds of the windows paired the
    plan keeps the single-window kernel, and results are unchanged."""
    rng = np.random.default_rng(72)
    c = gen.sweep(0.95, N=256, M=1024, K=4096, seed=72)
    rp, ci, v, B = dev(c, cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"], pair_windows=True)
    pairs = plan.export(tca_spmm.ARR_TC_PAIRS).reshape(-1, 2)
    if plan.info()["n_tc_windows"] == 0:
        pytest.skip("no tensor-core windows in this case")
    assert pairs.shape[0] == plan.info()["n_tc_windows"] - (pairs[:, 1] >= 0).sum()
    C = torch.empty((c["M"], 256), dtype=torch.float32, device=cuda)
    tca_spmm.spmm_batched([plan], [B], [C])
    torch.cuda.synchronize()
    check_f64(C, c)
    del rng
