"""Device-side failure detection of the tensor-core kernel.

Every mbarrier wait in the kernel is bounded (about one second of
%globaltimer); when one runs out the CTA records TCA_ERR_TIMEOUT in the plan's
status word, waits for the work it issued (its MMAs, a bounded time for bulk
copies), releases its tensor memory and ends. The test makes a wait run out
with the TCA_FLAG_TEST_WITHHOLD_ACCUM hook -- each CTA's last accumulator is
never announced, so the epilogue's wait for it expires -- and checks that:
the call itself succeeds, tca_plan_status reports TCA_ERR_TIMEOUT once (the
status word is read and cleared), rows the withheld items own stay unwritten
while the others are correct, and the context stays usable: the next forward
on the same plan is correct and its status is TCA_OK. No fault, trap or hang
is involved: the wait that runs out is one that nothing completes."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from tca_spmm import gen

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import tca_spmm  # noqa: E402

TCA_OK, TCA_ERR_TIMEOUT = 0, 5
FLAG_TEST_WITHHOLD_ACCUM = 1 << 31  # include/tca_spmm.h


def test_bounded_wait_runs_out_and_context_survives(cuda):
    c = gen.sweep(0.80, N=128, seed=7001)
    rp, ci, v = (torch.from_numpy(x.copy()).to(cuda) for x in (c["row_ptr"], c["col"], c["vals"]))
    B = torch.from_numpy(c["B"]).to(cuda)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    info = plan.info()
    assert info["n_tc_windows"] > 0, info
    L = tca_spmm.lib()
    ref = oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
    sentinel = 12345.0
    C = torch.full((c["M"], 128), sentinel, dtype=torch.float32, device=cuda)
    rc = L.tca_spmm(plan.handle, B.data_ptr(), B.stride(0), 128, C.data_ptr(), C.stride(0), tca_spmm.DTYPE_F32,
                    ctypes.c_float(1.0), ctypes.c_float(0.0), ctypes.c_uint(FLAG_TEST_WITHHOLD_ACCUM),
                    torch.cuda.current_stream().cuda_stream)
    assert rc == TCA_OK, L.tca_last_error_string()
    torch.cuda.synchronize()  # the launch ended (after the bounded wait), without a CUDA error
    assert L.tca_plan_status(plan.handle) == TCA_ERR_TIMEOUT
    assert b"bounded" in L.tca_last_error_string()
    assert L.tca_plan_status(plan.handle) == TCA_OK  # read and cleared
    got = C.cpu().numpy()
    unwritten = np.all(got == sentinel, axis=1)
    assert unwritten.any()  # the withheld items' rows
    ok_rows = ~unwritten
    assert np.abs(got[ok_rows] - ref[ok_rows]).max() <= 1e-3 * np.abs(ref).max()
    # the context and the plan are still usable
    C2 = plan.spmm(B, out_dtype=torch.float32)
    torch.cuda.synchronize()
    assert L.tca_plan_status(plan.handle) == TCA_OK
    assert np.linalg.norm(C2.cpu().numpy() - ref) <= 1e-3 * np.linalg.norm(ref)
