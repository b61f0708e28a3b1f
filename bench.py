"""Benchmark of the CSR x dense SpMM forward on B200.

Workload (one step): the plain FP16 forward of G independent copies of the
sweep matrix 4096 x 1024 at 80% sparsity (Zipf(1.2) row lengths, values
N(0, 0.03)), B 1024 x 256 FP16 U(-1, 1), FP16 output with FP32 accumulation.
Four seeded patterns are each replicated G/4 times into separate device
buffers, so that the inputs of one step (G = 32: ~245 MB) exceed the 126 MB
L2 and every problem is read from HBM.

  value      GFLOP/s (2 nnz N per problem) with inputs resident in HBM,
             device time of K steps (CUDA events), max over ranks
  e2e        the same metric through the host-buffer entry point
             (tca_spmm_host, the reference's calling convention): per step one
             problem's CSR and B are copied in from pinned memory, the plan is
             built, the forward runs and C is copied back
  roofline   HBM roofline of the dominant kernel: algorithmic bytes of the
             work it does per launch / its mean CUDA-event duration
  cpu_baseline  the oracle's OpenMP FP32 CSR x dense on the host cores, one
             problem, repeated for a bounded time
  fp8, batching, fwd_bwd  the E4M3 step, the 24-layer batch (graph vs
             sequential) and the differentiation config (forward vs forward +
             SDDMM + transpose SpMM, gradient errors vs FP64)

  per_problem  one problem per call at every point of the forward target
             (4096 x 1024 at 70-98 % sparsity, N = 64-512): this project, the
             reference's TCA kernel with its own schedule and the reference
             comparator's cuSPARSE call on the same device buffers, timed the
             same way (CUDA graph of 100 calls hot; one call after an L2 flush
             cold), with speed-ups, roofline fractions and errors vs FP64

--impl reference times the reference's own CPU implementation of the
product, naive_gemm (built from the reference sources into oracle/_ref), on
the host cores: the whole first problem per step when the run fits in
REF_BUDGET_S, else a row sample; the line also carries, under reference_gpu,
the reference's TCA kernel (our_spmm_balanced) through its host API on the
same problems and its cuSPARSE comparator.

Multi-GPU (torchrun): each rank runs its own G problems (row-independent
work, no collective on the data path): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "tca-spmm_b200" / "python"))
sys.path.insert(0, str(ROOT))

METRIC = "SpMM GFLOP/s (2*nnz*N), FP16 in, FP32 accumulate, FP16 out"
REF_BUDGET_S = 120.0  # CPU seconds the reference arm's warm-up + timed steps may take
WORKLOAD = "sweep 4096x1024 sparsity 0.80 zipf(1.2) N=256"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)  # ~65 ms timed: several clock samples
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--problems", type=int, default=32, help="independent problems per step")
    ap.add_argument("--sparsity", type=float, default=0.80)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-per-problem", action="store_true", help="skip the per-problem comparison leg")
    ap.add_argument("--only", choices=["step", "step_e4m3", "fwd_bwd", "batching", "e2e", "csr", "f64", "cc_mma",
                                       "pair"], default=None,
                    help="run only this leg (for profiling: ncu captures of one kernel); prints its own line")
    return ap.parse_args()


class ClockSampler:
    """Samples SM clock and throttle reasons with NVML while running."""

    def __init__(self, device_index=0, period=0.01):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._period = period
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # NVML missing: report it, do not guess
            self._nv = None
            self.error = str(e)

    def _run(self):
        nv = self._nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
            "hw_power_brake_slowdown": getattr(nv, "nvmlClocksEventReasonHwPowerBrakeSlowdown", 0x80),
        }
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for k, bit in names.items():
                    if mask & bit:
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(self._period)

    def __enter__(self):
        if self._nv is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._nv is not None:
            self._t.join()

    def summary(self):
        if self._nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": "NVML unavailable"}
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_problems(args):
    from tca_spmm import gen
    distinct = [gen.sweep(args.sparsity, N=args.n, seed=7000 + i) for i in range(4)]
    return distinct


def problem_bytes(c, N, c_bytes=2):
    nnz = int(c["col"].size)
    return nnz * (2 + 4) + (c["M"] + 1) * 4 + c["K"] * N * 2 + c["M"] * N * c_bytes


def cpu_model():
    """The host CPU's model name (Linux /proc/cpuinfo), or the platform string."""
    try:
        for line in pathlib.Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def cpu_baseline(c, seconds):
    """The oracle's OpenMP FP32 CSR x dense SpMM on every host core this
    process may run on: one warm-up run, then runs until `seconds` have passed
    (at least 10, at most 1000); the figure is the median run."""
    from oracle import oracle
    nthreads = len(os.sched_getaffinity(0))
    flops = 2.0 * c["col"].size * c["B"].shape[1]
    oracle.spmm_f32(c["row_ptr"], c["col"], c["vals"], c["B"], nthreads=nthreads)  # warm-up
    times, t_start = [], time.perf_counter()
    while True:
        t0 = time.perf_counter()
        oracle.spmm_f32(c["row_ptr"], c["col"], c["vals"], c["B"], nthreads=nthreads)
        times.append(time.perf_counter() - t0)
        el = time.perf_counter() - t_start
        if (el >= seconds and len(times) >= 10) or len(times) >= 1000:
            break
    med = statistics.median(times)
    return {"value": round(flops / med / 1e9, 3), "unit": "GFLOP/s", "cores": nthreads, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"median of {len(times)} runs of one {c['M']}x{c['K']} problem (nnz={c['col'].size}, "
                      f"N={c['B'].shape[1]}) in {el:.1f} s after one warm-up, OpenMP FP32 CSR x dense "
                      f"(oracle/tca_oracle.c orc_spmm_f32)"}


def dist_setup(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(x, world):
    import torch
    import torch.distributed as dist
    if world == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, world, rank):
    import torch
    import tca_spmm
    distinct = make_problems(args)
    G = args.problems
    dev = torch.device("cuda", torch.cuda.current_device())
    probs = []
    for g in range(G):
        c = distinct[g % len(distinct)]
        rp = torch.from_numpy(c["row_ptr"]).to(dev)
        ci = torch.from_numpy(c["col"]).to(dev)
        v = torch.from_numpy(c["vals"]).to(dev)
        B = torch.from_numpy(c["B"]).to(dev)
        C = torch.empty((c["M"], args.n), dtype=torch.float16, device=dev)
        plan = tca_spmm.Plan(rp, ci, v, c["K"])
        probs.append((c, plan, B, C))
    torch.cuda.synchronize()
    info = probs[0][1].info()
    flops_step = sum(2.0 * c["col"].size * args.n for c, *_ in probs)
    bytes_step = sum(problem_bytes(c, args.n) for c, *_ in probs)
    in_bytes_step = sum(problem_bytes(c, args.n) - c["M"] * args.n * 2 for c, *_ in probs)
    plans = [p for _, p, _, _ in probs]
    Bs = [B for _, _, B, _ in probs]
    Cs = [C for _, _, _, C in probs]
    # one batched call per step: tensor-core launches (<= 32 problems each, one
    # N-slice width here) then CUDA-core launches (<= 32 problems each)
    n_tc_jobs = sum(1 for p in plans if p.info()["n_tc_windows"] > 0)
    n_cc_jobs = sum(1 for p in plans if p.info()["n_cc_windows"] > 0)
    launches_per_step = -(-n_tc_jobs // 32) + -(-n_cc_jobs // 32)

    # the step replays the batch captured as a CUDA graph (tca_batch_graph_*):
    # the host side of an eager 32-problem call (argument checks, 64 TMA
    # descriptors) costs more than its device time
    graph16 = tca_spmm.BatchGraph(plans, Bs, Cs)

    def step():
        graph16.launch()

    for _ in range(args.warmup):
        step()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        barrier(world)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        barrier(world)
    ms_total = max_over_ranks(e0.elapsed_time(e1), world)
    ms_step = ms_total / args.steps
    value = world * flops_step / (ms_step * 1e-3) / 1e9

    # per-kernel device time: the same batch captured once more with CUDA
    # events recorded inside the graph around the tensor-core and the
    # CUDA-core launches, replayed n_prof times
    n_prof = max(1, min(args.steps, 20))
    tc_ms, cc_ms = kernel_times(tca_spmm, torch, plans, Bs, Cs, "f16", n_prof)
    # algorithmic bytes per launch, per problem part: the part's nonzeros
    # (2 B value + 4 B index), row offsets and output rows, plus B once
    tc_bytes = cc_bytes = 0
    for p in plans:
        inf = p.info()
        tc_rows = min(inf["M"], inf["n_tc_windows"] * 128)
        cc_rows = inf["M"] - tc_rows
        if inf["n_tc_windows"]:
            tc_bytes += inf["tc_nnz"] * 6 + (tc_rows + 1) * 4 + inf["K"] * args.n * 2 + tc_rows * args.n * 2
        if inf["n_cc_windows"]:
            cc_bytes += ((inf["nnz"] - inf["tc_nnz"]) * 6 + (cc_rows + 1) * 4 + inf["K"] * args.n * 2
                         + cc_rows * args.n * 2)
    tc_mean, cc_mean = float(np.mean(tc_ms)), float(np.mean(cc_ms))
    dominant = "spmm_tc_kernel" if n_tc_jobs and tc_mean >= cc_mean else "spmm_cc_stream_kernel"
    dom_ms, dom_bytes = (tc_mean, tc_bytes) if dominant == "spmm_tc_kernel" else (cc_mean, cc_bytes)
    peak, peak_kind = peaks()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(dominant)

    # FP8-E4M3 forward of the same step (per-row A / per-column B scales; B is
    # quantized inside every step), and the error of both precisions vs FP64
    graph8 = tca_spmm.BatchGraph(plans, Bs, Cs, precision="e4m3")

    def step8():
        graph8.launch()

    for _ in range(args.warmup):
        step8()
    barrier(world)
    e0.record()
    for _ in range(args.steps):
        step8()
    e1.record()
    barrier(world)
    ms8 = max_over_ranks(e0.elapsed_time(e1), world) / args.steps
    tc8_ms, cc8_ms = kernel_times(tca_spmm, torch, plans, Bs, Cs, "e4m3", n_prof)
    fp8 = {"value": round(world * flops_step / (ms8 * 1e-3) / 1e9, 3), "unit": "GFLOP/s",
           "ms_per_step": round(ms8, 5), "speedup_vs_fp16": round(ms_step / ms8, 3),
           "kernels_us": {"spmm_tc_kernel_e4m3": round(float(np.mean(tc8_ms)) * 1e3, 3),
                          "spmm_cc_stream_kernel_e4m3": round(float(np.mean(cc8_ms)) * 1e3, 3)},
           "quantization": "E4M3, per-row A and per-column B FP32 scales, FP32 accumulation, FP16 out; "
                           "B is quantized inside every step"}
    if rank == 0 and not args.no_cpu:
        from oracle import oracle
        c0 = probs[0][0]
        ref = oracle.spmm_f64(c0["row_ptr"], c0["col"], c0["vals"], c0["B"])
        y16 = plans[0].spmm(Bs[0]).float().cpu().numpy()
        y8 = plans[0].spmm_fp8(Bs[0]).float().cpu().numpy()
        nrm = np.linalg.norm(ref)
        fp8["rel_err_vs_f64"] = float(f"{np.linalg.norm(y8 - ref) / nrm:.4e}")
        fp8["fp16_rel_err_vs_f64"] = float(f"{np.linalg.norm(y16 - ref) / nrm:.4e}")

    # e2e through the host-buffer entry point
    e2e_steps = max(1, min(args.steps, 8))
    pinned = []
    for c in distinct:
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        pinned.append(dict(rp=pin(c["row_ptr"]), ci=pin(c["col"]), v=pin(c["vals"]), B=pin(np.ascontiguousarray(c["B"])),
                           C=torch.empty((c["M"], args.n), dtype=torch.float16).pin_memory().numpy(), c=c))
    tca_spmm.spmm_host(pinned[0]["rp"], pinned[0]["ci"], pinned[0]["v"], 1024, pinned[0]["B"], C=pinned[0]["C"],
                       keep_empty_rows=False)
    barrier(world)
    t0 = time.perf_counter()
    e2e_flops = 0.0
    h2d = d2h = 0
    for s in range(e2e_steps):
        p = pinned[s % len(pinned)]
        tca_spmm.spmm_host(p["rp"], p["ci"], p["v"], p["c"]["K"], p["B"], C=p["C"], keep_empty_rows=False)
        e2e_flops += 2.0 * p["c"]["col"].size * args.n
        h2d += p["rp"].nbytes + p["ci"].nbytes + p["v"].nbytes + p["B"].nbytes
        d2h += p["C"].nbytes
    barrier(world)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e = {"value": round(world * e2e_flops / e2e_s / 1e9, 3), "unit": "GFLOP/s",
           "h2d_bytes_per_step": h2d // e2e_steps, "d2h_bytes_per_step": d2h // e2e_steps,
           "steps": e2e_steps, "path": "tca_spmm_host (host buffers, plan build inside the timed region)"}

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16",
        "data": "synthetic (seeded numpy PCG64)",
        "config": {"workload": WORKLOAD, "problems_per_step": G, "distinct_patterns": len(distinct),
                   "M": 4096, "K": 1024, "N": args.n, "sparsity": args.sparsity,
                   "nnz_per_problem": [int(c["col"].size) for c in distinct],
                   "bytes_per_step": bytes_step, "input_bytes_per_step": in_bytes_step,
                   "l2": "inputs larger than L2 (126 MB): each problem's buffers are distinct",
                   "parallelism": f"dp{world} (independent problems per rank)",
                   "plan": info},
        "hbm_gbs_achieved_step": round(world * bytes_step / (ms_step * 1e-3) / 1e9, 1),
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes,
                     "mean_launch_us": round(dom_ms * 1e3, 3),
                     "kernels_us": {"spmm_tc_kernel": round(tc_mean * 1e3, 3),
                                    "spmm_cc_stream_kernel": round(cc_mean * 1e3, 3)},
                     "kernels_timing": "each kernel group alone (events serialize the two paths); in the "
                                       "timed step the CUDA-core launch runs beside the tensor-core launch "
                                       "as its programmatic dependent"},
        "e2e": e2e,
        "fp8": fp8,
        "batching": batching_leg(args, world),
        "fwd_bwd": fwd_bwd_leg(args, rank == 0 and not args.no_cpu),
        "per_problem": per_problem_leg(args, rank == 0 and not args.no_cpu) if not args.no_per_problem else None,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
    }
    return out, distinct


def run_only(args, world):
    """One leg alone, for profiling runs: the headline step (FP16 or E4M3)
    replayed `steps` times after `warmup`, the differentiation config, the
    batching config, or the host-buffer forward; or one of the kernels off
    the headline path on the headline problem: the plan-free forward (csr),
    the FP64 forward (f64), the step with the CUDA-core rows as mma.sync items
    (cc_mma) or with window pairs on CTA pairs (pair)."""
    import torch
    import tca_spmm
    if args.only == "fwd_bwd":
        return fwd_bwd_leg(args, False)
    if args.only == "batching":
        return batching_leg(args, world)
    distinct = make_problems(args)
    if args.only == "e2e":
        c = distinct[0]
        t0 = time.perf_counter()
        for _ in range(args.warmup + args.steps):
            tca_spmm.spmm_host(c["row_ptr"], c["col"], c["vals"], c["K"], c["B"],
                               C=np.empty((c["M"], args.n), np.float16), keep_empty_rows=False)
        return {"s": time.perf_counter() - t0}
    dev = torch.device("cuda", torch.cuda.current_device())
    if args.only in ("csr", "f64"):
        c = distinct[0]
        rp, ci = (torch.from_numpy(c[k]).to(dev) for k in ("row_ptr", "col"))
        if args.only == "csr":
            v, B = (torch.from_numpy(c[k]).to(dev) for k in ("vals", "B"))
            C = torch.empty((c["M"], args.n), dtype=torch.float16, device=dev)
            fn = lambda: tca_spmm.spmm_csr(rp, ci, v, B, K=c["K"], out=C)  # noqa: E731
        else:
            v = torch.from_numpy(c["vals"].astype(np.float64)).to(dev)
            B = torch.from_numpy(c["B"].astype(np.float64)).to(dev)
            C = torch.empty((c["M"], args.n), dtype=torch.float64, device=dev)
            fn = lambda: tca_spmm.spmm_csr_f64(rp, ci, v, B, K=c["K"], out=C)  # noqa: E731
        for _ in range(args.warmup + args.steps):
            fn()
        torch.cuda.synchronize()
        return {"problems": 1}
    plans, Bs, Cs = [], [], []
    for g in range(args.problems):
        c = distinct[g % len(distinct)]
        rp, ci, v, B = (torch.from_numpy(c[k]).to(dev) for k in ("row_ptr", "col", "vals", "B"))
        plans.append(tca_spmm.Plan(rp, ci, v, c["K"], pair_windows=args.only == "pair"))
        Bs.append(B)
        Cs.append(torch.empty((c["M"], args.n), dtype=torch.float16, device=dev))
    g = tca_spmm.BatchGraph(plans, Bs, Cs, precision="e4m3" if args.only == "step_e4m3" else "f16",
                            cc_cols=[tca_spmm.CC_COLS_MMA] * len(plans) if args.only == "cc_mma" else None)
    for _ in range(args.warmup + args.steps):
        g.launch()
    torch.cuda.synchronize()
    g.close()
    return {"problems": args.problems}


def kernel_times(tca_spmm, torch, plans, Bs, Cs, precision, reps):
    """(tensor-core ms, CUDA-core ms) per replay of the batch captured in a
    CUDA graph with events around each kernel group."""
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for e in ev:  # torch reads only events it has recorded itself once
        e.record()
    torch.cuda.synchronize()
    g = tca_spmm.BatchGraph(plans, Bs, Cs, precision=precision, events=ev)
    tc, cc = [], []
    for _ in range(reps):
        g.launch()
        torch.cuda.synchronize()
        tc.append(ev[0].elapsed_time(ev[1]))
        cc.append(ev[2].elapsed_time(ev[3]))
    g.close()
    return tc, cc


def graph_of(torch, fn):
    """fn (launches on torch's current stream) captured once as a CUDA graph."""
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
        fn()
    return g


def batching_leg(args, world):
    """The batching config: 24 layers of mixed shapes, sparsity and N. Device
    time per pass (CUDA events, median of runs) of: the autotuned batch
    (tca_spmm_batched, one CUDA graph); the same batch with one configuration
    for every layer (N slice 128, 8 CUDA-core columns a lane: the fewest
    launches); and 24 sequential forwards (tca_spmm per layer), both eager and
    captured as one CUDA graph of the 24 calls. Roofline: compulsory bytes of
    the 24 layers over the batch's time."""
    import torch
    import tca_spmm
    from tca_spmm import gen
    dev = torch.device("cuda", torch.cuda.current_device())
    ls = gen.batch_layers()
    plans, Bs, outs = [], [], []
    for c in ls:
        rp, ci, v = (torch.from_numpy(x.copy()).to(dev) for x in (c["row_ptr"], c["col"], c["vals"]))
        plans.append(tca_spmm.Plan(rp, ci, v, c["K"]))
        Bs.append(torch.from_numpy(c["B"].copy()).to(dev))
        outs.append(torch.empty((c["M"], c["N"]), dtype=torch.float16, device=dev))
    flops = sum(2.0 * c["col"].size * c["N"] for c in ls)
    nbytes = sum(problem_bytes(c, c["N"]) for c in ls)
    tuned = tca_spmm.autotune(plans, Bs, outs, reps=3)
    g = tca_spmm.BatchGraph(plans, Bs, outs, n_tiles=[t[0] for t in tuned], cc_cols=[t[1] for t in tuned])
    g1 = tca_spmm.BatchGraph(plans, Bs, outs, n_tiles=[128] * len(ls), cc_cols=[8] * len(ls))

    def seq():
        for p, B, C in zip(plans, Bs, outs):
            p.spmm(B, out=C)

    gseq = graph_of(torch, seq)

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) * 1e3)
        return float(np.median(ts))

    t_graph, t_one = timed(g.launch), timed(g1.launch)
    t_seq_graph, t_seq = timed(gseq.replay), timed(seq)
    g.close()
    g1.close()
    peak, _ = peaks()

    def launches(n_tiles, cc_cols):
        """(tensor-core, CUDA-core) launches of one batched call."""
        tc = {nt for p, nt in zip(plans, n_tiles) if p.info()["n_tc_windows"] > 0}
        cc = {w for p, w in zip(plans, cc_cols) if p.info()["n_cc_windows"] > 0}
        return len(tc), len(cc)

    return {"workload": "24 layers: 6 each of 512x2048, 2048x512, 512x512, 1024x4096; sparsity U[0.5, 0.98]; "
                        "N per layer from {64..1024}; FP16",
            "graph_us": round(t_graph, 2), "sequential_graph_us": round(t_seq_graph, 2),
            "sequential_eager_us": round(t_seq, 2), "one_config_graph_us": round(t_one, 2),
            "speedup_vs_sequential_graph": round(t_seq_graph / t_graph, 3),
            "speedup_vs_sequential_eager": round(t_seq / t_graph, 3),
            "launches": {"tuned": launches([t[0] for t in tuned], [t[1] for t in tuned]),
                         "one_config": launches([128] * len(ls), [8] * len(ls)),
                         "sequential": sum(sum(p.launch_counts(c["N"])) for p, c in zip(plans, ls))},
            "graph_gflops": round(flops / (t_graph * 1e-6) / 1e9, 1),
            "roofline_frac": round(nbytes / (t_graph * 1e-6) / 1e9 / peak, 4),
            "compulsory_bytes": nbytes,
            "tuned": [list(t) for t in tuned]}


# (sparsity, N) of the per-problem comparison: the sweep matrix 4096 x 1024
# (Zipf(1.2) rows) across the sparsities and widths the forward target names
PER_PROBLEM = [(0.70, 256), (0.80, 256), (0.90, 256), (0.95, 256), (0.98, 256), (0.80, 64), (0.80, 128),
               (0.80, 512)]


def time_hot_cold(torch, fn, flush, n_graph=100, reps=10, cold_reps=20):
    """Per-call device time of fn (one forward issued on torch's current
    stream), the same way for every implementation: hot = a CUDA graph of
    n_graph back-to-back calls, median over reps replays, divided by n_graph;
    cold = a graph of one call replayed after writing a buffer larger than L2,
    median over cold_reps replays. Falls back to the same loops without a graph
    when fn cannot be captured."""
    s = torch.cuda.Stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    with torch.cuda.stream(s):
        for _ in range(3):
            fn()
    torch.cuda.synchronize()
    method = "cuda graph"
    try:
        g, g1 = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
            for _ in range(n_graph):
                fn()
        with torch.cuda.graph(g1, stream=s, capture_error_mode="relaxed"):
            fn()
        run_n, run_1 = g.replay, g1.replay
    except Exception:  # noqa: BLE001 -- not capturable: time the plain launches
        torch.cuda.synchronize()
        method = "stream loop (not capturable)"

        def run_n():
            for _ in range(n_graph):
                fn()
        run_1 = fn
    hot, cold = [], []
    with torch.cuda.stream(s):
        run_n()
        for _ in range(reps):
            a, b = ev(), ev()
            a.record()
            run_n()
            b.record()
            b.synchronize()
            hot.append(a.elapsed_time(b) * 1e3 / n_graph)
        for _ in range(cold_reps):
            flush.zero_()
            a, b = ev(), ev()
            a.record()
            run_1()
            b.record()
            b.synchronize()
            cold.append(a.elapsed_time(b) * 1e3)
    torch.cuda.synchronize()
    return float(np.median(hot)), float(np.median(cold)), method


def per_problem_leg(args, check):
    """One problem per call, at every point of the forward target: this
    project's forward (FP16 C, the configuration's output, and FP32 C, the
    comparators' output), the reference's TCA kernel with its own schedule and
    the reference comparator's cuSPARSE call, all on the same device buffers
    in this process and timed the same way (time_hot_cold). With `check`,
    every output's relative Frobenius error against the FP64 oracle."""
    import torch
    import tca_spmm
    from tca_spmm import gen
    from oracle import oracle
    dev = torch.device("cuda", torch.cuda.current_device())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MB > 126 MB L2
    have_ref = oracle.ref_available()
    peak, _ = peaks()
    rows = []
    for sp, N in PER_PROBLEM:
        c = gen.sweep(sp, N=N, seed=7000)
        M, K, nnz = c["M"], c["K"], int(c["col"].size)
        rp, ci, v, B = (torch.from_numpy(np.ascontiguousarray(x)).to(dev)
                        for x in (c["row_ptr"], c["col"], c["vals"], c["B"]))
        plan = tca_spmm.Plan(rp, ci, v, K)
        outs = {"ours_f16": torch.empty((M, N), dtype=torch.float16, device=dev),
                "ours_f32": torch.empty((M, N), dtype=torch.float32, device=dev),
                "reference_tca": torch.zeros((M, N), dtype=torch.float32, device=dev),
                "cusparse": torch.zeros((M, N), dtype=torch.float32, device=dev)}
        fns = {"ours_f16": lambda: plan.spmm(B, out=outs["ours_f16"]),
               "ours_f32": lambda: plan.spmm(B, out=outs["ours_f32"])}
        closers = []
        if have_ref:
            tk = oracle.RefTcaKernel(M, N, K, c["row_ptr"], v.data_ptr(), rp.data_ptr(), ci.data_ptr(),
                                     B.data_ptr(), outs["reference_tca"].data_ptr())
            cs = oracle.RefCusparse(M, N, K, nnz, rp.data_ptr(), ci.data_ptr(), v.data_ptr(), B.data_ptr(),
                                    outs["cusparse"].data_ptr())
            closers += [tk, cs]
            fns["reference_tca"] = lambda: tk.launch(torch.cuda.current_stream().cuda_stream)
            fns["cusparse"] = lambda: cs.launch(torch.cuda.current_stream().cuda_stream)
        flops = 2.0 * nnz * N
        bytes16 = nnz * 6 + (M + 1) * 4 + K * N * 2 + M * N * 2
        row = {"sparsity": sp, "N": N, "nnz": nnz, "us": {}, "cold_us": {}, "timing": {}}
        for name, fn in fns.items():
            hot, cold, method = time_hot_cold(torch, fn, flush)
            row["us"][name], row["cold_us"][name], row["timing"][name] = round(hot, 3), round(cold, 3), method
        t = row["us"]["ours_f16"]
        row["gflops_ours_f16"] = round(flops / (t * 1e-6) / 1e9, 1)
        row["roofline_frac_ours_f16"] = round(bytes16 / (t * 1e-6) / 1e9 / peak, 4)
        row["roofline_frac_ours_f16_cold"] = round(bytes16 / (row["cold_us"]["ours_f16"] * 1e-6) / 1e9 / peak, 4)
        if have_ref:
            for ref_name in ("reference_tca", "cusparse"):
                row[f"speedup_vs_{ref_name}"] = round(row["us"][ref_name] / t, 3)
                row[f"speedup_vs_{ref_name}_cold"] = round(row["cold_us"][ref_name] / row["cold_us"]["ours_f16"], 3)
                row[f"speedup_f32_vs_{ref_name}"] = round(row["us"][ref_name] / row["us"]["ours_f32"], 3)
        if check:
            torch.cuda.synchronize()
            ref = oracle.spmm_f64(c["row_ptr"], c["col"], c["vals"], c["B"])
            nrm = np.linalg.norm(ref)
            row["rel_err_vs_f64"] = {k: float(f"{np.linalg.norm(o.double().cpu().numpy() - ref) / nrm:.3e}")
                                     for k, o in outs.items() if k in fns}
        for x in closers:
            x.close()
        plan.close()
        rows.append(row)
    return {"workload": "one 4096x1024 Zipf(1.2) problem per call (seed 7000), B U(-1,1)",
            "method": "per-call device time: hot = CUDA graph of 100 back-to-back calls (median of 10 replays "
                      "/ 100); cold = one call per replay after a 256 MB write (median of 20); the same "
                      "for every implementation, on the same device buffers",
            "impls": {"ours_f16": "tca_spmm, FP16 C", "ours_f32": "tca_spmm, FP32 C",
                      "reference_tca": "kernel_our_spmm_balanced<64> with workload_manager's schedule "
                                       "(reference sources, sm_100a), FP32 C",
                      "cusparse": "cusparseSpMM CSR ALG_DEFAULT with the reference comparator's parameters, "
                                  "FP32 C"},
            "target": "ours_f16 >= 1.5x both reference_tca and cusparse at >= 0.60 of the HBM roofline",
            "rows": rows}


def fwd_bwd_leg(args, check):
    """The differentiation config (A 2048 x 512 at 90 %, B 512 x 4096, dY
    2048 x 4096): forward alone vs forward + backward (dA = SDDMM(dY, B) on
    A's pattern, dB = A^T dY), device time per pass (CUDA events, median of
    runs), and with `check` the gradients' error against FP64."""
    import torch
    import tca_spmm
    from tca_spmm import gen
    dev = torch.device("cuda", torch.cuda.current_device())
    c = gen.diff()
    rp, ci, v = (torch.from_numpy(x.copy()).to(dev) for x in (c["row_ptr"], c["col"], c["vals"]))
    B = torch.from_numpy(c["B"]).to(dev)
    dY = torch.from_numpy(c["dY"]).to(dev)
    plan = tca_spmm.Plan(rp, ci, v, c["K"])
    Y = torch.empty((c["M"], c["N"]), dtype=torch.float16, device=dev)
    dA = torch.empty(c["col"].size, dtype=torch.float32, device=dev)
    dB = torch.empty((c["K"], c["N"]), dtype=torch.float32, device=dev)

    def fwd():
        plan.spmm(B, out=Y)

    def fwd_bwd():
        plan.spmm(B, out=Y)
        plan.sddmm(dY, B, out=dA)
        plan.spmm_t(dY, out=dB)

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) * 1e3)
        return float(np.median(ts))

    t_f, t_fb = timed(fwd), timed(fwd_bwd)
    flops = 2.0 * c["col"].size * c["N"]
    out = {"workload": "A 2048x512 90% (uniform rows), B 512x4096, dY 2048x4096, FP16 in, FP32 dA/dB",
           "fwd_us": round(t_f, 2), "fwd_bwd_us": round(t_fb, 2), "fwd_bwd_over_fwd": round(t_fb / t_f, 3),
           "fwd_gflops": round(flops / (t_f * 1e-6) / 1e9, 1),
           "fwd_bwd_gflops": round(3 * flops / (t_fb * 1e-6) / 1e9, 1)}
    if check:
        rows = np.repeat(np.arange(c["M"]), np.diff(c["row_ptr"]))
        B64, Y64 = c["B"].astype(np.float64), c["dY"].astype(np.float64)
        dA64 = np.einsum("jn,jn->j", Y64[rows], B64[c["col"]])
        dB64 = np.zeros_like(B64)
        np.add.at(dB64, c["col"], c["vals"].astype(np.float64)[:, None] * Y64[rows])
        out["dA_rel_err_vs_f64"] = float(f"{np.linalg.norm(dA.cpu().numpy() - dA64) / np.linalg.norm(dA64):.3e}")
        out["dB_rel_err_vs_f64"] = float(f"{np.linalg.norm(dB.cpu().numpy() - dB64) / np.linalg.norm(dB64):.3e}")
    return out


def run_reference(args, world, rank):
    import torch
    from oracle import oracle
    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libtcaref.so was not built (reference tree absent at build time)"}, None
    distinct = make_problems(args)
    n_iter = max(1, args.steps)
    ms_kernel, flops, wall = [], 0.0, 0.0
    sp_ms = []
    with oracle.quiet_stdout():
        oracle.ref_our_spmm_balanced(distinct[0]["row_ptr"], distinct[0]["col"], distinct[0]["vals"], 1024,
                                     distinct[0]["B"], n_iter=1)
        for c in distinct:
            t0 = time.perf_counter()
            _, ms = oracle.ref_our_spmm_balanced(c["row_ptr"], c["col"], c["vals"], c["K"], c["B"], n_iter=1)
            wall += time.perf_counter() - t0
            _, ms = oracle.ref_our_spmm_balanced(c["row_ptr"], c["col"], c["vals"], c["K"], c["B"], n_iter=n_iter)
            ms_kernel.append(ms)
            flops += 2.0 * c["col"].size * args.n
            A = oracle.csr_to_dense(c["M"], c["K"], c["row_ptr"], c["col"], c["vals"])
            _, ms_sp = oracle.ref_cusparse_spmm(A, c["B"], n_iter=n_iter)
            sp_ms.append(ms_sp)
    gpu_value = flops / (sum(ms_kernel) * 1e-3) / 1e9
    gpu_e2e = flops / wall / 1e9
    h2d = sum(c["row_ptr"].nbytes + c["col"].nbytes + c["vals"].nbytes + c["B"].nbytes + c["M"] * args.n * 4
              for c in distinct) // len(distinct)
    d2h = distinct[0]["M"] * args.n * 4

    # The arm proper: the reference's own CPU implementation of C = A B,
    # naive_gemm (src/miscalleneous.cu:114-134: dense FP32-accumulate GEMM,
    # OpenMP over the rows, all host threads), on the first problem of the
    # workload, counted by the metric's useful flops 2 nnz N. A step is the
    # whole problem when warm-up + steps fit in REF_BUDGET_S seconds; else
    # every r-th row (the sample keeps the skewed row lengths), r as small as
    # the budget allows.
    c = distinct[0]
    A_full = oracle.csr_to_dense(c["M"], c["K"], c["row_ptr"], c["col"], c["vals"])
    cores = len(os.sched_getaffinity(0))
    oracle.ref_naive_gemm(A_full, c["B"])  # warm-up (thread pool, pages)
    t0 = time.perf_counter()
    oracle.ref_naive_gemm(A_full, c["B"])
    t_full = time.perf_counter() - t0
    stride = max(1, int(np.ceil((args.steps + args.warmup) * t_full / REF_BUDGET_S)))
    rows = np.arange(0, c["M"], stride)
    A_s = A_full[rows] if stride > 1 else A_full
    nnz_s = int(np.diff(c["row_ptr"])[rows].sum())
    for _ in range(max(1, args.warmup)):
        oracle.ref_naive_gemm(A_s, c["B"])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.ref_naive_gemm(A_s, c["B"])
    el = time.perf_counter() - t0
    value = 2.0 * nnz_s * args.n * args.steps / el / 1e9
    if stride == 1:
        sample = (f"naive_gemm on the whole {c['M']}x{c['K']} problem (nnz {nnz_s}, N={args.n}) per step, "
                  f"{args.steps} steps in {el:.1f} s")
    else:
        sample = (f"naive_gemm on rows 0, {stride}, .. of one {c['M']}x{c['K']} problem ({rows.size} rows, "
                  f"nnz {nnz_s}, N={args.n}) per step, {args.steps} steps in {el:.1f} s (the whole problem "
                  f"takes {t_full:.2f} s: {args.steps + args.warmup} of them exceed {REF_BUDGET_S:.0f} s)")
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(el / args.steps * 1e3, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16",
        "data": "synthetic (seeded numpy PCG64)",
        "config": {"workload": WORKLOAD, "N": args.n, "sample": sample, "same_config": stride == 1},
        "reference_impl": "naive_gemm (the reference's CPU implementation of the product) from the unmodified "
                          "reference sources in oracle/_ref/libtcaref.so, on the host cores",
        "cpu_baseline": {"value": round(value, 3), "unit": "GFLOP/s", "cores": cores, "kind": "reference",
                         "cpu_model": cpu_model(), "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": {
            "value": round(gpu_value, 3), "unit": "GFLOP/s", "problems": len(distinct),
            "impl": "our_spmm_balanced (TCA kernel, mma.sync) from the unmodified reference sources, compiled "
                    "for sm_100a into oracle/_ref/libtcaref.so; run through its host API",
            "timing": "the reference's own event timing of n_iter back-to-back launches per call "
                      "(src/our_spmm.cu:552-574), hot L2; FP32 output",
            "e2e": {"value": round(gpu_e2e, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "path": "our_spmm_balanced(n_iter=1), wall clock"},
            "cusparse": {"value": round(flops / (sum(sp_ms) * 1e-3) / 1e9, 3), "unit": "GFLOP/s",
                         "impl": "perform_cuSPARSE_SpMM (reference comparator, cusparseSpMM CSR ALG_DEFAULT)"}},
    }
    return out, distinct


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        if rank != 0:
            return
        out, _ = run_reference(args, 1, 0)
        print(json.dumps(out), flush=True)
        return
    if args.only is not None:
        print(json.dumps({"only": args.only, **run_only(args, world)}), flush=True)
        return
    out, distinct = run_ours(args, world, rank)
    if rank == 0:
        if world == 1 and not args.no_cpu:
            out["cpu_baseline"] = cpu_baseline(distinct[0], args.cpu_seconds)
        else:
            out["cpu_baseline"] = None
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
