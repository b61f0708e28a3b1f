"""Failure of a rank in the sharded SpMM (tca_spmm.shard), on the CPU with two
`gloo` ranks in separate processes. The failures are made on the host, never
on a GPU: one rank leaves between steps (it exits after joining, before the
step's collective), or never joins at all. The surviving rank must not wait
for good: with a short process-group timeout its next collective -- the dB
all-reduce of the row sharding, reduce_grad_b -- or its join ends with an
error, which the test reads back together with how long it took."""
import datetime
import os
import socket
import time

import pytest

from tca_spmm import shard

torch = pytest.importorskip("torch")

PG_TIMEOUT_S = 5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    if rank == 1 and mode == "never_joins":
        return
    t0 = time.monotonic()
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=PG_TIMEOUT_S))
    except Exception as e:  # noqa: BLE001 -- the outcome under test
        q.put((rank, "join_error", type(e).__name__, time.monotonic() - t0))
        return
    if rank == 1 and mode == "leaves":
        os._exit(0)  # between steps: joined, no collective in flight
    partial = torch.ones((64, 16), dtype=torch.float64)
    t0 = time.monotonic()
    try:
        shard.reduce_grad_b(partial)
        q.put((rank, "ok", "", time.monotonic() - t0))
    except Exception as e:  # noqa: BLE001 -- the outcome under test
        q.put((rank, "error", type(e).__name__, time.monotonic() - t0))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001 -- the group may be broken already
            pass


def _run(mode):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = []
    deadline = time.monotonic() + 20 * PG_TIMEOUT_S
    try:
        while time.monotonic() < deadline and not any(r[0] == 0 for r in results):
            try:
                results.append(q.get(timeout=1.0))
            except Exception:  # noqa: BLE001 -- queue.Empty: keep waiting
                pass
    finally:
        for p in procs:
            p.join(timeout=30)
        for p in procs:
            if p.is_alive():  # the exact child this test started
                p.kill()
                p.join()
    return [r for r in results if r[0] == 0]


def test_rank_leaving_between_steps_ends_the_next_collective_with_an_error():
    got = _run("leaves")
    assert got, "rank 0 never reported: its collective did not end"
    _, outcome, kind, elapsed = got[0]
    assert outcome == "error", got
    assert elapsed < 10 * PG_TIMEOUT_S, got


def test_rank_never_joining_ends_the_join_with_an_error():
    got = _run("never_joins")
    assert got, "rank 0 never reported: its join did not end"
    _, outcome, kind, elapsed = got[0]
    assert outcome == "join_error", got
    assert elapsed < 10 * PG_TIMEOUT_S, got


def test_healthy_ranks_complete_the_collective():
    got = _run("healthy")
    assert got and got[0][1] == "ok", got
    assert got[0][3] < 10 * PG_TIMEOUT_S, got
