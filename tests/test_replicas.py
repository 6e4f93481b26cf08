"""The N > 1 plumbing of bench.py on CPU: two gloo ranks (world size 2) that
run the same barrier / max-over-ranks / whole-job-rate steps as the GPU ranks
do over NCCL, a rank that dies between steps (the other gets an error from its
next collective instead of waiting for good), and the reference arm's ranks
other than 0, which do no work."""
import multiprocessing as mp
import os
import socket
import sys
import time

import pytest

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, mode: str, q) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    try:
        from set_intersection_b200.replicas import Replicas
        rep = Replicas("gloo", timeout_s=8.0)
        rep.barrier()
        if mode == "die" and rank == 1:
            os._exit(3)  # leaves between steps, with no collective in flight
        t0 = time.time()
        try:
            ms = rep.max(10.0 * (rank + 1))
            q.put((rank, "ok", ms, rep.rate(1000, ms), rep.world, time.time() - t0))
        except Exception as e:  # the collective ended with an error
            q.put((rank, "error", type(e).__name__, 0.0, rep.world, time.time() - t0))
        rep.close()
    except Exception as e:
        q.put((rank, "setup-error", repr(e)[:200], 0.0, 0, 0.0))


def _run(world: int, mode: str, timeout: float = 120.0):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    deadline = time.time() + timeout
    for p in procs:
        p.join(max(1.0, deadline - time.time()))
    for p in procs:
        if p.is_alive():
            p.kill()
    out = {}
    while not q.empty():
        r = q.get()
        out[r[0]] = r[1:]
    return out, [p.exitcode for p in procs]


def test_two_gloo_ranks_time_the_job_by_the_slowest_rank():
    out, codes = _run(2, "ok")
    assert codes == [0, 0], (codes, out)
    for rank in (0, 1):
        status, ms, rate, world, _ = out[rank]
        assert status == "ok" and world == 2
        assert ms == 20.0  # every rank sees the slowest rank's time
        assert rate == pytest.approx(2 * 1000 / 20e-3)  # the units of both ranks over that time


def test_a_rank_that_dies_ends_the_others_next_collective_with_an_error():
    out, codes = _run(2, "die")
    assert codes[1] == 3
    status, what, _, _, waited = out[0]
    assert status == "error", out
    assert waited < 60.0


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    from set_intersection_b200.replicas import Replicas
    env = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE") if k in os.environ}
    try:
        rep = Replicas("gloo")
        assert rep.world == 1 and not rep.active
        rep.barrier()
        assert rep.max(4.5) == 4.5
        assert rep.rate(10, 2.0) == pytest.approx(5000.0)
        rep.close()
    finally:
        os.environ.update(env)


def test_reference_arm_ranks_above_zero_do_no_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    called = []
    monkeypatch.setattr(bench, "ref_sisi_measure", lambda *a, **k: called.append(a))
    monkeypatch.setattr(bench, "ref_pair", lambda *a, **k: called.append(a))

    class Args:
        workload, steps, warmup, gpus = "sisi_large", 3, 3, 2

    t0 = time.time()
    assert bench.run_reference_arm(Args, rank=1) is None
    assert not called and time.time() - t0 < 1.0
