"""The multi-GPU replica logic on CPU: two gloo ranks as separate processes
(127.0.0.1), the barrier around a timed region, the maximum over ranks and
the whole-job rate; and a rank that leaves before the collective makes its
peer fail within the process-group timeout instead of hanging."""
import multiprocessing as mp
import os
import socket
import time

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    try:
        from gaukuk_b200.replicas import Replicas
        reps = Replicas("gloo", timeout_s=5.0)
        if mode == "leave" and rank == 1:
            q.put((rank, "left"))
            q.close()
            q.join_thread()  # the message is out before the process goes
            os._exit(0)  # leaves between steps, with nothing in flight
        reps.barrier()
        t0 = time.perf_counter()
        time.sleep(0.05 * (rank + 1))  # the timed work of this replica
        reps.barrier()
        secs = time.perf_counter() - t0
        worst = reps.max(secs)
        rate = reps.rate(1000.0, secs)
        total = reps.sum(10.0 * (rank + 1))  # per-rank units that differ
        q.put((rank, (secs, worst, rate, reps.is_root, total)))
        reps.close()
    except Exception as e:  # reported to the test
        q.put((rank, "error: " + type(e).__name__))


def _run(mode, world=2, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    deadline = time.time() + timeout
    while len(out) < world and time.time() < deadline:
        try:
            r, v = q.get(timeout=max(0.1, deadline - time.time()))
            out[r] = v
        except Exception:
            break
    for p in procs:
        p.join(timeout=10)
        if p.is_alive():
            p.kill()
    return out


def test_two_replicas_time_the_slowest_rank():
    out = _run("ok")
    assert set(out) == {0, 1}, out
    (s0, w0, r0, root0, n0), (s1, w1, r1, root1, n1) = out[0], out[1]
    assert n0 == n1 == 30.0
    # the barrier after the work makes both ranks wait for the slower one
    assert w0 == w1 == pytest.approx(max(s0, s1))
    assert w0 >= 0.1 - 1e-3
    assert r0 == r1 == pytest.approx(2 * 1000.0 / w0)
    assert root0 and not root1


def test_a_rank_that_leaves_makes_its_peer_fail_not_hang():
    t0 = time.time()
    out = _run("leave", timeout=60)
    assert out.get(1) == "left"
    assert isinstance(out.get(0), str) and out[0].startswith("error"), out
    assert time.time() - t0 < 45
