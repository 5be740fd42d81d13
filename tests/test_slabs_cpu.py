"""Host logic of the y-slab split, on CPU (no device needed).

* The decomposition itself, run by two gloo ranks on the oracle: each rank
  advances its slab with the y ghost rows between slabs exchanged over gloo
  after every stage's ghost fill and the CFL maximum all-reduced every step;
  the slabs together are the undivided grid's bits, dt sequence included.

* The partition: every active row belongs to exactly one slab, the first
  ny % n slabs take one row more, neighbours form a chain (a ring under
  periodic y; a single periodic slab is its own neighbour).
* Two gloo ranks as separate processes (127.0.0.1): rank 0 makes the
  128-byte NCCL id, both ranks end up with the same bytes, and both compute
  the same layout of the whole grid, each knowing its own slab's rows and
  its neighbour ranks -- the information every rank needs before the first
  NCCL exchange, which must pair sends and receives between the right ranks.
"""
import multiprocessing as mp
import os
import socket
import time

import pytest


def test_partition_covers_every_row_once():
    from gaukuk_b200.slabs import layout
    for ny in (2, 7, 100, 4096, 3072):
        for n in (1, 2, 3, 5, 8):
            if ny // n < 2:
                continue
            for periodic in (False, True):
                rows = []
                for k in range(n):
                    j0, cnt, lo, up = layout(ny, n, k, periodic)
                    assert cnt in (ny // n, ny // n + 1) and cnt >= 2
                    rows.extend(range(j0, j0 + cnt))
                    assert lo == (k - 1 if k > 0 else (n - 1 if periodic else -1))
                    assert up == (k + 1 if k < n - 1 else (0 if periodic else -1))
                assert rows == list(range(ny))
                firsts = [layout(ny, n, k, periodic)[1] for k in range(n)]
                assert firsts == sorted(firsts, reverse=True)  # the extra rows go first


def _run_plans(n, periodic):
    """Match every rank's planned NCCL calls as NCCL pairs point-to-point
    operations (the k-th send from a to b meets the k-th receive on b from
    a) and return, per rank, which rows each receive delivered:
    {rank: {"lower": (src rank, "top"|"bottom"), "upper": ...}}."""
    from gaukuk_b200.slabs import exchange_plan
    sends, recvs = {}, {}
    for k in range(n):
        for kind, peer in exchange_plan(n, k, periodic):
            if kind in (0, 2):
                sends.setdefault((k, peer), []).append("top" if kind == 0 else "bottom")
            else:
                recvs.setdefault((peer, k), []).append("lower" if kind == 1 else "upper")
    got = {k: {} for k in range(n)}
    assert sorted(sends) == sorted(recvs)  # every send has a receive and back
    for (a, b), rows in sends.items():
        targets = recvs[(a, b)]
        assert len(rows) == len(targets)
        for r, t in zip(rows, targets):
            got[b][t] = (a, r)
    return got


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 8])
def test_nccl_exchange_plan_delivers_the_right_rows(n, periodic):
    """Each slab's lower ghost rows must come from its lower neighbour's top
    rows and its upper ghosts from its upper neighbour's bottom rows (a
    ring under periodic y; none at the grid's own sides), for the calls in
    the order the library makes them."""
    if n == 1 and not periodic:
        from gaukuk_b200.slabs import exchange_plan
        assert exchange_plan(1, 0, False) == []
        return
    got = _run_plans(n, periodic)
    for k in range(n):
        lower = k - 1 if k > 0 else (n - 1 if periodic else None)
        upper = k + 1 if k < n - 1 else (0 if periodic else None)
        if lower is None:
            assert "lower" not in got[k]
        else:
            assert got[k]["lower"] == (lower, "top"), (k, got[k])
        if upper is None:
            assert "upper" not in got[k]
        else:
            assert got[k]["upper"] == (upper, "bottom"), (k, got[k])


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        import datetime

        import torch.distributed as dist

        from gaukuk_b200.slabs import layout, nccl_id_broadcast
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=10))
        nid = nccl_id_broadcast(dist, make_id=lambda: bytes(range(128)))
        mine = layout(1030, world, rank, True)
        q.put((rank, (nid, mine)))
        dist.destroy_process_group()
    except Exception as e:  # reported to the test
        q.put((rank, "error: " + type(e).__name__ + ": " + str(e)))


def test_two_ranks_agree_on_id_and_layout():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    deadline = time.time() + 60
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
    assert sorted(out) == [0, 1], out
    for r in range(world):
        assert not isinstance(out[r], str), out[r]
    assert out[0][0] == out[1][0] == bytes(range(128))
    # rank 0 owns rows 0..514, rank 1 rows 515..1029; under periodic y each
    # is the other's lower and upper neighbour
    assert out[0][1] == (0, 515, 1, 1)
    assert out[1][1] == (515, 515, 0, 0)


def _split_case(name):
    from gaukuk_b200 import problems
    if name == "kh_periodic":
        return problems.kh(24, ny=20, seed=3)
    if name == "rt_walls_rk3_gravity":
        p, c = problems.rt(16, 24)
        assert p.integrator == 3 and p.bc[2] == p.bc[3] == 2 and p.grav[1] != 0
        return p, c
    raise KeyError(name)


def _split_worker(rank, world, port, case, nsteps, q):
    """One slab on the oracle: halo rows over gloo (sends of the top rows up
    with tag 0 and of the bottom rows down with tag 1), the maximum by
    all-reduce."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        import dataclasses
        import datetime

        import numpy as np
        import torch
        import torch.distributed as dist

        import gk_oracle
        from gaukuk_b200.slabs import layout
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=30))
        p, c = _split_case(case)
        g = p.ng
        periodic = p.bc[2] == 1
        j0, cnt, lo, up = layout(p.ny, world, rank, periodic)
        dy = (p.ymax - p.ymin) / p.ny
        bc = list(p.bc)
        bc[2] = 5 if lo >= 0 else p.bc[2]
        bc[3] = 5 if up >= 0 else p.bc[3]
        ps = dataclasses.replace(p, ny=cnt, ymin=p.ymin + j0 * dy, ymax=p.ymin + (j0 + cnt) * dy,
                                 bc=tuple(bc), stepmax=-1)
        sim = gk_oracle.OracleSim(ps, np.ascontiguousarray(c[:, :, j0:j0 + cnt + 2 * g, :]))
        L = gk_oracle.lib()
        L.gko_set_spacing(sim.h, (p.xmax - p.xmin) / p.nx, dy, (p.zmax - p.zmin) / p.nz)
        kb, ib, ie = g, g, g + p.nx

        def halo(user, ptr):
            u = np.ctypeslib.as_array(ptr, shape=ps.shape)
            reqs, got = [], {}
            if up >= 0:
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(u[:, kb, cnt:cnt + g, ib:ie])),
                                       up, tag=0))
            if lo >= 0:
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(u[:, kb, g:2 * g, ib:ie])),
                                       lo, tag=1))
            if lo >= 0:
                got["lo"] = torch.empty((5, g, p.nx), dtype=torch.float64)
                reqs.append(dist.irecv(got["lo"], lo, tag=0))
            if up >= 0:
                got["up"] = torch.empty((5, g, p.nx), dtype=torch.float64)
                reqs.append(dist.irecv(got["up"], up, tag=1))
            for r in reqs:
                r.wait()
            if "lo" in got:
                u[:, kb, 0:g, ib:ie] = got["lo"].numpy()
            if "up" in got:
                u[:, kb, cnt + g:cnt + 2 * g, ib:ie] = got["up"].numpy()

        def reduce(user, local):
            t = torch.tensor([local], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())

        hf, rf = gk_oracle.HALO_FN(halo), gk_oracle.MAX_FN(reduce)
        dts = np.zeros(nsteps)
        n = L.gko_advance_split(sim.h, 1e6, nsteps, hf, rf, None, gk_oracle._dp(dts), nsteps)
        q.put((rank, (j0, cnt, n, dts.tolist(), sim.get_cons()[:, kb, g:g + cnt, ib:ie].copy())))
        dist.destroy_process_group()
    except Exception:  # reported to the test
        import traceback
        q.put((rank, "error: " + traceback.format_exc()))


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", ["kh_periodic", "rt_walls_rk3_gravity"])
def test_gloo_ranks_advance_the_split_grid_bit_for_bit(case, world):
    """Two or three slabs, one per gloo rank: a periodic ring (KH, RK2) and
    a grid whose bottom and top are reflecting walls (RT, RK3 with constant
    gravity), 10 steps, against the oracle on the undivided grid.  With
    three ranks the middle slab has different neighbours below and above,
    and the ring's slabs have unequal rows (20 = 7 + 7 + 6)."""
    import dataclasses

    import numpy as np
    gk_oracle = pytest.importorskip("gk_oracle")
    nsteps = 10
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, case, nsteps, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    deadline = time.time() + 120
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
    assert sorted(out) == list(range(world)), out
    for r in range(world):
        assert not isinstance(out[r], str), out[r]
    p, c = _split_case(case)
    whole = gk_oracle.OracleSim(dataclasses.replace(p, stepmax=nsteps), c)
    ref_dts = whole.advance(1e6)
    g = p.ng
    ref = whole.get_cons()[:, g, g:g + p.ny, g:g + p.nx]
    assert len(ref_dts) == nsteps
    got = np.concatenate([out[r][4] for r in range(world)], axis=1)
    starts = [out[r][0] for r in range(world)]
    assert starts == [sum(out[q][1] for q in range(r)) for r in range(world)]
    for r in range(world):
        assert out[r][2] == nsteps and out[r][3] == ref_dts, (r, out[r][3], ref_dts)
    assert np.array_equal(got, ref)
