"""One grid split into y-slabs equals the undivided grid bit for bit.

The slabs run in one process on one GPU (gk_slabs_create: ghost rows
exchanged by a copy kernel between stages, the CFL maximum taken over all
slabs before each step's epilogue), and as one slab of a one-process NCCL
job (gk_slabs_create_nccl: the exchange is NCCL send/recv to itself around
the periodic ring, the maximum an NCCL all-reduce).  Compared with the same
problem run as one handle: the whole state (ghost rows included) and the dt
sequence, in parity mode and in fast mode (the slabs run the same kernels
as the undivided grid) -- bit for bit in parity mode; in fast mode within the
fast-mode tolerance, since the compiler may contract a tile's first row
(its prologue) differently from the rows after it, and the slabs' tiles
start at other rows than the whole grid's.
"""
import dataclasses

import numpy as np
import pytest

from gaukuk_b200 import problems
from gaukuk_b200.config import BC_COPY, BC_OUTFLOW, BC_PERIODIC, BC_REFLECTIVE
from helpers import active, rel_linf

pytestmark = pytest.mark.gpu


def _single(p, c, mode):
    from gaukuk_b200.sim import Sim
    with Sim(p, c, mode=mode) as s:
        s.run(p.tmax, p.dtoutput)
        return s.download(), s.dt_log()


def _case(name):
    if name == "kh_periodic":
        p, c = problems.kh(160, ny=150, seed=3)
        return dataclasses.replace(p, tmax=0.2, dtoutput=0.05, stepmax=40), c
    if name == "rt_rk3_gravity":
        p, c = problems.rt(64, 192)
        return dataclasses.replace(p, tmax=0.5, dtoutput=0.25, stepmax=30), c
    if name == "kh_outflow_copy":
        p, c = problems.kh(96, ny=130, seed=5)
        p = dataclasses.replace(p, bc=(BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_COPY,
                                       BC_PERIODIC, BC_PERIODIC))
        return dataclasses.replace(p, tmax=0.2, dtoutput=0.2, stepmax=25), c
    raise KeyError(name)


@pytest.mark.parametrize("mode", ["parity", "fast"])
@pytest.mark.parametrize("case,nslab", [("kh_periodic", 1), ("kh_periodic", 2),
                                        ("kh_periodic", 5), ("rt_rk3_gravity", 3),
                                        ("kh_outflow_copy", 4)])
def test_slabs_equal_the_whole_grid(case, nslab, mode):
    from gaukuk_b200.slabs import Slabs
    p, c = _case(case)
    want, want_dts = _single(p, c, mode)
    with Slabs(p, c, nslab, mode=mode) as s:
        info = s.info()
        assert info["local_slabs"] == nslab
        s.run(p.tmax, p.dtoutput)
        got = s.download()
        dts = s.dt_log()
    assert len(dts) == len(want_dts) > 0
    if mode == "parity":
        assert dts == want_dts
        assert np.array_equal(got, want)
    else:
        np.testing.assert_allclose(dts, want_dts, rtol=1e-12)
        errs = rel_linf(active(p, got), active(p, want))
        assert max(errs[v] for v in (0, 1, 2, 4)) <= 1e-12, errs


def test_slabs_refuse_what_the_fused_stage_does_not_run():
    from gaukuk_b200._lib import GkError
    from gaukuk_b200.slabs import Slabs
    p, c = problems.kh(64, seed=1)
    with pytest.raises(GkError):
        Slabs(dataclasses.replace(p, integrator=1), c, 2)  # forward Euler updates in place
    with pytest.raises(GkError):
        Slabs(p, c, 40)  # slabs of one row
    q = dataclasses.replace(p, bc=(1, 1, 1, 2, 1, 1))
    with pytest.raises(GkError):
        Slabs(q, c, 2)  # a periodic side without a periodic partner


def test_one_rank_nccl_ring_equals_the_whole_grid():
    """The NCCL exchange path on one GPU: a one-rank job whose single slab
    under periodic y sends its edge rows to itself and all-reduces its own
    CFL speed."""
    import datetime
    import socket

    import torch.distributed as dist

    from gaukuk_b200.slabs import DistSlabs
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    store = dist.TCPStore("127.0.0.1", port, 1, True, timeout=datetime.timedelta(seconds=30))
    dist.init_process_group("gloo", store=store, rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=30))
    try:
        p, c = _case("kh_periodic")
        want, want_dts = _single(p, c, "parity")
        with DistSlabs(p, c, dist, mode="parity") as s:
            s.run(p.tmax, p.dtoutput)
            got = s.download()
            dts = s.dt_log()
        assert dts == want_dts
        assert np.array_equal(got, want)
    finally:
        dist.destroy_process_group()
