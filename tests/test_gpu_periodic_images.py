"""Periodic ghost images written by the fused 2D stage (Phys::periodic_images).

On a grid periodic on all four x/y sides with at most 2^21 cells, no gravity,
host routine, fixed side, inner reset or immersed body, the stage stores every
edge cell's value also into the ghost cells the periodic fill (periodic.cpp)
would copy it to, and the steps launch no ghost fill.  Against the same run
with the images off (GK_PERIODIC_IMAGES=0 at upload, one ghost fill per
stage): the state, ghosts included, and the dt sequence bit for bit, in both
modes and after a host upload whose ghosts are stale."""
import dataclasses
import os

import pytest

from gaukuk_b200 import problems
from gaukuk_b200.config import BC_OUTFLOW, BC_PERIODIC

pytestmark = pytest.mark.gpu


class _Env:
    def __init__(self, value):
        self.value = value

    def __enter__(self):
        self.old = os.environ.get("GK_PERIODIC_IMAGES")
        os.environ["GK_PERIODIC_IMAGES"] = self.value

    def __exit__(self, *a):
        if self.old is None:
            del os.environ["GK_PERIODIC_IMAGES"]
        else:
            os.environ["GK_PERIODIC_IMAGES"] = self.old


def _launches(s):
    return s.graph_info()[1]


def _run(p, c, mode, images, steps, reupload=False):
    from gaukuk_b200.sim import Sim
    with _Env("1" if images else "0"):
        with Sim(p, c, mode=mode) as s:
            assert s.path == "fused2d"
            launches = _launches(s)
            s.run_steps(steps)
            if reupload:
                # a host edit of one active cell, with every ghost strip of the
                # evolved variables overwritten by values no fill would write
                u = s.download()
                u[0, ..., 40, 40] *= 1.01
                for v in (0, 1, 2, 4):
                    u[v, ..., :2, :] = 1e3
                    u[v, ..., -2:, :] = 1e3
                    u[v, ..., :, :2] = 1e3
                    u[v, ..., :, -2:] = 1e3
                s.upload(u)
                s.run_steps(steps)
            return s.download(), s.dt_log(), launches


@pytest.mark.parametrize("mode,integrator", [("parity", 2), ("fast", 2), ("parity", 3), ("fast", 3)])
def test_images_give_the_fill_paths_bits(mode, integrator):
    p, c = problems.kh(256, integrator=integrator)
    a, da, la = _run(p, c, mode, True, 40)
    b, db, lb = _run(p, c, mode, False, 40)
    stages = integrator
    assert la == stages and lb == 2 * stages  # the stage alone, or ghost fill + stage
    assert da == db and len(da) == 40
    assert a.tobytes() == b.tobytes()  # signed zeros too


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_images_refill_stale_ghosts_after_an_upload(mode):
    p, c = problems.kh(192, ny=160)
    a, da, _ = _run(p, c, mode, True, 25, reupload=True)
    b, db, _ = _run(p, c, mode, False, 25, reupload=True)
    assert da == db and len(da) == 25  # an upload restarts the dt log
    assert a.tobytes() == b.tobytes()


def test_images_only_on_small_all_periodic_grids():
    from gaukuk_b200.sim import Sim

    def launches(p, c):
        with _Env("1"):
            with Sim(p, c, mode="fast") as s:
                return _launches(s)

    # 1448^2 = 2,096,704 cells: at most 2^21, images on; 1449^2 past it
    assert launches(*problems.kh(1448)) == 2
    assert launches(*problems.kh(1449)) == 4
    # a y side that is not periodic keeps the fills
    p, c = problems.kh(256)
    p = dataclasses.replace(p, bc=(BC_PERIODIC,) * 2 + (BC_OUTFLOW,) * 2 + (BC_PERIODIC,) * 2)
    assert launches(p, c) == 4
    # gravity keeps them too (the kick sits between the fill and the stage)
    p, c = problems.rt(128, 384)
    assert launches(p, c) == 1 + 2 * 3
