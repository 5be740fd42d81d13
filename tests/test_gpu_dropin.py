"""The drop-in boundary end to end: the same .in file and problem hook run by
the reference build (oracle/_ref, strict IEEE flags) and by this package's
gaukuk_<hook>.sim, whose Sim::Advance runs on the GPU in parity mode.  Every
cons_XXXXX frame must be byte-identical (header, mesh, every cell including
ghosts), and the per-step log lines must agree."""
import os
import subprocess

import numpy as np
import pytest

from gaukuk_b200.config import Params

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "gaukuk_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")


def _run(exe, args, cwd):
    r = subprocess.run([exe] + args, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


def _steps(text):
    return [l for l in text.splitlines() if l.startswith("step = ")]


CASES = {
    "kh_baseline": (Params(nx=96, ny=64, tmax=0.05, dtoutput=0.02, cfl=0.4, integrator=2,
                           rc_order=2, bc=(1, 1, 1, 1, 1, 1)), {"seed": 3}),
    "rt_baseline": (Params(nx=32, ny=96, xmin=-0.25, xmax=0.25, ymin=-0.75, ymax=0.75,
                           zmin=-0.5, zmax=0.5, tmax=0.3, dtoutput=0.1, cfl=0.4, integrator=3,
                           rc_order=2, bc=(1, 1, 2, 2, 1, 1)),
                    {"gravAccY": -0.1, "p0": 2.5, "ny_ptb": 4.5, "rhoUp": 2.0, "rhoDown": 1.0,
                     "amp": 0.01}),
    "kh_outflow_rc1": (Params(nx=40, ny=50, tmax=0.04, dtoutput=0.02, cfl=0.4, integrator=2,
                              rc_order=1, bc=(3, 3, 2, 0, 1, 1)), {"seed": 1}),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_frames_byte_identical_to_reference(name, tmp_path):
    hook = "kh_baseline" if name.startswith("kh") else name
    ref_exe = os.path.join(REF, f"ref_strict_{hook}")
    if not os.path.exists(ref_exe):
        pytest.skip("reference build absent")
    p, extra = CASES[name]
    text = p.to_in_text(extra)
    a, b = tmp_path / "ref", tmp_path / "gpu"
    a.mkdir(); b.mkdir()
    (a / "run.in").write_text(text)
    (b / "run.in").write_text(text)
    out_ref = _run(ref_exe, ["-i", "run.in", "--frames"], a)
    out_gpu = _run(os.path.join(BIN, f"gaukuk_{hook}.sim"), ["-i", "run.in"], b)
    frames = sorted(f for f in os.listdir(a) if f.startswith("cons_"))
    assert len(frames) >= 3 and frames == sorted(f for f in os.listdir(b) if f.startswith("cons_"))
    for f in frames:
        x, y = (a / f).read_bytes(), (b / f).read_bytes()
        assert x == y, f"{f} differs"
    # same step count; the reference's lines carry 17 digits here (driver),
    # ours the stream's default precision, so compare the parsed numbers
    sr, sg = _steps(out_ref), _steps(out_gpu)
    assert len(sr) == len(sg) > 0
    for lr, lg in zip(sr, sg):
        nr = [float(v.split("=")[1]) for v in lr.split(",")]
        ng = [float(v.split("=")[1]) for v in lg.split(",")]
        assert nr[0] == ng[0]
        np.testing.assert_allclose(nr[1:], ng[1:], rtol=1e-5)


@pytest.mark.parametrize("hook", ["kh_baseline", "rt_baseline"])
def test_restart_continues_bit_identically(hook, tmp_path):
    """A run resumed from its own frame cons_00002 (input key restart = 2)
    writes frames 3, 4, ... byte-identical to those of the uninterrupted run:
    a frame holds the exact time and state, and the step is a function of
    them alone."""
    name = "kh_baseline" if hook == "kh_baseline" else "rt_baseline"
    p, extra = CASES[name]
    exe = os.path.join(BIN, f"gaukuk_{hook}.sim")
    a, b = tmp_path / "full", tmp_path / "resumed"
    a.mkdir(); b.mkdir()
    (a / "run.in").write_text(p.to_in_text(extra))
    _run(exe, ["-i", "run.in"], a)
    (b / "cons_00002").write_bytes((a / "cons_00002").read_bytes())
    (b / "run.in").write_text(p.to_in_text(dict(extra, restart=2)))
    _run(exe, ["-i", "run.in"], b)
    later = sorted(f for f in os.listdir(a) if f.startswith("cons_") and f > "cons_00002")
    assert later and later == sorted(f for f in os.listdir(b) if f.startswith("cons_") and f > "cons_00002")
    for f in later:
        assert (a / f).read_bytes() == (b / f).read_bytes(), f


def test_immersed_table_is_checked_and_switches_the_path():
    """gk_set_immersed takes the reference's shell table; a cell outside the
    active region is refused (the kernel indexes with it), a body sends a 2D
    run to the generic path, and without it the next upload (which checks
    MTZ again) brings the fused path back."""
    from gaukuk_b200 import problems
    from gaukuk_b200._lib import GkError
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(32, seed=4)
    g = p.ng
    ids = np.zeros((3, 1, 9), dtype=np.int32)
    ids[:, 0, 0] = (g + 10, g + 10, g)    # the shell cell (i, j, k)
    ids[:, 0, 1] = (g + 14, g + 10, g)    # one target, outside the body
    direction = np.array([[1.0], [0.0], [0.0], [1.0]])
    w = np.zeros((1, 9))
    w[0, :2] = (0.8, 0.2)
    with Sim(p, c, mode="parity") as s:
        assert s.path == "fused2d"
        bad = ids.copy()
        bad[0, 0, 1] = 1                  # a ghost column
        with pytest.raises(GkError) as e:
            s.set_immersed(bad, [1], direction, w)
        assert e.value.code == -1
        s.set_immersed(ids, [1], direction, w)
        assert s.path == "generic"
        s.run_steps(2)
        a = s.download()
        assert np.isfinite(a).all()
        s.set_immersed(None)
        s.upload(c)
        assert s.path == "fused2d"


def test_zero_z_momentum_plane_stays_on_the_host():
    """A 2D state whose z-momentum plane is +0.0 everywhere uploads four
    planes; a planes-only download on the fused path leaves that plane in the
    caller's array, and the full download returns it as zeros.  A plane with
    one non-zero ghost value is copied both ways (the run still takes the
    fused path: only active cells decide that)."""
    from gaukuk_b200 import problems
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(48, seed=2)
    plane = p.lenx * p.leny * 8
    k = p.ng
    with Sim(p, c, mode="parity") as s:
        up, _ = s.io_bytes()
        assert up == 4 * plane and s.path == "fused2d"
        s.run_steps(2)
        out = np.full(p.shape, 7.0)
        s.download(out, planes_only=True)
        assert (out[3, k] == 7.0).all()           # left as it was
        full = s.download()
        assert (full[3, k] == 0.0).all()
        np.testing.assert_array_equal(out[[0, 1, 2, 4], k], full[[0, 1, 2, 4], k])
        _, down = s.io_bytes()
        strips = 5 * 2 * p.ng * (p.nx + p.ny) * 8  # ghost strips from the stage buffer
        assert down == 5 * plane + strips
    c2 = c.copy()
    c2[3, k, 0, 0] = 1.0                          # a corner ghost
    with Sim(p, c2, mode="parity") as s:
        up, _ = s.io_bytes()
        assert up == 5 * plane and s.path == "fused2d"
        out = np.full(p.shape, 7.0)
        s.download(out, planes_only=True)
        assert out[3, k, 0, 0] == 1.0 and out[3, k, p.ng, p.ng] == 0.0


def test_metrics_log_matches_the_run(tmp_path):
    """With metrics = 1 the driver appends one JSON line per output interval:
    the steps add up to the run's, t is the frame time, the dt range brackets
    the printed steps' dt, and a smooth KH run repairs no cell."""
    import json
    p, extra = CASES["kh_baseline"]
    (tmp_path / "run.in").write_text(p.to_in_text(dict(extra, metrics=1)))
    out = _run(os.path.join(BIN, "gaukuk_kh_baseline.sim"), ["-i", "run.in"], tmp_path)
    recs = [json.loads(l) for l in (tmp_path / "metrics.jsonl").read_text().splitlines()]
    steps = _steps(out)
    dts = [float(l.split("dt =")[1]) for l in steps]
    assert [r["output"] for r in recs] == list(range(1, len(recs) + 1)) and len(recs) >= 3
    assert sum(r["steps"] for r in recs) == len(steps) == recs[-1]["step"]
    assert abs(recs[-1]["t"] - p.tmax) < 1e-12
    for r in recs:
        assert r["zone_updates_per_s"] > 0 and r["floor_density"] == r["floor_pressure"] == 0
        assert r["dt_min"] <= r["dt_max"]
    assert min(r["dt_min"] for r in recs) <= min(dts) * (1 + 1e-5)
    assert max(r["dt_max"] for r in recs) >= max(dts) * (1 - 1e-5)
