"""The reference's frame format (cons_XXXXX) and restarts on the host side:
the Python reader/writer against frames the reference build itself writes,
and the C++ driver reading a frame back (restart = N) without a GPU."""
import os
import subprocess

import numpy as np
import pytest

from gaukuk_b200 import frames, problems
from gaukuk_b200.config import Params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
BIN = os.path.join(ROOT, "gaukuk_b200", "bin")
KH = (Params(nx=48, ny=32, tmax=0.02, dtoutput=0.01, cfl=0.4, integrator=2, rc_order=2,
             bc=(1, 1, 1, 1, 1, 1)), {"seed": 3})


def test_frame_round_trip(tmp_path):
    p, c = problems.kh(24, ny=16, seed=2)
    path = str(tmp_path / "cons_00007")
    frames.write_frame(path, p, 0.125, c)
    fr = frames.read_frame(path)
    assert fr.t == 0.125 and (fr.nvar, fr.nx, fr.ny, fr.nz, fr.ng) == (5, 24, 16, 1, p.ng)
    assert np.array_equal(fr.data, c)
    xc, yc, zc = frames.cell_centres(p)
    assert np.array_equal(fr.xc, xc) and np.array_equal(fr.yc, yc) and np.array_equal(fr.zc, zc)


def test_frames_match_the_reference_writer(tmp_path):
    """A frame the reference build writes (Sim::WriteData) reads back, and
    writing it again gives the same bytes (header, mesh and data)."""
    exe = os.path.join(REF, "ref_strict_kh_baseline")
    if not os.path.exists(exe):
        pytest.skip("reference build absent")
    p, extra = KH
    (tmp_path / "run.in").write_text(p.to_in_text(extra))
    r = subprocess.run([exe, "-i", "run.in", "--frames", "--quiet"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-1000:]
    for name in ("cons_00000", "cons_00002"):
        raw = (tmp_path / name).read_bytes()
        fr = frames.read_frame(str(tmp_path / name))
        out = tmp_path / ("again_" + name)
        frames.write_frame(str(out), p, fr.t, fr.data)
        assert out.read_bytes() == raw, name
    assert abs(frames.read_frame(str(tmp_path / "cons_00002")).t - 0.02) < 1e-12


def test_driver_reads_a_frame_back(tmp_path):
    """gaukuk_<hook>.sim with `restart = 1` loads cons_00001 (time and state)
    and, with tmax at that time, stops without a step -- no GPU needed --
    while a frame of another grid is refused."""
    exe = os.path.join(BIN, "gaukuk_kh_baseline.sim")
    if not os.path.exists(exe):
        pytest.skip("host layer not built")
    p, extra = KH
    c = problems.kh(p.nx, ny=p.ny, seed=3)[1]
    frames.write_frame(str(tmp_path / "cons_00001"), p, 0.02, c)
    (tmp_path / "run.in").write_text(p.to_in_text(dict(extra, restart=1)))
    r = subprocess.run([exe, "-i", "run.in"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr[-1000:]
    assert "total steps =      0" in r.stdout
    assert not (tmp_path / "cons_00000").exists() and not (tmp_path / "cons_00002").exists()
    q = Params(nx=p.nx + 2, ny=p.ny, tmax=0.02, dtoutput=0.01, bc=p.bc)
    (tmp_path / "bad.in").write_text(q.to_in_text(dict(extra, restart=1)))
    r = subprocess.run([exe, "-i", "bad.in"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode != 0 and "grid differs" in r.stderr
