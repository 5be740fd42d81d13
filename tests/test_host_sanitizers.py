"""The C++ host layer under AddressSanitizer and UndefinedBehaviorSanitizer
(errors abort the run).  All nine of the reference's setup hooks run
through their first frame: the setup, the host ghost fill with fixed sides,
an immersed body's table and its fill, point and binary gravity enrollment,
and the frame writer.  The frames must equal the plain build's.
The probes of a hook's own boundary routine run under the sanitizers too:
one that writes outside its ghost strip is refused, and one that reads the
state gets its depth search (it then runs on the host at every ghost fill).
The probes come before any device work, so all of this runs on the CPU."""
import dataclasses
import os
import subprocess

import pytest

from gaukuk_b200 import _build_host
from gaukuk_b200.config import Params
from test_reference_setups import CASES, P3, ROOT

ENV = dict(os.environ, ASAN_OPTIONS="halt_on_error=1:detect_leaks=1",
           UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
REF_SETUP = os.path.join(_build_host.REFERENCE_SRC, "src", "setup")
NAMES = ["blast", "disk", "disk_planet", "example", "kh", "rt", "shock_tube", "solid_body",
         "wave_test"]


@pytest.fixture(scope="module")
def drivers(tmp_path_factory):
    hooks = [os.path.join(ROOT, "tests", "setups", "setup_inflow_sides.cpp")]
    hooks += [os.path.join(REF_SETUP, f"setup_{n}.cpp") for n in NAMES
              if os.path.exists(os.path.join(REF_SETUP, f"setup_{n}.cpp"))]
    out = str(tmp_path_factory.mktemp("asan"))
    exes = _build_host.build_sanitized(hooks, out)
    return {os.path.basename(e)[len("gaukuk_"):-len(".asan")]: e for e in exes}


def _run(exe, cwd):
    return subprocess.run([exe, "-i", "run.in"], cwd=cwd, capture_output=True, text=True,
                          timeout=600, env=ENV)


@pytest.mark.parametrize("name", NAMES)
def test_first_frame_is_clean_and_unchanged(name, drivers, tmp_path):
    if name not in drivers:
        pytest.skip("the reference's setup files are not here")
    p, extra = CASES[name]
    (tmp_path / "run.in").write_text(dataclasses.replace(p, tmax=0.0).to_in_text(extra))
    r = _run(drivers[name], tmp_path)
    assert r.returncode == 0 and "runtime error" not in r.stderr, r.stderr[-3000:]
    plain = tmp_path / "plain"
    plain.mkdir()
    (plain / "run.in").write_text((tmp_path / "run.in").read_text())
    exe = os.path.join(ROOT, "gaukuk_b200", "bin", f"gaukuk_ref_{name}.sim")
    subprocess.run([exe, "-i", "run.in"], cwd=plain, capture_output=True, timeout=600, check=True)
    assert (tmp_path / "cons_00000").read_bytes() == (plain / "cons_00000").read_bytes()


@pytest.mark.parametrize("variant", ["inflowWide", "inflowCopies"])
def test_side_probes_are_clean(variant, drivers, tmp_path):
    """The probes of a self-defined side: the refused one (it writes corner
    ghosts) and the depth search of one that reads the state."""
    p = Params(nx=16, ny=12, cfl=0.4, integrator=2, rc_order=2, bc=(3, 3, 3, 3, 1, 1),
               tmax=0.02, dtoutput=0.01, **P3)
    (tmp_path / "run.in").write_text(p.to_in_text({variant: 1}))
    r = _run(drivers["inflow_sides"], tmp_path)
    if variant == "inflowWide":
        assert "writes outside its ghost strip" in r.stderr, r.stderr[-3000:]
    else:
        assert "ghost strip" not in r.stderr, r.stderr[-3000:]
    # UBSan reports read "<file>:<line>:<col>: runtime error: ..." (a CUDA
    # error without a device only reads "CUDA runtime error")
    assert "AddressSanitizer" not in r.stderr and ": runtime error:" not in r.stderr, r.stderr[-3000:]
