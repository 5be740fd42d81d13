"""The bounds-checked build (lib/checked/libgk_cuda.so, GK_CHECKED) on the
small parity cases: every path's cell, face, stage-row and TMA-row
coordinates stay inside their arrays (gk_checked_report counts none), and the
results are the normal build's bits -- the learned correction included, in
the fused stage and as the generic path's pass.  The checked build runs in a child
process (GK_CHECKED=1 selects it when the library loads)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import ctypes, dataclasses, json, sys
import numpy as np
sys.path.insert(0, ROOT)
from gaukuk_b200 import _lib, problems
from gaukuk_b200.config import Params
from gaukuk_b200.sim import Sim
from gaukuk_b200.ensemble import Ensemble
from gaukuk_b200.slabs import Slabs
out = {}
def run(name, p, c, **kw):
    with Sim(p, c, mode=kw.get("mode", "parity")) as s:
        s.run(p.tmax, p.dtoutput)
        out[name] = (s.download(), s.dt_log(), s.path)
p, c = problems.kh(150, ny=130, seed=2)
run("fused2d", dataclasses.replace(p, stepmax=12), c)
run("fused2d_fast", dataclasses.replace(p, stepmax=12), c, mode="fast")
p, c = problems.rt(32, 96)
run("rt_rk3", dataclasses.replace(p, stepmax=10), c)
p = Params(nx=20, ny=16, nz=12, bc=(3, 2, 0, 1, 2, 3), integrator=2, tmax=1.0, dtoutput=1.0,
           stepmax=6)
run("stage3d", p, problems.random_smooth(p, seed=7, with_vz=True))
p, c = problems.sod(128)
run("generic1d", dataclasses.replace(p, stepmax=20), c)
p = Params(nx=24, ny=20, nz=1, integrator=3, tmax=1.0, dtoutput=1.0, stepmax=8)
run("generic2d_vz", p, problems.random_smooth(p, seed=4, with_vz=True))
inst = [problems.kh(n, seed=i) for i, n in enumerate((48, 64, 40))]
sims = [Sim(dataclasses.replace(q, tmax=0.02, dtoutput=0.02), d) for q, d in inst]
Ensemble(sims).run_steps(6)
for i, s in enumerate(sims):
    out["ens%d" % i] = (s.download(), s.dt_log(), s.path)
from gaukuk_b200 import learned
rng = np.random.default_rng(5)
blob = learned.init_model(rng.normal(size=(256, 16)).astype(np.float32),
                          (0.1 * rng.normal(size=(256, 4))).astype(np.float32), seed=2)
blob[learned.NPARAM + 36:] *= 1e-3
p, c = problems.kh(150, ny=70, seed=6)
for fused in (True, False):
    with Sim(dataclasses.replace(p, stepmax=6), c) as s:
        learned.install(s, blob, fused=fused, diss_frac=0.25)
        s.set_tiling(128, 5)
        s.run(p.tmax, p.dtoutput)
        out["learned_fused" if fused else "learned_pass"] = (s.download(), s.dt_log(), s.path)
p, c = problems.kh(96, ny=90, seed=3)
p = dataclasses.replace(p, stepmax=10)
with Slabs(p, c, 3) as s:
    s.run(p.tmax, p.dtoutput)
    out["slabs"] = (s.download(), s.dt_log(), "slabs")
cnt, first = ctypes.c_ulonglong(), ctypes.c_ulonglong()
rc = _lib.load().gk_checked_report(ctypes.byref(cnt), ctypes.byref(first))
np.savez(OUT, **{k: v[0] for k, v in out.items()})
print(json.dumps({"rc": rc, "count": cnt.value, "first": first.value,
                  "dts": {k: v[1] for k, v in out.items()},
                  "paths": {k: v[2] for k, v in out.items()}}))
'''


def _child(checked, tmp_path):
    out = str(tmp_path / ("checked.npz" if checked else "plain.npz"))
    code = CHILD.replace("ROOT", repr(ROOT)).replace("OUT", repr(out))
    env = dict(os.environ, GK_CHECKED="1" if checked else "0")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(out)


def test_checked_build_finds_no_stray_index_and_keeps_the_bits(tmp_path):
    if not os.path.exists(os.path.join(ROOT, "gaukuk_b200", "lib", "checked", "libgk_cuda.so")):
        pytest.skip("the checked build is not here")
    chk, a = _child(True, tmp_path)
    plain, b = _child(False, tmp_path)
    assert chk["rc"] == 0, chk  # the checked library answered
    assert plain["rc"] == -4    # the normal build has no counters
    assert chk["count"] == 0, f"first stray coordinate: {chk['first']:#x}"
    assert chk["paths"] == plain["paths"]
    assert {"fused2d", "stage3d", "generic"} <= set(chk["paths"].values())
    assert chk["paths"]["learned_fused"] == "fused2d" and chk["paths"]["learned_pass"] == "generic"
    assert np.array_equal(a["learned_fused"], a["learned_pass"])
    for k in b.files:
        if k == "fused2d_fast":
            # fast mode: the checks may change the compiler's FMA contraction
            np.testing.assert_allclose(chk["dts"][k], plain["dts"][k], rtol=1e-12)
            np.testing.assert_allclose(a[k], b[k], rtol=0, atol=1e-12 * np.abs(b[k]).max())
        else:
            assert chk["dts"][k] == plain["dts"][k], k
            assert np.array_equal(a[k], b[k]), k
