"""Generates the golden vectors in this folder from the reference itself.

Each case runs oracle/_ref/ref_strict -- the reference's own sources, built by
oracle/Makefile with strict IEEE flags -- on an initial state from
gaukuk_b200.problems, and stores the parameters, the initial state, the final
active cells and the full-precision dt log.  Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py
"""
import dataclasses
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from gaukuk_b200 import problems  # noqa: E402
from gaukuk_b200.config import Params  # noqa: E402
from gk_oracle import run_reference  # noqa: E402


def cases():
    p, c = problems.kh(32)
    yield "kh32_rk2", dataclasses.replace(p, stepmax=40), c
    p, c = problems.kh(24, ny=20, integrator=3, rc_order=1)
    yield "kh24x20_rk3_rc1", dataclasses.replace(p, stepmax=25), c
    p, c = problems.kh(20, ny=18, integrator=1, cfl=0.3)
    p = dataclasses.replace(p, bc=(3, 3, 2, 2, 1, 1), stepmax=30)
    yield "kh20x18_euler_outflow_reflect", p, c
    p, c = problems.sod(128, tmax=0.2)
    yield "sod128_outflow", p, c
    p, c = problems.sod(64, bc=0, tmax=0.1)
    yield "sod64_copy", p, c
    p, c = problems.rt(16, 48)
    yield "rt16x48_rk3_gravity", dataclasses.replace(p, stepmax=30), c
    p = Params(nx=10, ny=8, nz=6, bc=(1, 1, 2, 3, 0, 1), integrator=3, tmax=1.0, dtoutput=1.0,
               stepmax=8)
    yield "box10x8x6_rk3", p, problems.random_smooth(p, seed=5, with_vz=True)


def active(p, c):
    g = p.ng
    return c[:, g:g + p.nz, g:g + p.ny, g:g + p.nx]


def main():
    index = {}
    for name, p, c in cases():
        out, dts, stats = run_reference(p, c, flavour="strict", threads=1)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), ic=active(p, c),
                            final=active(p, out), dts=np.array(dts))
        index[name] = {"params": dataclasses.asdict(p), "steps": len(dts), "t": stats["t"]}
        print(name, len(dts), stats["t"])
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
