"""Shared test helpers: golden vectors, state comparison."""
import json
import os

import numpy as np

from gaukuk_b200.config import Params

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def load_golden(name):
    idx = golden_cases()[name]
    pd = dict(idx["params"])
    pd["bc"] = tuple(pd["bc"])
    pd["grav"] = tuple(pd["grav"])
    p = Params(**pd)
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cons = np.zeros(p.shape)
    set_active(p, cons, z["ic"])
    return p, cons, z["final"], z["dts"].tolist()


def active(p, c):
    g = p.ng
    return c[:, g:g + p.nz, g:g + p.ny, g:g + p.nx]


def set_active(p, c, a):
    g = p.ng
    c[:, g:g + p.nz, g:g + p.ny, g:g + p.nx] = a


def rel_linf(a, b):
    """max|a-b| / max|b| per conserved variable (absolute where max|b| == 0)."""
    out = []
    for v in range(a.shape[0]):
        d = float(np.max(np.abs(a[v] - b[v])))
        s = float(np.max(np.abs(b[v])))
        out.append(d / s if s > 0 else d)
    return out
