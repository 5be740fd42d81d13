"""Host-side logic: .in parsing, problem generators, the C-ABI library."""
import os
import re

import numpy as np

from gaukuk_b200 import problems
from gaukuk_b200.config import Params, parse_in_text

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_in_parsing_like_config_loader():
    text = """# comment
gamma           = 1.4           # for adiabatic eos
NX=256
  xleft   1
bad line
tmax = 2.0e-1 trailing
"""
    d = parse_in_text(text)
    assert d == {"gamma": 1.4, "NX": 256.0, "xleft": 1.0, "tmax": 0.2}


def test_params_roundtrip_in_text():
    p, _ = problems.rt(8, 24)
    q = Params.from_in(parse_in_text(p.to_in_text()))
    assert q == p


def test_kh_generator_layout_and_ghosts():
    p, c = problems.kh(16, seed=0)
    assert c.shape == (5, 5, 20, 20)
    g = p.ng
    assert np.all(c[:, :g] == 0) and np.all(c[:, g + 1:] == 0)  # inactive z planes
    a = c[:, g, g:-g, g:-g]
    assert np.all(a[0] > 0) and np.all(a[3] == 0)
    mask = np.ones(c.shape[2:], bool)
    mask[g:-g, g:-g] = False
    assert np.all(c[:, g][:, mask] == 0)  # ghosts zero as after PrimToCons


def test_noise_is_counter_based():
    a = problems.uniform_pm1(7, np.arange(10, dtype=np.uint64))
    b = problems.uniform_pm1(7, np.arange(5, 10, dtype=np.uint64))
    assert np.array_equal(a[5:], b)
    assert np.all(np.abs(a) <= 1)


def _header_symbols():
    with open(os.path.join(ROOT, "include", "gaukuk_cuda.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(gk_[a-z0-9_]+)\s*\(", text)))


def test_cabi_library_exports_every_declared_symbol():
    from gaukuk_b200 import _lib
    L = _lib.load()
    syms = _header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SIGNATURES)
    assert L.gk_strerror(0) == b"ok"
