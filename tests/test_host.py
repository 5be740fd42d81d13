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


_C_SCALARS = {"int": ("i", 4), "unsigned": ("u", 4), "unsigned int": ("u", 4),
              "long long": ("i", 8), "unsigned long long": ("u", 8), "size_t": ("u", 8),
              "float": ("f", 4), "double": ("f", 8), "void": "void"}


def _c_class(decl):
    """One parameter (or 'return-type name') of a C prototype: 'ptr' for data
    and function pointers, else (kind, bytes)."""
    words = decl.replace("*", " * ").replace("const", " ").split()
    if "*" in words or words[0].endswith("_fn"):
        return "ptr"
    return _C_SCALARS.get(" ".join(words[:-1]), "?" + decl)


def _py_class(t):
    import ctypes
    if t is None:
        return "void"
    if t in (ctypes.c_void_p, ctypes.c_char_p) or issubclass(t, (ctypes._Pointer, ctypes._CFuncPtr)):
        return "ptr"
    kind = {"i": "i", "l": "i", "q": "i", "I": "u", "L": "u", "Q": "u", "f": "f", "d": "f"}[t._type_]
    return kind, ctypes.sizeof(t)


def test_cabi_signatures_match_the_header():
    """Each prototype in include/gaukuk_cuda.h against the ctypes signature the
    Python binding declares: parameter count, pointer or scalar, and each
    scalar's kind and width."""
    from gaukuk_b200 import _lib
    with open(os.path.join(ROOT, "include", "gaukuk_cuda.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    protos = re.findall(r"([A-Za-z_][\w \t*]*?)\b(gk_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S)
    seen = set()
    for ret, name, params in protos:
        params = " ".join(params.split())
        want_args = [] if params in ("", "void") else [_c_class(q) for q in params.split(",")]
        want_ret = _c_class(ret.strip() + " f")
        rt, at = _lib.SIGNATURES[name]
        assert [_py_class(a) for a in at] == want_args, name
        assert _py_class(rt) == want_ret, name
        seen.add(name)
    assert seen == set(_lib.SIGNATURES)
