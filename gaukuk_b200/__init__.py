"""gaukuk_b200 -- the finite-volume update of Gaukuk (ShunqH/Gaukuk) on B200.

The hot path (Sim::Advance and everything under it) runs as hand-written
sm_100a kernels in lib/libgk_cuda.so behind the C ABI of include/gaukuk_cuda.h.
The C++ host layer in src/ keeps the reference's classes and problem hooks;
this Python package binds the same C ABI for tests and benchmarks.
"""
from .config import Params, load_in, parse_in_text  # noqa: F401
from . import problems  # noqa: F401


def Sim(*args, **kwargs):  # noqa: N802 - mirrors the reference class name
    from .sim import Sim as _Sim
    return _Sim(*args, **kwargs)
