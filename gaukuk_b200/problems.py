"""Initial conditions for the benchmark problems, in the reference layout.

Every generator returns ``(params, cons)`` where ``cons`` is a float64 array of
shape ``(5, lenz, leny, lenx)`` -- the TArray layout of ``Sim::cons``
(template_array.hpp:67-72, sim.cpp:49) -- with the active cells filled and the
ghosts zero, exactly what a reference setup hook leaves behind after
``eos.PrimToCons`` (adiabatic.cpp:162-198): ghost primitives are zero, so ghost
conserved values are zero too.

Cell centres follow Domain (sim.cpp:39-41):
``xc(i) = xmin - nGhost*dx + 0.5*dx + i*dx``.  The constant ``PI`` is the
reference's truncated value (gaukuk.hpp:19).
"""
from __future__ import annotations

import numpy as np

from .config import Params, BC_OUTFLOW, BC_PERIODIC, BC_REFLECTIVE

PI = 3.1415926535  # gaukuk.hpp:19

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea & Flood 2014), vectorised over uint64."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def uniform_pm1(seed: int, ids: np.ndarray) -> np.ndarray:
    """Counter-based U(-1, 1): one draw per global cell id, independent of tiling."""
    with np.errstate(over="ignore"):
        key = np.uint64(seed) * np.uint64(0xD1B54A32D192ED03) & _M64
        bits = splitmix64((ids.astype(np.uint64) ^ key) & _M64)
    u01 = (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u01 - 1.0


def cell_centres(p: Params):
    dx = (p.xmax - p.xmin) / p.nx
    dy = (p.ymax - p.ymin) / p.ny
    dz = (p.zmax - p.zmin) / p.nz
    xc = p.xmin - p.ng * dx + 0.5 * dx + np.arange(p.lenx, dtype=np.float64) * dx
    yc = p.ymin - p.ng * dy + 0.5 * dy + np.arange(p.leny, dtype=np.float64) * dy
    zc = p.zmin - p.ng * dz + 0.5 * dz + np.arange(p.lenz, dtype=np.float64) * dz
    return xc, yc, zc


def prim_to_cons(p: Params, rho, vx, vy, vz, pre) -> np.ndarray:
    """EquationOfState::PrimToCons (adiabatic.cpp:162-198) on the active cells;
    arguments are arrays of shape (nz, ny, nx)."""
    gm1rec = 1.0 / (p.gamma - 1.0)
    cons = np.zeros(p.shape, dtype=np.float64)
    a = (slice(p.ng, p.ng + p.nz), slice(p.ng, p.ng + p.ny), slice(p.ng, p.ng + p.nx))
    cons[(0,) + a] = rho
    cons[(1,) + a] = rho * vx
    cons[(2,) + a] = rho * vy
    cons[(3,) + a] = rho * vz
    cons[(4,) + a] = pre * gm1rec + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return cons


def _active_grids(p: Params):
    xc, yc, zc = cell_centres(p)
    x = xc[p.ng:p.ng + p.nx][None, None, :]
    y = yc[p.ng:p.ng + p.ny][None, :, None]
    z = zc[p.ng:p.ng + p.nz][:, None, None]
    shp = (p.nz, p.ny, p.nx)
    return (np.broadcast_to(x, shp), np.broadcast_to(y, shp), np.broadcast_to(z, shp))


def sod(n: int = 256, x0: float = 0.5, integrator: int = 2, cfl: float = 0.4,
        bc: int = BC_OUTFLOW, tmax: float = 0.2, **kw):
    """1D Sod shock tube on x in [0,1]: (1, 0, 1) left of x0, (0.125, 0, 0.1) right.
    y and z extents are 1 so that drmin = dx (sim.cpp:35)."""
    p = Params(nx=n, ny=1, nz=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
               gamma=1.4, cfl=cfl, integrator=integrator, rc_order=2,
               bc=(bc, bc, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC),
               tmax=tmax, dtoutput=tmax, **kw)
    x, _, _ = _active_grids(p)
    left = x < x0
    rho = np.where(left, 1.0, 0.125)
    pre = np.where(left, 1.0, 0.1)
    z = np.zeros_like(rho)
    return p, prim_to_cons(p, rho, z, z, z, pre)


def kh(n: int = 256, ny: int = None, seed: int = 0, rho_in: float = 2.0, rho_out: float = 1.0,
       half_width: float = 0.25, amp: float = 0.01, noise: float = 1e-3, pressure: float = 2.5,
       integrator: int = 2, cfl: float = 0.4, tmax: float = 2.0, rc_order: int = 2,
       smooth: float = 0.0, **kw):
    """2D Kelvin-Helmholtz on [0,1]^2, periodic: rho_in and vx=-0.5 where
    |y-0.5| < half_width, else rho_out and vx=+0.5; p uniform;
    vy = amp*sin(4*pi*x) + noise*U(-1,1) with U keyed on (seed, global cell id).
    With smooth > 0 the two shear layers are tanh profiles of that thickness,
    s(y) = (tanh((y - y1)/smooth) - tanh((y - y2)/smooth))/2 with
    y1,2 = 0.5 -+ half_width, rho = rho_out + (rho_in - rho_out) s, vx = 0.5 - s."""
    ny = n if ny is None else ny
    p = Params(nx=n, ny=ny, nz=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
               gamma=1.4, cfl=cfl, integrator=integrator, rc_order=rc_order,
               bc=(BC_PERIODIC,) * 6, tmax=tmax, dtoutput=tmax, **kw)
    x, y, _ = _active_grids(p)
    if smooth > 0.0:
        sh = 0.5 * (np.tanh((y - (0.5 - half_width)) / smooth) - np.tanh((y - (0.5 + half_width)) / smooth))
        rho = rho_out + (rho_in - rho_out) * sh
        vx = 0.5 - sh
    else:
        inside = np.abs(y - 0.5) < half_width
        rho = np.where(inside, rho_in, rho_out)
        vx = np.where(inside, -0.5, 0.5)
    ids = np.arange(p.nx * p.ny, dtype=np.uint64).reshape(1, p.ny, p.nx)
    vy = amp * np.sin(4.0 * PI * x) + noise * uniform_pm1(seed, ids)
    pre = np.full_like(rho, pressure)
    return p, prim_to_cons(p, rho, vx, vy, np.zeros_like(rho), pre)


def rt(nx: int = 1024, ny: int = 3072, g: float = -0.1, rho_up: float = 2.0,
       rho_down: float = 1.0, amp: float = 0.01, p0: float = 2.5, nx_ptb: float = 2.0,
       ny_ptb: float = 4.5, integrator: int = 3, cfl: float = 0.4, tmax: float = 5.0, **kw):
    """2D Rayleigh-Taylor on [-0.25,0.25]x[-0.75,0.75]: x periodic, y reflective,
    constant gravity g in y.  rho_up for y>0 else rho_down, p = p0 + g*rho*y,
    vy = amp*(1+cos(kx x))(1+cos(ky y))/4 with kx = nx_ptb*pi/Lx, ky = ny_ptb*pi/Ly
    (the shape of setup_rt.cpp:28-55 with p0 in place of 1/gamma)."""
    p = Params(nx=nx, ny=ny, nz=1, xmin=-0.25, xmax=0.25, ymin=-0.75, ymax=0.75,
               zmin=-0.5, zmax=0.5, gamma=1.4, cfl=cfl, integrator=integrator, rc_order=2,
               bc=(BC_PERIODIC, BC_PERIODIC, BC_REFLECTIVE, BC_REFLECTIVE, BC_PERIODIC, BC_PERIODIC),
               grav=(0.0, g, 0.0), tmax=tmax, dtoutput=tmax, **kw)
    x, y, _ = _active_grids(p)
    lx, ly = p.xmax - p.xmin, p.ymax - p.ymin
    kx, ky = nx_ptb * PI / lx, ny_ptb * PI / ly
    rho = np.where(y > 0.0, rho_up, rho_down)
    vy = amp * ((1.0 + np.cos(kx * x)) * (1.0 + np.cos(ky * y)) / 4.0)
    pre = p0 + g * rho * y
    z = np.zeros_like(rho)
    return p, prim_to_cons(p, rho, z, vy, z, pre)


def random_smooth(p: Params, seed: int = 0, with_vz: bool = False):
    """A smooth random state for unit parity tests: positive density and
    pressure, a few Fourier modes per field, on any grid shape."""
    rng = np.random.default_rng(seed)
    x, y, z = _active_grids(p)

    def field(base, ampl):
        f = np.full(x.shape, base)
        for _ in range(3):
            kx, ky, kz = rng.integers(1, 4, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            a = rng.uniform(-ampl, ampl)
            f = f + a * np.sin(2 * np.pi * kx * x + ph[0]) * np.cos(2 * np.pi * ky * y + ph[1]) \
                * np.cos(2 * np.pi * kz * z + ph[2])
        return f

    rho = field(1.5, 0.4)
    vx, vy = field(0.0, 0.5), field(0.0, 0.5)
    vz = field(0.0, 0.5) if with_vz else np.zeros_like(rho)
    pre = field(2.0, 0.5)
    if p.ny == 1:
        vy = np.zeros_like(rho) if not with_vz else vy
    return prim_to_cons(p, rho, vx, vy, vz, pre)


def kh_ensemble(n: int = 64, seed: int = 0, sizes=(128, 256, 512), tmax: float = 1.0, **kw):
    """Ensemble of independent KH problems.  Per instance, drawn from a seeded
    generator: grid size from `sizes`, density ratio U[1.5, 4] (rho_out = 1,
    rho_in = ratio), shear-layer half-width U[0.2, 0.3], perturbation
    amplitude U[0.005, 0.02]; periodic, PLM, HLLC, RK2.  Returns a list of
    (params, cons, draw) with the draws recorded."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = int(sizes[rng.integers(0, len(sizes))])
        draw = {"size": size, "ratio": float(rng.uniform(1.5, 4.0)),
                "half_width": float(rng.uniform(0.2, 0.3)), "amp": float(rng.uniform(0.005, 0.02))}
        p, c = kh(size, seed=seed * 1000 + i, rho_in=draw["ratio"], rho_out=1.0,
                  half_width=draw["half_width"], amp=draw["amp"], tmax=tmax, **kw)
        out.append((p, c, draw))
    return out
