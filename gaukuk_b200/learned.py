"""Learned flux correction for coarse grids (pattern 4).

A small MLP (16 -> 64 -> 64 -> 4, GELU) predicts, for every face of a coarse
grid, the difference between the flux a 4x finer run pushes through that face
(averaged over the fine faces, the RK stages and the fine steps) and the HLLC
flux of the coarse state.  The coarse solver adds the prediction to its FP64
HLLC flux at every stage (gk_set_flux_model), so the update stays conservative;
a shock / positivity detector keeps plain HLLC where it fires.

Everything that touches the grid runs in libgk_cuda.so: the fine runs (as
ensembles, gk_ens_*), the flux taps (gk_tap_substeps), the coarse HLLC fluxes (gk_face_fluxes), training
(gk_mlp_train: BF16 tensor-core forward, hand-written backward, Adam) and the
corrected coarse runs.  NumPy only assembles stencils and statistics.

Features per face (``face_features``): the 4 cells across the face, each as
(rho/rho_ref - 1, vn/c_ref, vt/c_ref, p/p_ref - 1), rho_ref and p_ref the
stencil means, c_ref = sqrt(gamma p_ref / rho_ref); targets are scaled by
rho_ref*c_ref (mass), rho_ref*c_ref^2 (momenta), rho_ref*c_ref^3 (energy).
The kernel k_flux_correct forms the same quantities on the device.

Where the correction applies (``install``): not where the detector fires,
not on faces whose stencil total variation G (``stencil_variation``) is below
tv_min, and each component at most diss_frac times the face's HLL
dissipation (``hll_dissipation``), so the corrected flux keeps part of the
scheme's own dissipation.
"""
from __future__ import annotations

import ctypes
import dataclasses
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib, problems
from .config import Params

NI, NH, NO = 16, 64, 4
NPARAM = NH * NI + NH + NH * NH + NH + NO * NH + NO
NMODEL = NPARAM + 2 * NI + 2 * NO
TV_GATE = 0.0     # default tv_min: faces with smoother stencils keep plain HLLC
DISS_FRAC = 0.25  # default diss_frac: corrections within this part of the HLL dissipation


# ------------------------------------------------------------------ grid helpers
def restrict(p: Params, cons: np.ndarray, ratio: int) -> Tuple[Params, np.ndarray]:
    """Conservative restriction of a 2D state (block means of the active cells)."""
    g = p.ng
    q = dataclasses.replace(p, nx=p.nx // ratio, ny=p.ny // ratio)
    a = cons[:, g, g:g + p.ny, g:g + p.nx]
    a = a.reshape(5, q.ny, ratio, q.nx, ratio).mean(axis=(2, 4))
    out = np.zeros(q.shape)
    out[:, q.ng, q.ng:q.ng + q.ny, q.ng:q.ng + q.nx] = a
    return q, out


def active2d(p: Params, cons: np.ndarray) -> np.ndarray:
    g = p.ng
    return cons[:, g, g:g + p.ny, g:g + p.nx]


def primitives(p: Params, a: np.ndarray):
    """ConsToPrim (adiabatic.cpp:41-57) on active cells: rho, vx, vy, p."""
    d = np.maximum(a[0], p.dfloor)
    inv = 1.0 / d
    vx, vy = a[1] * inv, a[2] * inv
    ek = 0.5 * inv * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3])
    pre = np.maximum((p.gamma - 1.0) * (a[4] - ek), p.pfloor)
    return d, vx, vy, pre


def face_features(p: Params, a: np.ndarray, direction: int):
    """Features (n, 16) and scales (n, 3) of the left (x) or lower (y) face of
    every active cell of a periodic 2D state."""
    rho, vx, vy, pre = primitives(p, a)
    ax = 1 if direction == 0 else 0
    vn, vt = (vx, vy) if direction == 0 else (vy, vx)
    st = [np.roll(f, s, axis=ax) for s in (2, 1, 0, -1)
          for f in (rho, vn, vt, pre)]  # cells -2, -1, 0, +1 relative to the face
    r = [st[4 * c + 0] for c in range(4)]
    pr = [st[4 * c + 3] for c in range(4)]
    rr = 0.25 * (r[0] + r[1] + r[2] + r[3])
    pp = 0.25 * (pr[0] + pr[1] + pr[2] + pr[3])
    cr = np.sqrt(p.gamma * pp / rr)
    feats = []
    for c in range(4):
        feats += [st[4 * c + 0] / rr - 1.0, st[4 * c + 1] / cr, st[4 * c + 2] / cr,
                  st[4 * c + 3] / pp - 1.0]
    X = np.stack([f.ravel() for f in feats], axis=1)
    S = np.stack([(rr * cr).ravel(), (rr * cr * cr).ravel(), (rr * cr ** 3).ravel()], axis=1)
    return X, S


def stencil_variation(X: np.ndarray) -> np.ndarray:
    """Total variation G of each face's stencil: the sum over the 3 pairs of
    neighbouring cells and the 4 features of |difference|."""
    X = np.asarray(X, dtype=np.float64)
    return np.abs(X[:, 4:] - X[:, :-4]).sum(axis=1)


def hll_dissipation(p: Params, a: np.ndarray, direction: int) -> np.ndarray:
    """(1/2) max(|vn| + c) |U_R - U_L| per face (n, 4: mass, normal momentum,
    tangential momentum, energy), U_L, U_R the van Leer PLM face states of
    the stencil; k_flux_correct clips the correction to diss_frac times it."""
    rho, vx, vy, pre = primitives(p, a)
    ax = 1 if direction == 0 else 0
    vn, vt = (vx, vy) if direction == 0 else (vy, vx)

    def slope(x, y):
        m = x * y
        return np.where(m > 0, 2.0 * m / np.where(m > 0, x + y, 1.0), 0.0)

    wl, wr = [], []
    for q in (rho, vn, vt, pre):
        c = [np.roll(q, s, axis=ax).ravel() for s in (2, 1, 0, -1)]
        wl.append(c[1] + 0.5 * slope(c[1] - c[0], c[2] - c[1]))
        wr.append(c[2] - 0.5 * slope(c[2] - c[1], c[3] - c[2]))

    def cons(w):
        d, u, v, pp = np.maximum(w[0], 1e-300), w[1], w[2], np.maximum(w[3], 0.0)
        return (np.stack([d, d * u, d * v, pp / (p.gamma - 1.0) + 0.5 * d * (u * u + v * v)], axis=1),
                np.abs(u) + np.sqrt(p.gamma * pp / d))

    (ul, sl), (ur, sr) = cons(wl), cons(wr)
    return 0.5 * np.maximum(sl, sr)[:, None] * np.abs(ur - ul)


def rotate_to_face(delta: np.ndarray, direction: int) -> np.ndarray:
    """(DEN, MTX, MTY, ENG) planes -> (mass, normal, tangential, energy) columns."""
    d, mx, my, e = delta
    n, t = (mx, my) if direction == 0 else (my, mx)
    return np.stack([d.ravel(), n.ravel(), t.ravel(), e.ravel()], axis=1)


# ------------------------------------------------------------------ device views
def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def face_fluxes(sim) -> Tuple[np.ndarray, np.ndarray]:
    """HLLC face fluxes of a Sim's current state: x [4][ny][nx+1], y [4][ny+1][nx]."""
    p = sim.params
    fx = np.empty((4, p.ny, p.nx + 1))
    fy = np.empty((4, p.ny + 1, p.nx))
    _lib.check(sim._L.gk_face_fluxes(sim.h, fx.ctypes.data_as(ctypes.c_void_p),
                                     fy.ctypes.data_as(ctypes.c_void_p)), sim.h)
    return fx, fy


def tap(sim, nsub: int, dt_sub: float, ratio: int) -> Tuple[np.ndarray, np.ndarray]:
    """Advance nsub fixed steps; restricted face fluxes [4][ny/r][nx/r] x and y."""
    p = sim.params
    nxc, nyc = p.nx // ratio, p.ny // ratio
    fx = np.empty((4, nyc, nxc))
    fy = np.empty((4, nyc, nxc))
    _lib.check(sim._L.gk_tap_substeps(sim.h, int(nsub), float(dt_sub), int(ratio),
                                      fx.ctypes.data_as(ctypes.c_void_p),
                                      fy.ctypes.data_as(ctypes.c_void_p)), sim.h)
    return fx, fy


# ------------------------------------------------------------------ data
# Shear-layer thickness of the KH instances.  With sharp layers the
# pointwise solution does not converge under refinement (secondary
# instabilities seeded at the grid scale: plain 256^2 is no closer to a
# 1024^2 run than plain 128^2), so an L1 error against a finer run would not
# measure accuracy; tanh layers of thickness 0.01 converge at second order up
# to t = 1 between 128^2 and 1024^2.
KH_SMOOTH = 0.01


def kh_instance(seed: int, n: int, tmax: float,
                smooth: float = KH_SMOOTH) -> Tuple[Params, np.ndarray, Dict]:
    """One KH problem with the ensemble's parameter ranges (density ratio,
    half-width, perturbation amplitude), no cell noise, tanh shear layers of
    thickness `smooth`, at resolution n."""
    rng = np.random.default_rng(seed)
    draw = {"ratio": float(rng.uniform(1.5, 4.0)), "half_width": float(rng.uniform(0.2, 0.3)),
            "amp": float(rng.uniform(0.005, 0.02))}
    p, c = problems.kh(n, seed=seed, rho_in=draw["ratio"], rho_out=1.0,
                       half_width=draw["half_width"], amp=draw["amp"], noise=0.0,
                       smooth=smooth, tmax=tmax)
    return p, c, draw


def perturb(p: Params, cons: np.ndarray, ratio: int, sigma: float, rng) -> np.ndarray:
    """A 2D state with noise that is constant over each ratio x ratio block:
    rho (1 + sigma u1), vx + sigma c u2, vy + sigma c u3, p (1 + sigma u4),
    u uniform in [-1, 1] per block, c the local sound speed."""
    rho, vx, vy, pre = primitives(p, active2d(p, cons))
    nyc, nxc = p.ny // ratio, p.nx // ratio

    def field():
        return np.repeat(np.repeat(rng.uniform(-1.0, 1.0, (nyc, nxc)), ratio, axis=0), ratio, axis=1)

    c = np.sqrt(p.gamma * pre / rho)
    rho2, vx2 = rho * (1.0 + sigma * field()), vx + sigma * c * field()
    vy2, pre2 = vy + sigma * c * field(), pre * (1.0 + sigma * field())
    return problems.prim_to_cons(p, rho2[None], vx2[None], vy2[None], np.zeros((1,) + rho.shape),
                                 pre2[None])


def generate(seeds: Sequence[int], coarse: int = 256, ratio: int = 4, t_end: float = 2.0,
             snapshots: int = 16, frac: float = 0.25, mode: str = "fast",
             sample_seed: int = 0, tv_min: float = TV_GATE, noise: float = 0.0,
             noisy: int = 1, first: float = 1.0, pairs: bool = False, batch: int = 16,
             log=print) -> Tuple[np.ndarray, np.ndarray]:
    """Training pairs from fine runs (coarse*ratio)^2 restricted to coarse^2.

    The fine runs are the plain method run as ensembles (``Ensemble``: one
    persistent launch per RK stage over every instance of a batch of `batch`
    seeds, whole steps in a CUDA graph).  At `snapshots` times
    t_end (s + first) / (snapshots + first), s = 0 .. snapshots - 1, every
    instance's fine state is copied into a scratch fine handle and restricted;
    one coarse RK2 step of the restricted state is taken with the coarse
    solver, recording its stage-averaged face fluxes (1/2)(F(U) + F(U*)), and
    the scratch fine state is advanced over the same interval in `ratio`
    fixed sub-steps while the fluxes through the coarse faces are accumulated.
    The target is their difference: added to both coarse stages it makes the
    coarse step reproduce the restricted fine step.  The ensemble's own
    trajectories are not touched by the taps.  A fraction `frac` of the faces
    whose stencil variation is at least `tv_min` (the faces the correction is
    applied to) is kept.

    With noise > 0 each snapshot also yields `noisy` sets of pairs from the
    fine state perturbed by ``perturb`` (block noise of relative amplitude
    `noise` on the coarse cells): the fine solver's response to grid-scale
    perturbations, which restricted states alone never show and which a
    correction must damp for a coarse run to stay stable.

    With pairs=True each kept face f is followed by its neighbour across the
    next cell in the normal direction (rows 2m, 2m + 1), the layout of the
    pair loss (Trainer.set_pair_loss); a pair is kept when f's variation is
    at least `tv_min`."""
    from .ensemble import Ensemble
    from .sim import Sim
    rng = np.random.default_rng(sample_seed)
    Xs, Ys = [], []

    def add_pairs(pc, cc, fine, crs, dt_c):
        fx_c, fy_c = tap(crs, 1, dt_c, 1)
        fx_f, fy_f = tap(fine, ratio, dt_c / ratio, ratio)
        a = active2d(pc, cc)
        for direction, Ff, Fc in ((0, fx_f, fx_c), (1, fy_f, fy_c)):
            X, S = face_features(pc, a, direction)
            G = stencil_variation(X)
            D = rotate_to_face(Ff - Fc, direction)
            Y = np.stack([D[:, 0] / S[:, 0], D[:, 1] / S[:, 1], D[:, 2] / S[:, 1],
                          D[:, 3] / S[:, 2]], axis=1)
            keep = (rng.random(len(X)) < frac) & (G >= tv_min)
            if pairs:
                f = np.flatnonzero(keep)
                j, i = f // pc.nx, f % pc.nx
                nb = j * pc.nx + (i + 1) % pc.nx if direction == 0 else ((j + 1) % pc.ny) * pc.nx + i
                sel = np.stack([f, nb], axis=1).ravel()
                Xs.append(X[sel].astype(np.float32))
                Ys.append(Y[sel].astype(np.float32))
            else:
                Xs.append(X[keep].astype(np.float32))
                Ys.append(Y[keep].astype(np.float32))

    seeds = list(seeds)
    for b0 in range(0, len(seeds), batch):
        t0 = time.time()
        group = seeds[b0:b0 + batch]
        inst = [kh_instance(seed, coarse * ratio, t_end) for seed in group]
        fines = [Sim(pf, cf, mode=mode) for pf, cf, _ in inst]
        ens = Ensemble(fines)
        pf, cf0 = inst[0][0], inst[0][1]  # every instance has the same grid and physics
        scratch = Sim(pf, cf0, mode=mode)
        pc, cc = restrict(pf, cf0, ratio)
        crs = Sim(pc, cc, mode=mode)
        drmin_c = min((pc.xmax - pc.xmin) / pc.nx, (pc.ymax - pc.ymin) / pc.ny)
        t = 0.0
        for s in range(snapshots):
            ts = t_end * (s + first) / (snapshots + first)
            if ts > t + 1e-12:
                ens.advance(ts - t)  # every instance from t to ts
                t = fines[0].get_time()
            for fine in fines:
                f0 = fine.download()
                states = [perturb(pf, f0, ratio, noise, rng) for _ in range(noisy)] if noise > 0 else []
                for st in states + [f0]:
                    scratch.upload(st)
                    scratch.set_time(t, 0)
                    _, cc = restrict(pf, st, ratio)
                    crs.set_time(0.0, 0)
                    crs.upload(cc)
                    add_pairs(pc, cc, scratch, crs, pc.cfl * drmin_c / crs.cmax())
        ens.close()
        for h in fines + [scratch, crs]:
            h.close()
        if log:
            log(f"instances {b0 + 1}-{b0 + len(group)}/{len(seeds)}: {time.time() - t0:.1f} s")
    return np.concatenate(Xs), np.concatenate(Ys)


# ------------------------------------------------------------------ model
def init_model(X: np.ndarray, Y: np.ndarray, seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases, small last layer, and the data's
    standardisation appended (gk_mlp model blob)."""
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, np.sqrt(2.0 / NI), (NH, NI))
    w2 = rng.normal(0, np.sqrt(2.0 / NH), (NH, NH))
    w3 = rng.normal(0, 0.1 * np.sqrt(1.0 / NH), (NO, NH))
    xm, xs = X.mean(0), X.std(0) + 1e-6
    ym, ys = Y.mean(0), Y.std(0) + 1e-12
    blob = np.concatenate([w1.ravel(), np.zeros(NH), w2.ravel(), np.zeros(NH), w3.ravel(),
                           np.zeros(NO), xm, xs, ym, ys]).astype(np.float32)
    assert blob.size == NMODEL
    return blob


def standardise(blob: np.ndarray, X: np.ndarray, Y: Optional[np.ndarray] = None):
    xm, xs = blob[NPARAM:NPARAM + NI], blob[NPARAM + NI:NPARAM + 2 * NI]
    Xn = (X - xm) / xs
    if Y is None:
        return Xn
    ym, ys = blob[NPARAM + 2 * NI:NPARAM + 2 * NI + NO], blob[NPARAM + 2 * NI + NO:]
    return Xn, (Y - ym) / ys


class Trainer:
    """Device-side training state (gk_mlp): the model, Adam moments and the
    standardised data set in HBM (BF16 inputs, FP32 targets)."""

    def __init__(self, blob: np.ndarray, X: np.ndarray, Y: np.ndarray, device: int = 0):
        import torch
        self._L = _lib.load()
        b = np.ascontiguousarray(blob, dtype=np.float32)
        m = ctypes.c_void_p()
        _lib.check(self._L.gk_mlp_create(b.ctypes.data_as(ctypes.c_void_p), ctypes.byref(m)))
        self.m = m
        Xn, Yn = standardise(b, X, Y)
        dev = torch.device("cuda", device)
        self.X = torch.from_numpy(np.ascontiguousarray(Xn, dtype=np.float32)).to(dev).to(torch.bfloat16)
        self.Y = torch.from_numpy(np.ascontiguousarray(Yn, dtype=np.float32)).to(dev)
        self.n = len(X)

    def close(self):
        if getattr(self, "m", None):
            self._L.gk_mlp_destroy(self.m)
            self.m = None

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 0) -> float:
        loss = ctypes.c_float()
        _lib.check(self._L.gk_mlp_train(self.m, _ptr(self.X), _ptr(self.Y), self.n, int(batch),
                                        int(steps), float(lr), int(seed), ctypes.byref(loss)))
        return loss.value

    def set_pair_loss(self, w: float) -> None:
        """w < 0: per-face squared error; 0 <= w <= 1: the data are
        neighbouring-face pairs and the loss weights their difference by w
        (gk_mlp_set_pair_loss)."""
        _lib.check(self._L.gk_mlp_set_pair_loss(self.m, float(w)))

    def gradient(self, batch: int):
        g = np.empty(NPARAM, dtype=np.float32)
        loss = ctypes.c_float()
        _lib.check(self._L.gk_mlp_grad(self.m, _ptr(self.X), _ptr(self.Y), self.n, int(batch),
                                       g.ctypes.data_as(ctypes.c_void_p), ctypes.byref(loss)))
        return g, loss.value

    def forward(self, n: Optional[int] = None) -> np.ndarray:
        import torch
        n = self.n if n is None else n
        out = torch.empty((n, NO), dtype=torch.float32, device=self.Y.device)
        _lib.check(self._L.gk_mlp_forward(self.m, _ptr(self.X), int(n), _ptr(out)))
        return out.cpu().numpy()

    def model(self) -> np.ndarray:
        b = np.empty(NMODEL, dtype=np.float32)
        _lib.check(self._L.gk_mlp_get(self.m, b.ctypes.data_as(ctypes.c_void_p)))
        return b


def r2(blob: np.ndarray, X: np.ndarray, Y: np.ndarray, device: int = 0) -> List[float]:
    """Coefficient of determination of each output of the model on (X, Y),
    in standardised units, with the device forward (gk_mlp_forward)."""
    t = Trainer(blob, X, Y, device=device)
    try:
        pred = t.forward()
    finally:
        t.close()
    _, Yn = standardise(np.asarray(blob, dtype=np.float32), X, Y)
    res = ((pred - Yn) ** 2).sum(0)
    tot = ((Yn - Yn.mean(0)) ** 2).sum(0) + 1e-30
    return (1.0 - res / tot).tolist()


def install(sim, blob: Optional[np.ndarray], shock_jump: float = 0.5, pos_frac: float = 0.02,
            tv_min: float = TV_GATE, diss_frac: float = DISS_FRAC, fused: bool = True):
    """Installs (or, with None, removes) the correction on a 2D Sim.  fused:
    the network runs inside the fused 2D stage where the run takes it
    (gk_set_flux_model_fused), else as a pass on the generic path."""
    if blob is None:
        _lib.check(sim._L.gk_set_flux_model(sim.h, None, 0, 0.0, 0.0, 0.0, 0.0), sim.h)
        return
    b = np.ascontiguousarray(blob, dtype=np.float32)
    _lib.check(sim._L.gk_set_flux_model_fused(sim.h, 1 if fused else 0), sim.h)
    _lib.check(sim._L.gk_set_flux_model(sim.h, b.ctypes.data_as(ctypes.c_void_p), b.size,
                                        float(shock_jump), float(pos_frac), float(tv_min),
                                        float(diss_frac)), sim.h)


def detector_count(sim) -> int:
    c = ctypes.c_uint()
    _lib.check(sim._L.gk_flux_model_fired(sim.h, ctypes.byref(c)), sim.h)
    return c.value


# ------------------------------------------------------------------ evaluation
def _timed_run(sim, times: Sequence[float]) -> Tuple[List[np.ndarray], float, bool]:
    """Runs to each time in `times`; returns the density at each, the GPU
    wall time spent inside the advance calls, and whether the run diverged:
    it failed, or its step limit (the run's stepmax) stopped it short of a
    time.  The densities after a divergence are NaN."""
    import torch
    out, spent, diverged = [], 0.0, False
    for tt in times:
        if not diverged:
            torch.cuda.synchronize()
            a = time.perf_counter()
            try:
                sim.advance(tt - sim.get_time())
            except _lib.GkError:
                diverged = True
            torch.cuda.synchronize()
            spent += time.perf_counter() - a
            if not sim.is_continue and sim.get_time() < tt - 1e-12:
                diverged = True
        rho = active2d(sim.params, sim.download())[0].copy()
        out.append(np.full_like(rho, np.nan) if diverged else rho)
    return out, spent, diverged


def _restrict_rho(rho: np.ndarray, r: int) -> np.ndarray:
    ny, nx = rho.shape
    return rho.reshape(ny // r, r, nx // r, r).mean(axis=(1, 3))


def evaluate(blob: np.ndarray, seeds: Sequence[int], coarse: int = 256, t_end: float = 2.0,
             times: Sequence[float] = (0.5, 1.0, 2.0), mode: str = "fast",
             shock_jump: float = 0.5, pos_frac: float = 0.02, tv_min: float = TV_GATE,
             diss_frac: float = DISS_FRAC, log=print) -> Dict:
    """L1 density error against the 4x fine plain run (the truth) for plain
    coarse, plain 2x coarse and learned coarse, each started from the
    restriction of the same fine initial state, and their GPU times.  A
    learned run that takes more than 4x the steps of the plain run at its
    resolution (a collapsed time step) is stopped by that step limit on the
    device and recorded as diverged."""
    from .sim import Sim
    rows = []
    for seed in seeds:
        pf, cf, draw = kh_instance(seed, 4 * coarse, t_end)
        js = Sim(pf, cf, mode=mode)
        truth, _, _ = _timed_run(js, times)
        js.close()
        res = {"seed": seed, **draw}
        for name, ratio, learned in (("plain_%d" % coarse, 4, False),
                                     ("plain_%d" % (2 * coarse), 2, False),
                                     ("learned_%d" % coarse, 4, True)):
            pc, cc = restrict(pf, cf, ratio)
            if learned:  # a collapsing time step ends at the step limit, on the device
                pc = dataclasses.replace(pc, stepmax=4 * res["plain_%d" % coarse]["steps"])
            s = Sim(pc, cc, mode=mode)
            if learned:
                install(s, blob, shock_jump, pos_frac, tv_min, diss_frac)
            s.run_steps(1)  # build the graph outside the timing
            s.set_time(0.0, 0)
            s.upload(cc)
            rho, secs, diverged = _timed_run(s, times)
            m0 = active2d(pc, cc)[0].sum()
            res[name] = {
                "seconds": secs,
                "steps": s.get_step(),
                "diverged": diverged,
                "l1": [float(np.mean(np.abs(r - _restrict_rho(j, ratio)))) for r, j in zip(rho, truth)],
                "l1_at_%d" % coarse: [float(np.mean(np.abs(_restrict_rho(r, 4 // ratio) - _restrict_rho(j, 4))))
                                      for r, j in zip(rho, truth)],
                "mass_drift": None if diverged else float(abs(rho[-1].sum() - m0) / m0),
            }
            if learned:
                res[name]["detector_faces"] = detector_count(s)
            s.close()
        rows.append(res)
        if log:
            log(json_line(res))
    return {"runs": rows, "summary": summarise(rows, coarse)}


def json_line(d) -> str:
    import json
    return json.dumps(d)


def summarise(rows: List[Dict], coarse: int) -> Dict:
    keys = ["plain_%d" % coarse, "plain_%d" % (2 * coarse), "learned_%d" % coarse]
    out = {}
    for k in keys:
        ok = [r for r in rows if not r[k].get("diverged")]
        l1 = np.array([r[k]["l1_at_%d" % coarse] for r in ok]) if ok else np.full((1, 1), np.nan)
        out[k] = {"mean_l1_at_%d" % coarse: l1.mean(axis=0).tolist(),
                  "median_l1_at_%d" % coarse: np.median(l1, axis=0).tolist(),
                  "mean_seconds": float(np.mean([r[k]["seconds"] for r in ok])) if ok else None,
                  "runs": len(ok), "diverged": len(rows) - len(ok)}
    return out
