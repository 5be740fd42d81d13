// gk_kernels.cuh -- the device kernels of one arithmetic mode.
//
// Included by gk_kernels_parity.cu (GK_NS = gk_parity, GK_SEL = 0,
// compiled with -fmad=false) and gk_kernels_fast.cu (GK_NS = gk_fast,
// GK_SEL = 1, FMA contraction allowed); GK_SEL is the HLLC side selection
// of gk_physics.cuh.
//
// Two implementations of one RK stage share the pointwise physics:
//   * the generic path, one kernel per reference phase (ghost fill,
//     ConsToPrim, one flux sweep per direction, UpdateCons), any dimension,
//     five variables;
//   * the fused 2D stage kernel (k_stage2d), which for a 2D run with vz = 0
//     does ConsToPrim + PLM + HLLC in x and y + flux divergence + RK combine
//     + floors in one pass, marching up columns.
// Both end each step in k_cfl, whose last CTA runs the step epilogue of
// Sim::Advance on the device clock (DevTime).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <math_constants.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstdio>

#include "gk_internal.h"

#ifndef GK_NS
#error "define GK_NS"
#endif

namespace GK_NS {

#include "gk_physics.cuh"
#include "gk_learn.cuh"

using gk::Ctx;
using gk::DevTime;
using gk::Geom;
using gk::Phys;

constexpr int kSel = GK_SEL;

#ifndef GK_CHECKED
#define GK_CHECKED 0
#endif
#if GK_CHECKED
// Bounds-checked build (-DGK_CHECKED=1: lib/checked/libgk_cuda.so).  Every
// cell coordinate that indexes a state or face array (sidx, fidx), every row
// the stage kernels store and every TMA row coordinate is checked against
// its array.  A coordinate outside is counted, the first one recorded (site,
// coordinate, bound: gk_checked_report) and clamped into the array, so the
// access stays inside the buffer; a TMA row that fails is not issued and its
// barrier is released empty.  Sites: 1-3 state k, j, i; 4-6 face k, j, i;
// 7 stage store row; 8 TMA row.
__device__ unsigned long long gk_chk_count;
__device__ unsigned long long gk_chk_first;
__device__ __noinline__ int chk_fail(int x, int lo, int hi, int site) {
    if (atomicAdd(&gk_chk_count, 1ull) == 0ull)
        gk_chk_first = ((unsigned long long)(site & 0xffff) << 48) |
                       ((unsigned long long)((unsigned)x & 0xffffffu) << 24) |
                       (unsigned long long)((unsigned)hi & 0xffffffu);
    return x < lo ? lo : (hi > lo ? hi - 1 : lo);
}
__device__ __forceinline__ int chk(int x, int lo, int hi, int site) {
    return (x < lo || x >= hi) ? chk_fail(x, lo, hi, site) : x;
}
#define GK_CHK(x, lo, hi, site) chk((x), (lo), (hi), (site))
#else
#define GK_CHK(x, lo, hi, site) (x)
#endif

// The counters of the checked build (1 when this build has none).
int checked_report(unsigned long long* count, unsigned long long* first) {
#if GK_CHECKED
    if (cudaMemcpyFromSymbol(count, gk_chk_count, sizeof(*count)) != cudaSuccess) return -1;
    if (cudaMemcpyFromSymbol(first, gk_chk_first, sizeof(*first)) != cudaSuccess) return -1;
    return 0;
#else
    (void)count;
    (void)first;
    return 1;
#endif
}

__device__ __forceinline__ long long sidx(const Geom& g, int k, int j, int i) {
    k = GK_CHK(k, g.kofs, g.kofs + g.nzs, 1);
    j = GK_CHK(j, 0, g.leny, 2);
    i = GK_CHK(i, 0, g.pitch, 3);
    return (long long)(k - g.kofs) * g.kstride + (long long)j * g.pitch + i;
}
__device__ __forceinline__ long long fidx(const Geom& g, int k, int j, int i) {
    k = GK_CHK(k, g.kofs, g.kofs + g.nzs + 1, 4);
    j = GK_CHK(j, 0, g.leny + 1, 5);
    i = GK_CHK(i, 0, g.fpitch, 6);
    return (long long)(k - g.kofs) * g.fkstride + (long long)j * g.fpitch + i;
}

// ---------------------------------------------------------------- ghost fill
// Boundary::UpdateBD (boundary.cpp:127-142) with the routines of
// boundary/{outflow_copy,periodic,reflective,outflow}.cpp.  Ghosts of active
// rows/columns only; corners untouched.  With n >= nghost in every filled
// direction each ghost depends on one active cell, so all sides fill in one
// launch.  blockIdx.y = 2*dir + side.
// One ghost cell (id enumerates ghost layer fastest, then the transverse
// active cells) of side `side` in direction `dir`, every variable.
__device__ __forceinline__ void bc_fill_one(double* __restrict__ u, const Geom& g, const Phys& ph,
                                            int dir, int side, long long id) {
    const int n3[3] = {g.nx, g.ny, g.nz};
    const int type = ph.bc[2 * dir + side];
    const int ta = dir == 0 ? g.ny : g.nx;
    const int gi = (int)(id % g.ng);
    const long long r = id / g.ng;
    const int a = (int)(r % ta), b = (int)(r / ta);
    const int e = g.ng + n3[dir];
    const int gc = side == 0 ? gi : e + gi;  // ghost coordinate along dir
    int sc;                                  // source coordinate along dir
    if (type == 1) sc = side == 0 ? gc + n3[dir] : gc - n3[dir];
    else if (type == 0) sc = side == 0 ? g.ng : e - 1;
    else sc = side == 0 ? (g.ng + g.ng - gc - 1) : (e + e - gc - 1);
    int ci, cj, ck, si, sj, sk;
    if (dir == 0) { ci = gc; si = sc; cj = sj = g.jb + a; ck = sk = g.kb + b; }
    else if (dir == 1) { cj = gc; sj = sc; ci = si = g.ib + a; ck = sk = g.kb + b; }
    else { ck = gc; sk = sc; ci = si = g.ib + a; cj = sj = g.jb + b; }
    const long long dst = sidx(g, ck, cj, ci), src = sidx(g, sk, sj, si);
    if (type == 5) return;  // a slab's side filled by the halo exchange (gk_slab.cu)
    if (type == 4) {
        // FixedBD* (fixed.cpp:16-176): the ghost keeps its value at enrollment
        // (the host refuses to run a type-4 side without data; never read null)
        if (!ph.fixed_bd) return;
#pragma unroll
        for (int v = 0; v < 5; ++v) u[v * g.vstride + dst] = ph.fixed_bd[v * g.vstride + dst];
        return;
    }
    double q[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v] = u[v * g.vstride + src];
    const int mom = dir == 0 ? gk::S_MTX : (dir == 1 ? gk::S_MTY : gk::S_MTZ);
    if (type == 2) {
        q[mom] = -q[mom];
    } else if (type == 3) {
        // outflow.cpp:36-60: clamp inflow momentum, floor e_int at 1e-16.
        double mt = q[mom];
        double mc = side == 0 ? smin(mt, 0.0) : smax(mt, 0.0);
        double rho = smax(q[gk::S_DEN], ph.dmin);
        double rhoInv = 1.0 / rho;
        double keOld = 0.5 * rhoInv * mt * mt;
        double keNew = 0.5 * rhoInv * mc * mc;
        double eint = q[gk::S_ENG] - keOld;
        eint = smax(eint, 1e-16);
        q[gk::S_DEN] = rho;
        q[mom] = mc;
        q[gk::S_ENG] = eint + keNew;
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v * g.vstride + dst] = q[v];
}

// Boundary::UpdateBD (boundary.cpp:127-142) for the run's dimensions: one
// grid row per side (blockIdx.y = 2 * direction + side), one ghost cell per
// thread through bc_fill_one.
__global__ void k_bc(double* __restrict__ u, Geom g, Phys ph, const DevTime* __restrict__ tm) {
    if (!tm->active) return;
    const int dir = blockIdx.y >> 1, side = blockIdx.y & 1;
    const int n3[3] = {g.nx, g.ny, g.nz};
    if (n3[dir] <= 1) return;
    if (dir == 2 && !((ph.fill_z >> side) & 1)) return;
    const int ta = dir == 0 ? g.ny : g.nx;
    const int tb = dir == 2 ? g.ny : g.nz;
    const long long count = (long long)g.ng * ta * tb;
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= count) return;
    bc_fill_one(u, g, ph, dir, side, id);
}

// Cell centres in Domain's order of operations (sim.cpp:36-41).
__device__ __forceinline__ double centre(double lo, int ng, double d, int i) {
    return lo - ng * d + 0.5 * d + i * d;
}

// Boundary::FixedBDInner (fixed.cpp:180-206): inside the index box, cells
// with x^2 + y^2 + z^2 < 0.5^2 get back their values at enrollment; run
// after the sides (boundary.cpp:127-142).
__global__ void k_fix_inner(double* __restrict__ u, Geom g, Phys ph, const DevTime* __restrict__ tm) {
    if (!tm->active) return;
    const int i = ph.inner[0] + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = ph.inner[2] + blockIdx.y;
    const int k = g.kb + blockIdx.z;
    if (i >= ph.inner[1]) return;
    const double x = centre(g.xmin, g.ng, g.dx, i);
    const double y = centre(g.ymin, g.ng, g.dy, j);
    const double z = centre(g.zmin, g.ng, g.dz, k);
    const double r2 = x * x + y * y + z * z;
    if (!(r2 < 0.5 * 0.5)) return;
    const long long c = sidx(g, k, j, i);
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v * g.vstride + c] = ph.fixed_bd[v * g.vstride + c];
}

// Boundary::ImmersedReflective (immersed.cpp:243-303), run after the sides
// and before the inner reset (boundary.cpp:127-142): each shell cell of an
// immersed body takes the weighted state at its image point, with the
// radial velocity reversed.  Targets lie outside the body and shell cells
// inside it, so no cell is both read and written: one thread per shell cell
// gives the reference's serial result.  Expression order is the reference's
// (CarToLocal / LocalToCar at immersed.cpp:72-85 inlined).
__global__ void k_immersed(double* __restrict__ u, Geom g, Phys ph, const DevTime* __restrict__ tm) {
    if (!tm->active) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ph.nshell) return;
    const gk::Shell& sh = ph.shells[s];
    const double cosp = sh.dir[0], sinp = sh.dir[1], cost = sh.dir[2], sint = sh.dir[3];
    const double w0 = sh.w[0];
    const long long vs = g.vstride;
    double dens = 0, vr = 0, vp = 0, vt = 0, pres = 0;
    for (int n = 1; n <= sh.ntar; ++n) {
        const long long c = sh.tgt[n - 1];
        const double wn = sh.w[n];
        const double denTar = smax(u[gk::S_DEN * vs + c], ph.dmin);
        const double denInv = GK_RCP(denTar);
        dens += GK_RCP(1 - w0) * wn * denTar;
        const double vx = u[gk::S_MTX * vs + c] * denInv;
        const double vy = u[gk::S_MTY * vs + c] * denInv;
        const double vz = u[gk::S_MTZ * vs + c] * denInv;
        const double vrloc = vx * cosp * sint + vy * sinp * sint + vz * cost;
        const double vploc = -vx * sinp + vy * cosp;
        const double vtloc = vx * cosp * cost + vy * sinp * cost - vz * sint;
        vr += GK_RCP(-1. - w0) * wn * vrloc;
        vp += GK_RCP(1. - w0) * wn * vploc;
        vt += GK_RCP(1. - w0) * wn * vtloc;
        const double engTar = u[gk::S_ENG * vs + c];
        const double engKin = 0.5 * denTar * (vx * vx + vy * vy + vz * vz);
        double preTar = ph.gm1 * (engTar - engKin);
        preTar = (preTar > ph.pmin) ? preTar : ph.pmin;
        pres += GK_RCP(1. - w0) * wn * preTar;
    }
    const double vx = vr * sint * cosp + vt * cost * cosp - vp * sinp;
    const double vy = vr * sint * sinp + vt * cost * sinp + vp * cosp;
    const double vz = vr * cost - vt * sint;
    const long long c = sh.cell;
    u[gk::S_DEN * vs + c] = dens;
    u[gk::S_MTX * vs + c] = dens * vx;
    u[gk::S_MTY * vs + c] = dens * vy;
    u[gk::S_MTZ * vs + c] = dens * vz;
    const double engKin = 0.5 * dens * (vx * vx + vy * vy + vz * vz);
    u[gk::S_ENG * vs + c] = engKin + pres * ph.gm1Rec;
}

// ------------------------------------------------------------ ConsToPrim
// EquationOfState::ConsToPrim (adiabatic.cpp:18-61) over every stored cell.
__device__ __forceinline__ void cons_to_prim5(double d, double mx, double my, double mz, double e,
                                              const Phys& ph, double w[5]) {
    d = GK_FLOOR(d, ph.dmin);
    w[gk::P_RHO] = d;
    double denInv = GK_RCP(d);
    w[gk::P_VX] = mx * denInv;
    w[gk::P_VY] = my * denInv;
    w[gk::P_VZ] = mz * denInv;
    double engKin = 0.5 * denInv * (mx * mx + my * my + mz * mz);
    double pre = ph.gm1 * (e - engKin);
    w[gk::P_PRE] = GK_BELOW(ph.pmin, pre) ? pre : ph.pmin;
}

// EquationOfState::ConsToPrim (adiabatic.cpp:18-61) of every stored cell,
// ghosts included.
__global__ void k_c2p(const double* __restrict__ u, double* __restrict__ w, Geom g, Phys ph,
                      const DevTime* __restrict__ tm) {
    if (!tm->active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int k = g.kofs + blockIdx.z;
    if (i >= g.lenx) return;
    const long long c = sidx(g, k, j, i);
    double q[5];
    cons_to_prim5(u[gk::S_DEN * g.vstride + c], u[gk::S_MTX * g.vstride + c],
                  u[gk::S_MTY * g.vstride + c], u[gk::S_MTZ * g.vstride + c],
                  u[gk::S_ENG * g.vstride + c], ph, q);
#pragma unroll
    for (int v = 0; v < 5; ++v) w[v * g.vstride + c] = q[v];
}

// ------------------------------------------------------------ flux sweeps
// Flux::CalFlux (cal_flux.cpp:13-160): faces ib..ie along the sweep, active
// in the other directions.  dir 0 = x (flx1), 1 = y (flx2), 2 = z (flx3).
// For z the reference forms the face states with ReconstructYZPLM, whose
// slope is along y (recon_piecewise_linear.cpp:29-50); that is kept.
__global__ void k_flux(const double* __restrict__ w, double* __restrict__ F, Geom g, Phys ph,
                       int dir, const DevTime* __restrict__ tm) {
    if (!tm->active) return;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int bidx = blockIdx.y, cidx = blockIdx.z;
    int i, j, k;
    if (dir == 0) { i = g.ib + a; j = g.jb + bidx; k = g.kb + cidx; if (i > g.ie) return; }
    else if (dir == 1) { i = g.ib + a; j = g.jb + bidx; k = g.kb + cidx; if (i >= g.ie) return; }
    else { i = g.ib + a; j = g.jb + bidx; k = g.kb + cidx; if (i >= g.ie) return; }
    // cells m (left of the face) and p (right); stencil offsets
    double wl[5], wr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        double l1, l2, l3, r1, r2, r3;
        const double* p = w + v * g.vstride;
        if (dir == 0) {
            l1 = p[sidx(g, k, j, i - 2)]; l2 = p[sidx(g, k, j, i - 1)]; l3 = p[sidx(g, k, j, i)];
            r1 = l2; r2 = l3; r3 = p[sidx(g, k, j, i + 1)];
        } else if (dir == 1) {
            l1 = p[sidx(g, k, j - 2, i)]; l2 = p[sidx(g, k, j - 1, i)]; l3 = p[sidx(g, k, j, i)];
            r1 = l2; r2 = l3; r3 = p[sidx(g, k, j + 1, i)];
        } else {
            l1 = p[sidx(g, k - 1, j - 1, i)]; l2 = p[sidx(g, k - 1, j, i)];
            l3 = p[sidx(g, k - 1, j + 1, i)];
            r1 = p[sidx(g, k, j - 1, i)]; r2 = p[sidx(g, k, j, i)]; r3 = p[sidx(g, k, j + 1, i)];
        }
        if (ph.plm) {
#if GK_FASTMATH
            wl[v] = l2 + vanleer_half(l2 - l1, l3 - l2);
            wr[v] = r2 - vanleer_half(r2 - r1, r3 - r2);
#else
            wl[v] = l2 + 0.5 * vanleer(l2 - l1, l3 - l2);
            wr[v] = r2 - 0.5 * vanleer(r2 - r1, r3 - r2);
#endif
        } else {
            wl[v] = l2;
            wr[v] = r2;
        }
    }
    // rotation (hllc.cpp:25-27): x (vx | vy, vz), y (vy | vz, vx), z (vz | vx, vy)
    const int sn = dir == 0 ? gk::P_VX : (dir == 1 ? gk::P_VY : gk::P_VZ);
    const int s1 = dir == 0 ? gk::P_VY : (dir == 1 ? gk::P_VZ : gk::P_VX);
    const int s2 = dir == 0 ? gk::P_VZ : (dir == 1 ? gk::P_VX : gk::P_VY);
    Flux5 f;
    hllc<true, kSel>(wl[gk::P_RHO], wl[sn], wl[s1], wl[s2], wl[gk::P_PRE], wr[gk::P_RHO], wr[sn],
                     wr[s1], wr[s2], wr[gk::P_PRE], ph, f);
    // momentum slots of the rotated components (slot ids equal prim ids)
    const long long c = fidx(g, k, j, i);
    F[gk::S_DEN * g.fvstride + c] = f.d;
    F[sn * g.fvstride + c] = f.n;
    F[s1 * g.fvstride + c] = f.t1;
    F[s2 * g.fvstride + c] = f.t2;
    F[gk::S_ENG * g.fvstride + c] = f.e;
}

// ------------------------------------------------------------ UpdateCons
// Sim::UpdateCons, both overloads (update_cons.cpp:11-133, 135-269).
// update_cons.cpp:55-68, five slots (DEN, MTX, MTY, ENG, MTZ).
__device__ __forceinline__ void floors5(double (&r)[5], const Phys& ph, DevTime* tm) {
    if (GK_BELOW(r[gk::S_DEN], ph.dmin)) {
        r[gk::S_DEN] = ph.dmin;
        r[gk::S_MTX] = 0.0;
        r[gk::S_MTY] = 0.0;
        r[gk::S_MTZ] = 0.0;
        r[gk::S_ENG] = ph.pmin / ph.gm1 + 0.0;
        atomicAdd(&tm->floor_den, 1ull);
    } else {
        double inv_den = GK_RCP(r[gk::S_DEN]);
        double ke = 0.5 * inv_den *
                    (r[gk::S_MTX] * r[gk::S_MTX] + r[gk::S_MTY] * r[gk::S_MTY] +
                     r[gk::S_MTZ] * r[gk::S_MTZ]);
        double press = ph.gm1 * (r[gk::S_ENG] - ke);
        if (GK_BELOW(press, ph.pmin)) {
            r[gk::S_ENG] = ph.pmin / ph.gm1 + ke;
            atomicAdd(&tm->floor_pre, 1ull);
        }
    }
}

// The same with mz = 0 (four slots DEN, MTX, MTY, ENG): the mz terms are
// exact zeros.
__device__ __forceinline__ void floors4(double (&r)[4], const Phys& ph, DevTime* tm) {
    if (r[0] < ph.dmin) {
        r[0] = ph.dmin;
        r[1] = 0.0;
        r[2] = 0.0;
        r[3] = ph.pmin / ph.gm1 + 0.0;
        atomicAdd(&tm->floor_den, 1ull);
    } else {
        double inv_den = GK_RCP(r[0]);
        double ke = 0.5 * inv_den * (r[1] * r[1] + r[2] * r[2]);
        double press = ph.gm1 * (r[3] - ke);
        if (press < ph.pmin) {
            r[3] = ph.pmin / ph.gm1 + ke;
            atomicAdd(&tm->floor_pre, 1ull);
        }
    }
}

// floors4 that also returns the reciprocal density of the result (for the
// CFL speed of the same cell).
__device__ __forceinline__ double floors4_inv(double (&r)[4], const Phys& ph, DevTime* tm) {
    if (GK_BELOW(r[0], ph.dmin)) {
        r[0] = ph.dmin;
        r[1] = 0.0;
        r[2] = 0.0;
        r[3] = ph.pmin / ph.gm1 + 0.0;
        atomicAdd(&tm->floor_den, 1ull);
        return GK_RCP(ph.dmin);
    }
    double inv_den = GK_RCP(r[0]);
#if GK_FASTMATH
    const double m2 = r[1] * r[1] + r[2] * r[2];
    double press = fma(-ph.hgm1 * inv_den, m2, ph.gm1 * r[3]);
    if (GK_BELOW(press, ph.pmin)) {
        r[3] = ph.pmin / ph.gm1 + 0.5 * inv_den * m2;
        atomicAdd(&tm->floor_pre, 1ull);
    }
#else
    double ke = 0.5 * inv_den * (r[1] * r[1] + r[2] * r[2]);
    double press = ph.gm1 * (r[3] - ke);
    if (GK_BELOW(press, ph.pmin)) {
        r[3] = ph.pmin / ph.gm1 + ke;
        atomicAdd(&tm->floor_pre, 1ull);
    }
#endif
    return inv_den;
}

// Sim::UpdateCons (update_cons.cpp:11-68) of one RK stage: the flux
// difference of every active cell, the stage combine and the floors.
__global__ void k_update(const double* u0, const double* uc, double* out,
                         const double* __restrict__ F1, const double* __restrict__ F2,
                         const double* __restrict__ F3, Geom g, Phys ph, int three, double c1,
                         double c2, double c3, DevTime* tm) {
    if (!tm->active) return;
    const int i = g.ib + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = g.jb + blockIdx.y;
    const int k = g.kb + blockIdx.z;
    if (i >= g.ie) return;
    const double dt = tm->dt;
    const double dtdx = dt * g.dxRec, dtdy = dt * g.dyRec, dtdz = dt * g.dzRec;
    const long long c = sidx(g, k, j, i);
    const long long fc = fidx(g, k, j, i);
    double r[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        double dF = (F1[v * g.fvstride + fc + 1] - F1[v * g.fvstride + fc]) * dtdx;
        if (g.ndim == 2) {
            dF = dF + (F2[v * g.fvstride + fc + g.fpitch] - F2[v * g.fvstride + fc]) * dtdy;
        } else if (g.ndim == 3) {
            dF = dF + (F2[v * g.fvstride + fc + g.fpitch] - F2[v * g.fvstride + fc]) * dtdy +
                 (F3[v * g.fvstride + fc + g.fkstride] - F3[v * g.fvstride + fc]) * dtdz;
        }
        if (three) r[v] = c1 * u0[v * g.vstride + c] + c2 * uc[v * g.vstride + c] - c3 * dF;
        else r[v] = c1 * uc[v * g.vstride + c] - c2 * dF;
    }
    floors5(r, ph, tm);
#pragma unroll
    for (int v = 0; v < 5; ++v) out[v * g.vstride + c] = r[v];
}

// ------------------------------------------------------------ gravity kick
// SourceTerm::ConstGravity (const_gravity.cpp:10-69) with dt/2, applied
// before and after the integrator (sim.cpp:85-91): E += m*g*dt; m += rho*g*dt.
// SourceTerm::UpdateSource (source.cpp:12-21) for one half step dt/2 of
// the Strang splitting (sim.cpp:85-91): constant gravity, then one point
// mass (point_gravity.cpp:11-92) or two (binary_gravity.cpp), whose second
// mass orbits at angle omega*t + theta1 with t = t_n + dt/2 for the first
// half kick (which = 0) and t_n + dt for the second (which = 1).
__global__ void k_kick(double* __restrict__ u, Geom g, Phys ph, const DevTime* __restrict__ tm,
                       int which) {
    if (!tm->active) return;
    const int i = g.ib + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = g.jb + blockIdx.y;
    const int k = g.kb + blockIdx.z;
    if (i >= g.ie) return;
    const double hdt = 0.5 * tm->dt;
    const long long c = sidx(g, k, j, i);
    const int moms[3] = {gk::S_MTX, gk::S_MTY, gk::S_MTZ};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double gd = ph.grav[d];
        if (gd == 0) continue;
        double& E = u[gk::S_ENG * g.vstride + c];
        double& m = u[moms[d] * g.vstride + c];
        E += m * gd * hdt;
        m += u[gk::S_DEN * g.vstride + c] * gd * hdt;
    }
    if (ph.npoint == 0) return;
    const double xnow = centre(g.xmin, g.ng, g.dx, i);
    const double ynow = centre(g.ymin, g.ng, g.dy, j);
    const double znow = centre(g.zmin, g.ng, g.dz, k);
    double gxdt, gydt, gzdt;
    {
        const double delx = xnow - ph.pm[1], dely = ynow - ph.pm[2], delz = znow - ph.pm[3];
        const double r2 = delx * delx + dely * dely + delz * delz;
        const double rs = ph.pm[4];
        const double rInv = 1.0 / sqrt(r2 + rs * rs);
        const double gv = -(ph.pm[0] * hdt) * rInv * rInv * rInv;
        gxdt = gv * delx;
        gydt = gv * dely;
        gzdt = gv * delz;
        if (ph.npoint == 2) {
            const double t = which == 0 ? tm->t + 0.5 * tm->dt : tm->t + tm->dt;
            const double theta = ph.pm[8] * t + ph.pm[10];
            const double x1 = ph.pm[9] * cos(theta), y1 = ph.pm[9] * sin(theta), z1 = ph.pm[6];
            const double dx1 = xnow - x1, dy1 = ynow - y1, dz1 = znow - z1;
            const double r1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1;
            const double rs1 = ph.pm[7];
            const double r1Inv = 1.0 / sqrt(r1 + rs1 * rs1);
            const double g1 = -(ph.pm[5] * hdt) * r1Inv * r1Inv * r1Inv;
            const double gInd = 0.0;  // the indirect term, zeroed in binary_gravity.cpp
            gxdt = gv * delx + g1 * dx1 + gInd * x1;
            gydt = gv * dely + g1 * dy1 + gInd * y1;
            gzdt = gv * delz + g1 * dz1 + gInd * z1;
        }
    }
    double& D = u[gk::S_DEN * g.vstride + c];
    double& E = u[gk::S_ENG * g.vstride + c];
    double& MX = u[gk::S_MTX * g.vstride + c];
    double& MY = u[gk::S_MTY * g.vstride + c];
    double& MZ = u[gk::S_MTZ * g.vstride + c];
    E += MX * gxdt + MY * gydt + MZ * gzdt;
    MX += D * gxdt;
    MY += D * gydt;
    MZ += D * gzdt;
}

// ------------------------------------------------------------ CFL + epilogue
// EquationOfState::CalCmax (adiabatic.cpp:115-160) on the active cells,
// reduced in registers -> warp shuffles -> shared memory -> one atomicMax per
// CTA on the bit pattern (non-negative doubles order like their bits; NaN
// and inf sort above every finite value, so they reach the check below).
// With epilogue = 1 the last CTA to finish runs the tail of the Sim::Advance
// loop body (sim.cpp:93-98) and the next step's dt (sim.cpp:77-81).
__device__ __forceinline__ double cell_cmax(double d, double mx, double my, double mz, double e,
                                            const Phys& ph, bool has_z) {
    d = GK_FLOOR(d, ph.dmin);
    double denInv = GK_RCP(d);
    double vx = mx * denInv, vy = my * denInv, vz = mz * denInv;
    double engKin = has_z ? 0.5 * (vx * mx + vy * my + vz * mz) : 0.5 * (vx * mx + vy * my);
    double pres = ph.gm1 * (e - engKin);
    pres = GK_BELOW(ph.pmin, pres) ? pres : ph.pmin;
    double cs = GK_SQRT(ph.gamma * pres * denInv);
    double local = fabs(vx) + cs;
    local = GK_MAXNN(local, fabs(vy) + cs);
    if (has_z) local = GK_MAXNN(local, fabs(vz) + cs);
    return local;
}

// cell_cmax of a 2D cell (vz = 0) whose density is at least the floor,
// given its reciprocal density: the same operations as cell_cmax without
// recomputing 1/rho.
__device__ __forceinline__ double cell_cmax_inv(double mx, double my, double e, double denInv,
                                                const Phys& ph) {
    double vx = mx * denInv, vy = my * denInv;
#if GK_FASTMATH
    double pres = fma(-ph.hgm1, vx * mx + vy * my, ph.gm1 * e);
#else
    double engKin = 0.5 * (vx * mx + vy * my);
    double pres = ph.gm1 * (e - engKin);
#endif
    pres = GK_BELOW(ph.pmin, pres) ? pres : ph.pmin;
    double cs = GK_SQRT(ph.gamma * pres * denInv);
    double local = fabs(vx) + cs;
    local = GK_MAXNN(local, fabs(vy) + cs);
    return local;
}

__device__ void step_epilogue(DevTime* tm, const Geom& g, const Phys& ph, int epilogue) {
    unsigned long long bits = atomicAdd(&tm->cmax_acc, 0ull);
    double cm = __longlong_as_double((long long)bits);
    tm->cmax_acc = (unsigned long long)__double_as_longlong(1e-16);
    tm->done_ctas = 0;
    tm->cmax_last = cm;
    if (!(cm <= DBL_MAX)) tm->status |= gk::STATUS_NONFINITE;
    if (epilogue) {
        tm->t += tm->dt;
        tm->step += 1;
        tm->dtUntilOutput = tm->tNext - tm->t;
        if (ph.stepmax > 0 && tm->step >= ph.stepmax) tm->is_continue = 0;
        if (tm->nlog < tm->log_cap) tm->log[tm->nlog] = tm->dt;
        tm->nlog += 1;
        if (tm->steps_left > 0) tm->steps_left -= 1;
        int act = (fabs(tm->tNext - tm->t) > 1e-12) && tm->is_continue && tm->status == 0 &&
                  tm->steps_left != 0;
        if (act) {
            double dt = ph.cfl * g.drmin / cm;
            tm->dt = smin(dt, tm->dtUntilOutput);
        }
        tm->active = act;
    }
}

// EquationOfState::CalCmax (adiabatic.cpp:115-160) as a maximum of the
// non-negative doubles' bit patterns folded into tm->cmax_acc; with
// `epilogue` the last CTA to finish runs the tail of the Sim::Advance loop
// body (sim.cpp:92-103) through step_epilogue.
template <bool HAS_Z>
__global__ void __launch_bounds__(256) k_cfl(const double* __restrict__ u, Geom g, Phys ph,
                                             DevTime* tm, int epilogue) {
    if (epilogue && !tm->active) return;
    unsigned long long best = 0ull;
    const long long ncell = (long long)g.nx * g.ny * g.nz;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < ncell;
         id += (long long)gridDim.x * blockDim.x) {
        const int i = g.ib + (int)(id % g.nx);
        const long long r = id / g.nx;
        const int j = g.jb + (int)(r % g.ny);
        const int k = g.kb + (int)(r / g.ny);
        const long long c = sidx(g, k, j, i);
        double mz = HAS_Z ? u[gk::S_MTZ * g.vstride + c] : 0.0;
        double local = cell_cmax(u[gk::S_DEN * g.vstride + c], u[gk::S_MTX * g.vstride + c],
                                 u[gk::S_MTY * g.vstride + c], mz, u[gk::S_ENG * g.vstride + c],
                                 ph, HAS_Z);
        unsigned long long b = (unsigned long long)__double_as_longlong(local);
        best = b > best ? b : best;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
        best = x > best ? x : best;
    }
    __shared__ unsigned long long wmax[8];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long m = wmax[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = wmax[w] > m ? wmax[w] : m;
        atomicMax(&tm->cmax_acc, m);
        __threadfence();
        unsigned int prev = atomicAdd(&tm->done_ctas, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        step_epilogue(tm, g, ph, epilogue);
    }
}

// Start of a Sim::Advance call (sim.cpp:70-72, 77-81) or of a fixed-count
// run (steps > 0: no output time, step budget).
__device__ __forceinline__ void begin_one(DevTime* tm, const Geom& g, const Phys& ph,
                                          double dtoutput, int steps) {
    if (steps > 0) {
        tm->tNext = CUDART_INF;
        tm->dtUntilOutput = CUDART_INF;
        tm->steps_left = steps;
    } else {
        tm->tNext = tm->t + dtoutput;
        tm->dtUntilOutput = dtoutput;
        tm->steps_left = -1;
    }
    int act = (fabs(tm->tNext - tm->t) > 1e-12) && tm->is_continue && tm->status == 0;
    if (act) {
        double dt = ph.cfl * g.drmin / tm->cmax_last;
        tm->dt = smin(dt, tm->dtUntilOutput);
    }
    tm->active = act;
}

// begin_one on the device clock (sim.cpp:70-72, 77-81).
__global__ void k_begin(DevTime* tm, Geom g, Phys ph, double dtoutput, int steps) {
    begin_one(tm, g, ph, dtoutput, steps);
}

// The step epilogue of a slab whose last stage deferred it: cmax_acc holds
// the maximum over every slab of the grid by now.
__global__ void k_epilogue(DevTime* tm, Geom g, Phys ph) {
    if (!tm->active) return;
    step_epilogue(tm, g, ph, 1);
}

// ------------------------------------------------------------ 1D in one CTA
// A 1D run of up to 1024 cells per array row (lenx) in one CTA: each step
// runs the generic path's phases -- ghost fill (x sides), ConsToPrim of the
// row, x fluxes, UpdateCons per RK stage, then CalCmax and the step
// epilogue -- with the generic kernels' expressions in their order (the
// same bits), the primitives and fluxes in shared memory and a barrier
// where the generic path has a launch.  Up to nsteps steps per launch,
// while the run is active.
template <bool HAS_Z>
__global__ void __launch_bounds__(1024) k_run1d(double* A, double* B, Geom g, Phys ph, DevTime* tm,
                                                int nsteps) {
    extern __shared__ double sh1[];
    const int t = threadIdx.x;
    const int nf = g.nx + 1;
    double* W = sh1;               // primitives [5][lenx]
    double* F = sh1 + 5 * g.lenx;  // x fluxes [5][nx + 1], face ib + f
    const long long vs = g.vstride;
    const long long row = sidx(g, g.kb, g.jb, 0);
    __shared__ unsigned long long wmax[32];
    // one RK stage: out = c1*uc - c2*dF (three = 0) or c1*u0 + c2*uc - c3*dF
    auto stage = [&](double* uc, const double* u0, double* out, bool three, double c1, double c2,
                     double c3) {
        if (t < 2 * g.ng) bc_fill_one(uc, g, ph, 0, t / g.ng, t % g.ng);
        __syncthreads();
        if (t < g.lenx) {
            const long long c = row + t;
            double q[5];
            cons_to_prim5(uc[gk::S_DEN * vs + c], uc[gk::S_MTX * vs + c], uc[gk::S_MTY * vs + c],
                          uc[gk::S_MTZ * vs + c], uc[gk::S_ENG * vs + c], ph, q);
#pragma unroll
            for (int v = 0; v < 5; ++v) W[v * g.lenx + t] = q[v];
        }
        __syncthreads();
        if (t < nf) {
            const int i = g.ib + t;  // the face between cells i-1 and i
            double wl[5], wr[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                const double* p = W + v * g.lenx;
                const double l1 = p[i - 2], l2 = p[i - 1], l3 = p[i];
                const double r1 = l2, r2 = l3, r3 = p[i + 1];
                if (ph.plm) {
#if GK_FASTMATH
                    wl[v] = l2 + vanleer_half(l2 - l1, l3 - l2);
                    wr[v] = r2 - vanleer_half(r2 - r1, r3 - r2);
#else
                    wl[v] = l2 + 0.5 * vanleer(l2 - l1, l3 - l2);
                    wr[v] = r2 - 0.5 * vanleer(r2 - r1, r3 - r2);
#endif
                } else {
                    wl[v] = l2;
                    wr[v] = r2;
                }
            }
            Flux5 f;
            hllc<true, kSel>(wl[gk::P_RHO], wl[gk::P_VX], wl[gk::P_VY], wl[gk::P_VZ], wl[gk::P_PRE],
                             wr[gk::P_RHO], wr[gk::P_VX], wr[gk::P_VY], wr[gk::P_VZ], wr[gk::P_PRE],
                             ph, f);
            F[gk::S_DEN * nf + t] = f.d;
            F[gk::P_VX * nf + t] = f.n;
            F[gk::P_VY * nf + t] = f.t1;
            F[gk::P_VZ * nf + t] = f.t2;
            F[gk::S_ENG * nf + t] = f.e;
        }
        __syncthreads();
        if (t < g.nx) {
            const long long c = row + g.ib + t;
            const double dt = tm->dt;
            const double dtdx = dt * g.dxRec;
            double r[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                double dF = (F[v * nf + t + 1] - F[v * nf + t]) * dtdx;
                if (three) r[v] = c1 * u0[v * vs + c] + c2 * uc[v * vs + c] - c3 * dF;
                else r[v] = c1 * uc[v * vs + c] - c2 * dF;
            }
            floors5(r, ph, tm);
#pragma unroll
            for (int v = 0; v < 5; ++v) out[v * vs + c] = r[v];
        }
        __syncthreads();
    };
    const double frac13 = 1.0 / 3.0;
    for (int s = 0; s < nsteps; ++s) {
        if (!tm->active) break;  // set by the previous step's epilogue (or the begin kernel)
        if (ph.integrator == 1) {
            stage(A, nullptr, A, false, 1.0, 1.0, 0.0);
        } else {
            stage(A, nullptr, B, false, 1.0, 1.0, 0.0);
            if (ph.integrator == 3) {
                stage(B, A, B, true, 0.75, 0.25, 0.25);
                stage(B, A, A, true, frac13, 2 * frac13, 2 * frac13);
            } else {
                stage(B, A, A, true, 0.5, 0.5, 0.5);
            }
        }
        // CalCmax of the new state and the step epilogue (k_cfl's)
        unsigned long long best = 0ull;
        if (t < g.nx) {
            const long long c = row + g.ib + t;
            const double mz = HAS_Z ? A[gk::S_MTZ * vs + c] : 0.0;
            const double local = cell_cmax(A[gk::S_DEN * vs + c], A[gk::S_MTX * vs + c],
                                           A[gk::S_MTY * vs + c], mz, A[gk::S_ENG * vs + c], ph,
                                           HAS_Z);
            best = (unsigned long long)__double_as_longlong(local);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
            best = x > best ? x : best;
        }
        if ((t & 31) == 0) wmax[t >> 5] = best;
        __syncthreads();
        if (t == 0) {
            unsigned long long m = wmax[0];
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = wmax[w] > m ? wmax[w] : m;
            atomicMax(&tm->cmax_acc, m);
            step_epilogue(tm, g, ph, 1);
        }
        __syncthreads();
    }
}

// Sets *flag when MTZ is non-zero on an active cell: the fused 2D path
// evolves four variables and needs MTZ = 0 (no reference counterpart; the
// reference evolves all five everywhere).
__global__ void k_mtz_check(const double* __restrict__ u, Geom g, int* flag) {
    const long long ncell = (long long)g.nx * g.ny * g.nz;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < ncell;
         id += (long long)gridDim.x * blockDim.x) {
        const int i = g.ib + (int)(id % g.nx);
        const long long r = id / g.nx;
        const int j = g.jb + (int)(r % g.ny);
        const int k = g.kb + (int)(r / g.ny);
        if (u[gk::S_MTZ * g.vstride + sidx(g, k, j, i)] != 0.0) *flag = 1;
    }
}

// ------------------------------------------------------------ fused 2D stage
// One RK stage of a 2D run with vz = 0 (four variables) in one pass:
// ConsToPrim (adiabatic.cpp:18-61) -> PLM (recon_piecewise_linear.cpp:8-50)
// -> HLLC x and y (hllc.cpp:22-101) -> dF (update_cons.cpp:38-47) -> RK
// combine -> floors (update_cons.cpp:55-68).
//
// A CTA of 128 threads owns buffer columns x0-2 .. x0+125 (124 updated
// columns plus a 2-cell halo each side) and marches up rows y0 .. y1-1.
// Along y everything stays in registers: each thread carries its column's
// primitives, the left state of the next y face and the flux of the face
// below.  Along x, neighbours exchange through shared memory once per row.
// Every lane runs the same straight-line body (halo lanes read clamped
// neighbours and discard their results); the x-face and the y-face Riemann
// problems of a row are independent, so they sit side by side between the
// same barriers and their instruction streams interleave.  Raw rows are
// prefetched two rows ahead, the RK base state u0 one row ahead.
constexpr int kStageThreads = 128;
constexpr int kStageCols = kStageThreads - 4;

// The periodic images of a cell the fused 2D stage writes (row = its row,
// xi = its column, oc = its offset): on a grid periodic on all four sides
// (ph.periodic_images) the stage stores the values the ghost fill would copy
// from the cell into the x and y ghosts, so the steps need no ghost fill.
// Corners, which no fill touches, stay as they are.  Planes DEN, MTX, MTY,
// ENG (the fused path never writes MTZ).
__device__ __forceinline__ void store_images(double* out, long long vs, long long P, long long oc,
                                             int xi, int row, const Geom& g, const double (&r)[4]) {
    auto put = [&](long long o) {
        out[o] = r[0];
        out[vs + o] = r[1];
        out[2 * vs + o] = r[2];
        out[3 * vs + o] = r[3];
    };
    if (xi < g.ib + g.ng) put(oc + (GK_CHK(xi + g.nx, 0, g.lenx, 10) - xi));
    if (xi >= g.ie - g.ng) put(oc + (GK_CHK(xi - g.nx, 0, g.lenx, 10) - xi));
    if (row < g.jb + g.ng) put(oc + (long long)(GK_CHK(row + g.ny, 0, g.leny, 11) - row) * P);
    if (row >= g.je - g.ng) put(oc + (long long)(GK_CHK(row - g.ny, 0, g.leny, 11) - row) * P);
}

struct W4 {
    double r, vx, vy, p;
};
struct Q4 {
    double d, mx, my, e;
};

__device__ __forceinline__ W4 c2p4(const Q4& q, const Phys& ph) {
    W4 w;
    double d = GK_FLOOR(q.d, ph.dmin);
    w.r = d;
    double denInv = GK_RCP(d);
    w.vx = q.mx * denInv;
    w.vy = q.my * denInv;
#if GK_FASTMATH
    // p = (gamma-1) E - ((gamma-1)/2) |m|^2 / rho
    double pre = fma(-ph.hgm1 * denInv, q.mx * q.mx + q.my * q.my, ph.gm1 * q.e);
#else
    double engKin = 0.5 * denInv * (q.mx * q.mx + q.my * q.my);
    double pre = ph.gm1 * (q.e - engKin);
#endif
    w.p = GK_BELOW(ph.pmin, pre) ? pre : ph.pmin;
    return w;
}

#if GK_FASTMATH
// Fast mode: vl4 returns half slopes and the face states add them directly.
__device__ __forceinline__ W4 vl4(const W4& a, const W4& b, const W4& c) {
    W4 s;
    s.r = vanleer_half(b.r - a.r, c.r - b.r);
    s.vx = vanleer_half(b.vx - a.vx, c.vx - b.vx);
    s.vy = vanleer_half(b.vy - a.vy, c.vy - b.vy);
    s.p = vanleer_half(b.p - a.p, c.p - b.p);
    return s;
}
__device__ __forceinline__ W4 plus_half(const W4& u, const W4& h) {
    return W4{u.r + h.r, u.vx + h.vx, u.vy + h.vy, u.p + h.p};
}
__device__ __forceinline__ W4 minus_half(const W4& u, const W4& h) {
    return W4{u.r - h.r, u.vx - h.vx, u.vy - h.vy, u.p - h.p};
}
#else
__device__ __forceinline__ W4 vl4(const W4& a, const W4& b, const W4& c) {
    W4 s;
    s.r = vanleer(b.r - a.r, c.r - b.r);
    s.vx = vanleer(b.vx - a.vx, c.vx - b.vx);
    s.vy = vanleer(b.vy - a.vy, c.vy - b.vy);
    s.p = vanleer(b.p - a.p, c.p - b.p);
    return s;
}
__device__ __forceinline__ W4 plus_half(const W4& u, const W4& s) {
    return W4{u.r + 0.5 * s.r, u.vx + 0.5 * s.vx, u.vy + 0.5 * s.vy, u.p + 0.5 * s.p};
}
__device__ __forceinline__ W4 minus_half(const W4& u, const W4& s) {
    return W4{u.r - 0.5 * s.r, u.vx - 0.5 * s.vx, u.vy - 0.5 * s.vy, u.p - 0.5 * s.p};
}
#endif

__device__ __forceinline__ Q4 ldq(const double* __restrict__ u, long long vs, long long c) {
    return Q4{__ldg(u + c), __ldg(u + vs + c), __ldg(u + 2 * vs + c), __ldg(u + 3 * vs + c)};
}

// y face: rotation (vy | vz, vx) with vz = 0, so tangential 1 carries vx.
__device__ __forceinline__ void hllc_y(const W4& l, const W4& r, const Phys& ph, Flux5& f) {
    hllc<false, kSel>(l.r, l.vy, l.vx, 0.0, l.p, r.r, r.vy, r.vx, 0.0, r.p, ph, f);
}
// x face: rotation (vx | vy, vz).
__device__ __forceinline__ void hllc_x(const W4& l, const W4& r, const Phys& ph, Flux5& f) {
    hllc<false, kSel>(l.r, l.vx, l.vy, 0.0, l.p, r.r, r.vx, r.vy, 0.0, r.p, ph, f);
}

// KIND 0: u' = c1*uc - c2*dF (stage 1); 1: u' = c1*u0 + c2*uc - c3*dF
// (later stages); 2: as 1 and the last stage of the step, which also applies
// the gravity half kick (sim.cpp:89-91), reduces the CFL speed of the new
// state and, in its last CTA, runs the step epilogue -- the separate kick and
// CFL passes over the state disappear.
template <int KIND, bool PLM>
__global__ void __launch_bounds__(kStageThreads, 3)
    k_stage2d(const double* __restrict__ uc, const double* u0, double* out, Geom g, Phys ph,
              double c1, double c2, double c3, DevTime* tm, int rows) {
    constexpr bool THREE = KIND >= 1;
    constexpr bool LAST = KIND == 2;
    if (!tm->active) return;
    unsigned long long cbest = 0ull;  // CFL speed of this thread's cells (bit pattern)
    __shared__ double sP[4][kStageThreads];
    __shared__ double sXL[4][kStageThreads];
    __shared__ double sF[4][kStageThreads];

    const double dt = tm->dt;
    const double dtdx = dt * g.dxRec, dtdy = dt * g.dyRec;
    const int t = threadIdx.x;
    const int tl = t > 0 ? t - 1 : 0;                       // clamped neighbours
    const int tr = t < kStageThreads - 1 ? t + 1 : t;
    const int xi = g.ib - 2 + blockIdx.x * kStageCols + t;
    const int xl = xi < g.lenx ? xi : g.lenx - 1;           // clamped load column
    const bool do_cell = t >= 2 && t <= kStageThreads - 3 && xi < g.ie;
    const int y0 = g.jb + blockIdx.y * rows;
    const int y1 = min(y0 + rows, g.je);
    const long long vs = g.vstride;
    const long long P = g.pitch;
    const long long cbase = sidx(g, g.kb, 0, xl);

    // prologue: primitives of rows y0-2, y0-1, y0; raw row y0+1 in flight
    const W4 Pm2 = c2p4(ldq(uc, vs, cbase + (y0 - 2) * P), ph);
    W4 Pm1 = c2p4(ldq(uc, vs, cbase + (y0 - 1) * P), ph);
    Q4 Q0 = ldq(uc, vs, cbase + y0 * P);
    W4 P0 = c2p4(Q0, ph);
    Q4 Qn = ldq(uc, vs, cbase + (y0 + 1) * P);
    Q4 Qm1;
    Q4 U0n{0, 0, 0, 0};
    // left state of y face y0 (cell y0-1)
    W4 wlNext = PLM ? plus_half(Pm1, vl4(Pm2, Pm1, P0)) : Pm1;
    Flux5 fyPrev;
    {
        // y face y0 (no cell of this segment is complete yet)
        const Q4 Q1 = Qn;
        Qn = ldq(uc, vs, cbase + (y0 + 2) * P);
        if (THREE) {
            const long long c0 = cbase + y0 * P;  // u0 may alias out: plain loads
            U0n = Q4{u0[c0], u0[vs + c0], u0[2 * vs + c0], u0[3 * vs + c0]};
        }
        const W4 P1 = c2p4(Q1, ph);
        W4 wr = P0, wlNew = P0;
        if (PLM) {
            const W4 s = vl4(Pm1, P0, P1);
            wr = minus_half(P0, s);
            wlNew = plus_half(P0, s);
        }
        hllc_y(wlNext, wr, ph, fyPrev);
        wlNext = wlNew;
        Pm1 = P0;
        P0 = P1;
        Qm1 = Q0;
        Q0 = Q1;
    }

    for (int f = y0 + 1; f <= y1; ++f) {
        // loads in flight across the arithmetic of this row
        const Q4 Q1 = Qn;  // raw row f+1
        if (f + 2 <= y1 + 1) Qn = ldq(uc, vs, cbase + (f + 2) * P);
        const Q4 U0 = U0n;  // base state of row f-1
        if (THREE && f <= y1 - 1) {
            const long long c0 = cbase + f * P;
            U0n = Q4{u0[c0], u0[vs + c0], u0[2 * vs + c0], u0[3 * vs + c0]};
        }
        const W4 P1 = c2p4(Q1, ph);

        // x neighbours of row f-1
        sP[0][t] = Pm1.r; sP[1][t] = Pm1.vx; sP[2][t] = Pm1.vy; sP[3][t] = Pm1.p;
        __syncthreads();
        W4 xr = Pm1, wr = P0, wlNew = P0;
        if (PLM) {
            const W4 a{sP[0][tl], sP[1][tl], sP[2][tl], sP[3][tl]};
            const W4 c{sP[0][tr], sP[1][tr], sP[2][tr], sP[3][tr]};
            const W4 sx = vl4(a, Pm1, c);
            const W4 sy = vl4(Pm1, P0, P1);
            const W4 xlft = plus_half(Pm1, sx);
            xr = minus_half(Pm1, sx);
            wr = minus_half(P0, sy);
            wlNew = plus_half(P0, sy);
            sXL[0][t] = xlft.r; sXL[1][t] = xlft.vx; sXL[2][t] = xlft.vy; sXL[3][t] = xlft.p;
        } else {
            sXL[0][t] = Pm1.r; sXL[1][t] = Pm1.vx; sXL[2][t] = Pm1.vy; sXL[3][t] = Pm1.p;
        }
        __syncthreads();
        // the two Riemann problems of this row: x face at the left of cell
        // (f-1, xi) and y face f below cell (f, xi)
        const W4 xl_state{sXL[0][tl], sXL[1][tl], sXL[2][tl], sXL[3][tl]};
        Flux5 fx, fy;
        hllc_x(xl_state, xr, ph, fx);
        hllc_y(wlNext, wr, ph, fy);
        sF[0][t] = fx.d; sF[1][t] = fx.n; sF[2][t] = fx.t1; sF[3][t] = fx.e;
        __syncthreads();
        if (do_cell) {
            // update_cons.cpp:38-53: (Fx(i+1)-Fx(i))*dtdx + (Fy(j+1)-Fy(j))*dtdy
            double dF0 = (sF[0][tr] - fx.d) * dtdx + (fy.d - fyPrev.d) * dtdy;
            double dF1 = (sF[1][tr] - fx.n) * dtdx + (fy.t1 - fyPrev.t1) * dtdy;
            double dF2 = (sF[2][tr] - fx.t1) * dtdx + (fy.n - fyPrev.n) * dtdy;
            double dF3 = (sF[3][tr] - fx.e) * dtdx + (fy.e - fyPrev.e) * dtdy;
            double r[4];
            if (THREE) {
                r[0] = c1 * U0.d + c2 * Qm1.d - c3 * dF0;
                r[1] = c1 * U0.mx + c2 * Qm1.mx - c3 * dF1;
                r[2] = c1 * U0.my + c2 * Qm1.my - c3 * dF2;
                r[3] = c1 * U0.e + c2 * Qm1.e - c3 * dF3;
            } else {
                r[0] = c1 * Qm1.d - c2 * dF0;
                r[1] = c1 * Qm1.mx - c2 * dF1;
                r[2] = c1 * Qm1.my - c2 * dF2;
                r[3] = c1 * Qm1.e - c2 * dF3;
            }
            floors4(r, ph, tm);
            if (LAST) {
                if (ph.has_grav) {
                    // SourceTerm::ConstGravity with dt/2 (const_gravity.cpp:28-46)
                    const double hdt = 0.5 * dt;
                    if (ph.grav[0] != 0) {
                        r[3] += r[1] * ph.grav[0] * hdt;
                        r[1] += r[0] * ph.grav[0] * hdt;
                    }
                    if (ph.grav[1] != 0) {
                        r[3] += r[2] * ph.grav[1] * hdt;
                        r[2] += r[0] * ph.grav[1] * hdt;
                    }
                }
                const double local = cell_cmax(r[0], r[1], r[2], 0.0, r[3], ph, false);
                const unsigned long long b = (unsigned long long)__double_as_longlong(local);
                cbest = b > cbest ? b : cbest;
            }
            const long long oc = cbase + (long long)GK_CHK(f - 1, g.jb, g.je, 7) * P;
            out[oc] = r[0];
            out[vs + oc] = r[1];
            out[2 * vs + oc] = r[2];
            out[3 * vs + oc] = r[3];
            if (ph.periodic_images) store_images(out, vs, P, oc, xi, f - 1, g, r);
        }
        fyPrev = fy;
        wlNext = wlNew;
        Pm1 = P0;
        P0 = P1;
        Qm1 = Q0;
        Q0 = Q1;
    }
    if (LAST) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, cbest, o);
            cbest = x > cbest ? x : cbest;
        }
        __shared__ unsigned long long wmax[kStageThreads / 32];
        __shared__ bool last;
        if ((t & 31) == 0) wmax[t >> 5] = cbest;
        __syncthreads();
        if (t == 0) {
            unsigned long long m = wmax[0];
            for (int w = 1; w < kStageThreads / 32; ++w) m = wmax[w] > m ? wmax[w] : m;
            atomicMax(&tm->cmax_acc, m);
            __threadfence();
            const unsigned int prev = atomicAdd(&tm->done_ctas, 1u);
            last = (prev == gridDim.x * gridDim.y - 1);
        }
        __syncthreads();
        if (last && t == 0) {
            __threadfence();
            step_epilogue(tm, g, ph, 1);
        }
    }
}



// ------------------------------------------------------------ fused 2D stage, TMA rows
// The same stage with its input rows staged in shared memory by the tensor
// memory accelerator instead of registers.  One cp.async.bulk.tensor load
// brings a 3D box of NT columns x 1 row x 4 variable planes into a ring
// slot; an mbarrier per slot counts its bytes.  Raw rows run four ahead of
// the row being converted (ring of 6: rows f-2 .. f+3 live); the RK base
// state u0 runs three ahead (ring of 4).  A slot is refilled only after the
// barrier that follows its last read, behind a proxy fence.  The box origin
// is column (NT-4)*strip, a multiple of 16 bytes for NT = 64, 128, 256;
// columns past the last one read as zero (TMA out-of-bounds fill) and feed
// only halo lanes.  Waits are bounded: a wait that gives up sets
// STATUS_TMA_TIMEOUT and the kernel carries on, so it cannot hang.
//
// stage_tile_tma does one tile (strip bx, segment by).  The single-problem
// kernel runs one tile per CTA; the ensemble kernel (k_ens_stage) is
// persistent: each CTA takes tiles of any instance from a tile table through
// an atomic counter, reusing its ring and barriers.
constexpr int kRing = 6;
constexpr int kRing0 = 4;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_row(double* dst, const CUtensorMap* map, int x, int y,
                                        unsigned bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(0), "r"(smem_u32(bar))
        : "memory");
}
// A plain arrival (no transaction bytes): completes the phase of a
// one-arrival barrier without a copy (the checked build's refused rows).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_wait(uint64_t* bar, unsigned phase, int* status) {
    for (int it = 0; it < (1 << 22); ++it) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(phase)
            : "memory");
        if (ok) return;
    }
    atomicOr(status, gk::STATUS_TMA_TIMEOUT);
}

// Row exchanges of the stage: each thread's four values as two 16-byte
// pairs, [pair][thread], so a warp's 16-byte accesses are conflict-free and
// each exchange is two loads instead of four.
template <int NT>
struct StageShared {
    double2 sP[2][NT];
    double2 sXL[2][NT];
    double2 sF[2][NT];
    uint64_t bar[kRing];
    uint64_t bar0[kRing0];
    unsigned long long wmax[NT / 32];
    int cur;
    int last;
};

// The learned flux correction inside the fused stage (the stage with LEARN):
// each row's x and y faces get the correction the generic path's pass
// (k_flux_correct, gk_mlp.cu) would add, from the same functions
// (gk_learn.cuh).  Per warp and row, the 32 x faces and 32 y faces of its
// lanes are 4 tiles of 16 for the tensor cores: slots 0..31 the x faces of
// lanes 0..31, slots 32..63 their y faces.
struct LearnWarp {
    alignas(16) __nv_bfloat16 x[64 * gklearn::NI];  // standardised inputs per slot
    float y[64][4];                                 // standardised outputs per slot
    gklearn::FaceScale fs[64];                      // detector and scales per slot
};
struct LearnArgs {
    const gklearn::MlpWeights* w;  // shared memory
    LearnWarp* warps;              // shared memory, one per warp
    gk::FluxGate gate;
    unsigned* fired;               // faces the detector left to plain HLLC
};

// The stencil of a face from four cells along its normal: density, normal
// and tangential velocity, pressure.
struct Stencil4 {
    double r[4], vn[4], vt[4], p[4];
};
__device__ __forceinline__ Stencil4 stencil_x(const W4& a, const W4& b, const W4& c, const W4& d) {
    return Stencil4{{a.r, b.r, c.r, d.r}, {a.vx, b.vx, c.vx, d.vx}, {a.vy, b.vy, c.vy, d.vy},
                    {a.p, b.p, c.p, d.p}};
}
__device__ __forceinline__ Stencil4 stencil_y(const W4& a, const W4& b, const W4& c, const W4& d) {
    return Stencil4{{a.r, b.r, c.r, d.r}, {a.vy, b.vy, c.vy, d.vy}, {a.vx, b.vx, c.vx, d.vx},
                    {a.p, b.p, c.p, d.p}};
}

// Corrects this lane's x face (side 0, when hasx) and y face (side 1, when
// hasy); every lane of the warp takes part.  stencil(side) gives the face's
// stencil.  The two sides run as rolled loops, so each piece of the code is
// in the kernel once per call site.  A vetoed face keeps its flux; nfired
// counts the vetoed faces this lane owns (countx / county).
template <class StencilFn>
__device__ __forceinline__ void learn_faces(const LearnArgs& la, const StencilFn& stencil,
                                            bool hasx, bool countx, Flux5& fx, double dtdx,
                                            bool hasy, bool county, Flux5& fy, double dtdy,
                                            const Phys& ph, unsigned& nfired) {
    using namespace gklearn;
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    LearnWarp& lw = la.warps[threadIdx.x >> 5];
    const MlpWeights& w = *la.w;
    unsigned needx = 0, needy = 0;
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        const int slot = 32 * side + lane;
        FaceScale& fs = lw.fs[slot];
        fs.gate = 2.f;
        if (side ? hasy : hasx) {
            const Stencil4 st = stencil(side);
            face_inputs(st.r, st.vn, st.vt, st.p, ph.gamma, ph.gm1Rec, la.gate, w.norm,
                        lw.x + slot * NI, fs);
        } else {
#pragma unroll
            for (int e = 0; e < NI; ++e) lw.x[slot * NI + e] = __float2bfloat16_rn(0.f);
        }
        // the tiles of a side run only where a face needs the network (none
        // keep plain HLLC because they are absent or smooth)
        const unsigned need = __ballot_sync(0xffffffffu, fs.gate != 2.f);
        if (side) needy = need;
        else needx = need;
    }
    __syncwarp();
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        if (!(side ? needy : needx)) continue;
        float y[2][4];
        forward_tiles<2>(w, lw.x + side * 32 * NI, y);
        if (t < 2) {
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                const int s0 = 32 * side + 16 * m + g;
                lw.y[s0][2 * t] = y[m][0];
                lw.y[s0][2 * t + 1] = y[m][1];
                lw.y[s0 + 8][2 * t] = y[m][2];
                lw.y[s0 + 8][2 * t + 1] = y[m][3];
            }
        }
    }
    __syncwarp();
    double cx[4] = {0.0, 0.0, 0.0, 0.0}, cy[4] = {0.0, 0.0, 0.0, 0.0};
    bool okx = false, oky = false;
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        const int slot = 32 * side + lane;
        const FaceScale& fs = lw.fs[slot];
        if (fs.gate == 2.f) continue;
        double c[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) c[o] = face_correction(lw.y[slot][o], o, fs, w.norm);
        if (face_vetoed(c[0], c[3], side ? dtdy : dtdx, fs, la.gate)) {
            nfired += (side ? county : countx) ? 1u : 0u;
            continue;
        }
        if (side) {
#pragma unroll
            for (int o = 0; o < 4; ++o) cy[o] = c[o];
            oky = true;
        } else {
#pragma unroll
            for (int o = 0; o < 4; ++o) cx[o] = c[o];
            okx = true;
        }
    }
    if (okx) {
        fx.d += cx[0];
        fx.n += cx[1];
        fx.t1 += cx[2];
        fx.e += cx[3];
    }
    if (oky) {
        fy.d += cy[0];
        fy.n += cy[1];
        fy.t1 += cy[2];
        fy.e += cy[3];
    }
    __syncwarp();  // lw may be refilled
}

template <int NT>
__device__ __forceinline__ void stage_init_barriers(StageShared<NT>& sm) {
    if (threadIdx.x == 0) {
        for (int i = 0; i < kRing; ++i) mbar_init(&sm.bar[i], 1);
        for (int i = 0; i < kRing0; ++i) mbar_init(&sm.bar0[i], 1);
        fence_proxy_async();
    }
    __syncthreads();
}

// seq / seq0: rows of raw state / base state this CTA has loaded so far;
// they fix each row's ring slot and mbarrier phase across tiles.
// tiles_total: tiles of this problem; the LAST stage's last tile runs the
// step epilogue.
// LEARN: the learned flux correction of every face (la, k_stage2d_learn).
template <int NT, int KIND, bool PLM, bool LEARN = false>
__device__ __forceinline__ void stage_tile_tma(const CUtensorMap* mapc, const CUtensorMap* map0,
                                               double* out, const Geom& g, const Phys& ph,
                                               double c1, double c2, double c3, DevTime* tm,
                                               int rows, int bx, int by, unsigned tiles_total,
                                               double* ring, double* ring0, StageShared<NT>& sm,
                                               unsigned& seq, unsigned& seq0,
                                               const LearnArgs* la = nullptr) {
    constexpr bool THREE = KIND >= 1;
    constexpr bool LAST = KIND == 2;
    constexpr int COLS = NT - 4;
    constexpr int RD = 4 * NT;
    constexpr unsigned RB = RD * sizeof(double);
    unsigned long long cbest = 0ull;
    const bool unit = !THREE && c1 == 1.0 && c2 == 1.0;

    const double dt = tm->dt;
    const double dtdx = dt * g.dxRec, dtdy = dt * g.dyRec;
    const int t = threadIdx.x;
    const int tl = t > 0 ? t - 1 : 0;
    const int tr = t < NT - 1 ? t + 1 : t;
    const int x0 = g.ib - 2 + bx * COLS;  // box origin column
    const int xi = x0 + t;
    const bool do_cell = t >= 2 && t <= NT - 3 && xi < g.ie;
    const int y0 = g.jb + by * rows;
    const int y1 = min(y0 + rows, g.je);
    const int rlo = y0 - 2;
    const long long vs = g.vstride;
    const long long P = g.pitch;
    const long long cbase = sidx(g, g.kb, 0, xi < g.lenx ? xi : g.lenx - 1);
    int* status = &tm->status;

    auto rs = [&](int r) { return seq + (unsigned)(r - rlo); };
    auto rs0 = [&](int r) { return seq0 + (unsigned)(r - y0); };
    auto issue = [&](int r) {
        const unsigned q = rs(r) % kRing;
#if GK_CHECKED
        if ((x0 & 1) || x0 < 0 || x0 >= g.pitch || r < 0 || r >= g.leny) {
            chk_fail(r, 0, g.leny, 8);
            mbar_arrive(&sm.bar[q]);
            return;
        }
#endif
        tma_row(ring + q * RD, mapc, x0, r, RB, &sm.bar[q]);
    };
    auto issue0 = [&](int r) {
        const unsigned q = rs0(r) % kRing0;
#if GK_CHECKED
        if ((x0 & 1) || x0 < 0 || x0 >= g.pitch || r < 0 || r >= g.leny) {
            chk_fail(r, 0, g.leny, 8);
            mbar_arrive(&sm.bar0[q]);
            return;
        }
#endif
        tma_row(ring0 + q * RD, map0, x0, r, RB, &sm.bar0[q]);
    };
    auto wait = [&](int r) { mbar_wait(&sm.bar[rs(r) % kRing], (rs(r) / kRing) & 1u, status); };
    auto wait0 = [&](int r) {
        mbar_wait(&sm.bar0[rs0(r) % kRing0], (rs0(r) / kRing0) & 1u, status);
    };
    auto rowq = [&](int r) {
        const double* p = ring + (rs(r) % kRing) * RD;
        return Q4{p[t], p[NT + t], p[2 * NT + t], p[3 * NT + t]};
    };
    auto rowq0 = [&](int r) {
        const double* p = ring0 + (rs0(r) % kRing0) * RD;
        return Q4{p[t], p[NT + t], p[2 * NT + t], p[3 * NT + t]};
    };

    __syncthreads();  // the previous tile is done with every ring slot
    if (t == 0) {
        fence_proxy_async();
        for (int r = rlo; r <= min(y0 + 3, y1 + 1); ++r) issue(r);
        if (THREE)
            for (int r = y0; r <= min(y0 + 2, y1 - 1); ++r) issue0(r);
    }

    // prologue: primitives of rows y0-2, y0-1, y0
    wait(y0 - 2);
    W4 Pm2 = c2p4(rowq(y0 - 2), ph);
    unsigned nfired = 0;  // LEARN: vetoed faces this thread owns
    wait(y0 - 1);
    W4 Pm1 = c2p4(rowq(y0 - 1), ph);
    wait(y0);
    W4 P0 = c2p4(rowq(y0), ph);
    W4 wlNext = PLM ? plus_half(Pm1, vl4(Pm2, Pm1, P0)) : Pm1;
    Flux5 fyPrev;
    {
        // y face y0
        wait(y0 + 1);
        const W4 P1 = c2p4(rowq(y0 + 1), ph);
        __syncthreads();  // row y0-2 is read by all: its slot may be refilled
        if (t == 0 && y0 + 4 <= y1 + 1) {
            fence_proxy_async();
            issue(y0 + 4);
        }
        W4 wr = P0, wlNew = P0;
        if (PLM) {
            const W4 s = vl4(Pm1, P0, P1);
            wr = minus_half(P0, s);
            wlNew = plus_half(P0, s);
        }
        hllc_y(wlNext, wr, ph, fyPrev);
        if constexpr (LEARN) {
            // y face y0 (rows y0-2 .. y0+1); the segment below computes it
            // too, so only the grid's first segment counts its veto
            Flux5 none{};
            const auto st = [&](int) { return stencil_y(Pm2, Pm1, P0, P1); };
            learn_faces(*la, st, false, false, none, dtdx, do_cell, do_cell && by == 0, fyPrev,
                        dtdy, ph, nfired);
            Pm2 = Pm1;
        }
        wlNext = wlNew;
        Pm1 = P0;
        P0 = P1;
    }

    for (int f = y0 + 1; f <= y1; ++f) {
        wait(f + 1);
        const W4 P1 = c2p4(rowq(f + 1), ph);
        sm.sP[0][t] = make_double2(Pm1.r, Pm1.vx); sm.sP[1][t] = make_double2(Pm1.vy, Pm1.p);
        __syncthreads();
        if (t == 0) {
            // raw row f-2 and base-state row f-2 were last read in iteration f-1
            fence_proxy_async();
            if (f + 4 <= y1 + 1) issue(f + 4);
            if (THREE && f + 2 <= y1 - 1) issue0(f + 2);
        }
        W4 xr = Pm1, wr = P0, wlNew = P0;
        if (PLM) {
            const double2 a0 = sm.sP[0][tl], a1 = sm.sP[1][tl];
            const double2 c0 = sm.sP[0][tr], c1v = sm.sP[1][tr];
            const W4 a{a0.x, a0.y, a1.x, a1.y};
            const W4 c{c0.x, c0.y, c1v.x, c1v.y};
            const W4 sx = vl4(a, Pm1, c);
            const W4 sy = vl4(Pm1, P0, P1);
            const W4 xlft = plus_half(Pm1, sx);
            xr = minus_half(Pm1, sx);
            wr = minus_half(P0, sy);
            wlNew = plus_half(P0, sy);
            sm.sXL[0][t] = make_double2(xlft.r, xlft.vx); sm.sXL[1][t] = make_double2(xlft.vy, xlft.p);
        } else {
            sm.sXL[0][t] = make_double2(Pm1.r, Pm1.vx); sm.sXL[1][t] = make_double2(Pm1.vy, Pm1.p);
        }
        __syncthreads();
        const double2 x0v = sm.sXL[0][tl], x1v = sm.sXL[1][tl];
        const W4 xl_state{x0v.x, x0v.y, x1v.x, x1v.y};
        Flux5 fx, fy;
        hllc_x(xl_state, xr, ph, fx);
        hllc_y(wlNext, wr, ph, fy);
        if constexpr (LEARN) {
            // x face (xi-1 | xi) of row f-1: cells xi-2 .. xi+1 of sP; a face
            // computed by two strips counts its veto in the strip that
            // updates cell xi (the grid's last face: cell xi-1)
            const int ta = t >= 2 ? t - 2 : 0;
            const auto st = [&](int side) {
                if (side) return stencil_y(Pm2, Pm1, P0, P1);
                const double2 e0 = sm.sP[0][ta], e1 = sm.sP[1][ta];
                const double2 l0 = sm.sP[0][tl], l1 = sm.sP[1][tl];
                const double2 r0 = sm.sP[0][tr], r1 = sm.sP[1][tr];
                return stencil_x(W4{e0.x, e0.y, e1.x, e1.y}, W4{l0.x, l0.y, l1.x, l1.y}, Pm1,
                                 W4{r0.x, r0.y, r1.x, r1.y});
            };
            const bool hasx = t >= 2 && t <= NT - 2 && xi >= g.ib && xi <= g.ie;
            learn_faces(*la, st, hasx, hasx && (t <= NT - 3 || xi == g.ie), fx, dtdx, do_cell,
                        do_cell, fy, dtdy, ph, nfired);
        }
        sm.sF[0][t] = make_double2(fx.d, fx.n); sm.sF[1][t] = make_double2(fx.t1, fx.e);
        __syncthreads();
        if (THREE) wait0(f - 1);
        if (do_cell) {
            const Q4 Qm1 = rowq(f - 1);
            const double2 fr0 = sm.sF[0][tr], fr1 = sm.sF[1][tr];
            double dF0 = (fr0.x - fx.d) * dtdx + (fy.d - fyPrev.d) * dtdy;
            double dF1 = (fr0.y - fx.n) * dtdx + (fy.t1 - fyPrev.t1) * dtdy;
            double dF2 = (fr1.x - fx.t1) * dtdx + (fy.n - fyPrev.n) * dtdy;
            double dF3 = (fr1.y - fx.e) * dtdx + (fy.e - fyPrev.e) * dtdy;
            double r[4];
            if (THREE) {
                const Q4 U0 = rowq0(f - 1);
                r[0] = c1 * U0.d + c2 * Qm1.d - c3 * dF0;
                r[1] = c1 * U0.mx + c2 * Qm1.mx - c3 * dF1;
                r[2] = c1 * U0.my + c2 * Qm1.my - c3 * dF2;
                r[3] = c1 * U0.e + c2 * Qm1.e - c3 * dF3;
            } else if (unit) {
                // c1 = c2 = 1 (every integrator's first stage): the products are exact
                r[0] = Qm1.d - dF0;
                r[1] = Qm1.mx - dF1;
                r[2] = Qm1.my - dF2;
                r[3] = Qm1.e - dF3;
            } else {
                r[0] = c1 * Qm1.d - c2 * dF0;
                r[1] = c1 * Qm1.mx - c2 * dF1;
                r[2] = c1 * Qm1.my - c2 * dF2;
                r[3] = c1 * Qm1.e - c2 * dF3;
            }
            const double invk = floors4_inv(r, ph, tm);  // r[0] >= dmin after it
            if (LAST) {
                if (ph.has_grav) {
                    const double hdt = 0.5 * dt;
                    if (ph.grav[0] != 0) {
                        r[3] += r[1] * ph.grav[0] * hdt;
                        r[1] += r[0] * ph.grav[0] * hdt;
                    }
                    if (ph.grav[1] != 0) {
                        r[3] += r[2] * ph.grav[1] * hdt;
                        r[2] += r[0] * ph.grav[1] * hdt;
                    }
                }
                const double local = cell_cmax_inv(r[1], r[2], r[3], invk, ph);
                const unsigned long long b = (unsigned long long)__double_as_longlong(local);
                cbest = b > cbest ? b : cbest;
            }
            const long long oc = cbase + (long long)GK_CHK(f - 1, g.jb, g.je, 7) * P;
            out[oc] = r[0];
            out[vs + oc] = r[1];
            out[2 * vs + oc] = r[2];
            out[3 * vs + oc] = r[3];
            if (ph.periodic_images) store_images(out, vs, P, oc, xi, f - 1, g, r);
        }
        fyPrev = fy;
        wlNext = wlNew;
        if (LEARN) Pm2 = Pm1;
        Pm1 = P0;
        P0 = P1;
    }
    if constexpr (LEARN) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) nfired += __shfl_xor_sync(0xffffffffu, nfired, o);
        if ((t & 31) == 0 && nfired && la->fired) atomicAdd(la->fired, nfired);
    }
    if (LAST) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, cbest, o);
            cbest = x > cbest ? x : cbest;
        }
        if ((t & 31) == 0) sm.wmax[t >> 5] = cbest;
        __syncthreads();
        if (t == 0) {
            unsigned long long m = sm.wmax[0];
            for (int w = 1; w < NT / 32; ++w) m = sm.wmax[w] > m ? sm.wmax[w] : m;
            atomicMax(&tm->cmax_acc, m);
            sm.last = false;
            if (!ph.defer_epilogue) {
                // a slab of a split grid runs its epilogue after the max over
                // all slabs (launch_epilogue)
                __threadfence();
                const unsigned int prev = atomicAdd(&tm->done_ctas, 1u);
                sm.last = (prev == tiles_total - 1);
            }
        }
        __syncthreads();
        if (sm.last && t == 0) {
            __threadfence();
            step_epilogue(tm, g, ph, 1);
        }
    }
    seq += (unsigned)(y1 + 2 - rlo);
    if (THREE) seq0 += (unsigned)(y1 - y0);
}

template <int NT, bool THREE>
__host__ __device__ constexpr size_t stage_dyn_bytes() {
    return (size_t)(kRing + (THREE ? kRing0 : 0)) * 4 * NT * sizeof(double);
}

// One RK stage of a 2D run (ConsToPrim, PLM, HLLC x and y, UpdateCons with
// the stage combine and floors: adiabatic.cpp:18-61, recon_piecewise_linear.cpp:8-50,
// hllc.cpp:22-101, update_cons.cpp:11-68), tiles staged by TMA: stage_tile_tma.
template <int NT, int KIND, bool PLM>
__global__ void __launch_bounds__(NT, 512 / NT)
    k_stage2d_tma(const __grid_constant__ CUtensorMap mapc, const __grid_constant__ CUtensorMap map0,
                  double* out, Geom g, Phys ph, double c1, double c2, double c3, DevTime* tm,
                  int rows) {
    if (!tm->active) return;
    extern __shared__ __align__(128) double dyn[];
    __shared__ StageShared<NT> sm;
    stage_init_barriers(sm);
    unsigned seq = 0, seq0 = 0;
    stage_tile_tma<NT, KIND, PLM>(&mapc, &map0, out, g, ph, c1, c2, c3, tm, rows, blockIdx.x,
                                  blockIdx.y, gridDim.x * gridDim.y, dyn, dyn + kRing * 4 * NT, sm,
                                  seq, seq0);
}

// The fused stage with the learned flux correction at every face.  Dynamic
// shared memory: the row rings, then the network (BF16 weights) and one
// LearnWarp per warp.
template <int NT, bool THREE>
__host__ __device__ constexpr size_t learn_dyn_bytes() {
    return stage_dyn_bytes<NT, THREE>() + sizeof(gklearn::MlpWeights) + (NT / 32) * sizeof(LearnWarp);
}

// k_stage2d_tma with the learned correction added to every face's HLLC flux
// (hllc.cpp:90-95, cal_flux.cpp:89-121), the model's weights in shared memory.
template <int NT, int KIND, bool PLM>
__global__ void __launch_bounds__(NT, 256 / NT)
    k_stage2d_learn(const __grid_constant__ CUtensorMap mapc, const __grid_constant__ CUtensorMap map0,
                    double* out, Geom g, Phys ph, double c1, double c2, double c3, DevTime* tm,
                    int rows, const float* __restrict__ model, gk::FluxGate gate, unsigned* fired) {
    if (!tm->active) return;
    extern __shared__ __align__(128) double dyn[];
    __shared__ StageShared<NT> sm;
    unsigned char* lp = reinterpret_cast<unsigned char*>(dyn) + stage_dyn_bytes<NT, (KIND >= 1)>();
    auto* w = reinterpret_cast<gklearn::MlpWeights*>(lp);
    auto* lw = reinterpret_cast<LearnWarp*>(lp + sizeof(gklearn::MlpWeights));
    gklearn::load_weights(*w, model);
    stage_init_barriers(sm);  // its barrier also publishes the weights
    const LearnArgs la{w, lw, gate, fired};
    unsigned seq = 0, seq0 = 0;
    stage_tile_tma<NT, KIND, PLM, true>(&mapc, &map0, out, g, ph, c1, c2, c3, tm, rows, blockIdx.x,
                                        blockIdx.y, gridDim.x * gridDim.y, dyn, dyn + kRing * 4 * NT,
                                        sm, seq, seq0, &la);
}

// Persistent stage over an ensemble: tiles[i] = (instance, tile of that
// instance), claimed through *counter (zeroed before the launch).  Stage
// KIND 0 reads A and writes B; KIND 2 reads B and A and writes A.
template <int NT, int KIND, bool PLM>
__global__ void __launch_bounds__(NT, 512 / NT)
    k_ens_stage(const gk::EnsInst* __restrict__ inst, const int2* __restrict__ tiles, int ntiles,
                unsigned* counter, double c1, double c2, double c3) {
    extern __shared__ __align__(128) double dyn[];
    __shared__ StageShared<NT> sm;
    stage_init_barriers(sm);
    unsigned seq = 0, seq0 = 0;
    for (;;) {
        if (threadIdx.x == 0) sm.cur = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int id = sm.cur;
        __syncthreads();
        if (id >= ntiles) break;
        const int2 tl = tiles[id];
        const gk::EnsInst* I = inst + tl.x;
        DevTime* tm = I->tm;
        if (!tm->active) continue;
        const Geom g = I->g;
        const Phys ph = I->ph;
        const int bx = tl.y % I->tiles_x, by = tl.y / I->tiles_x;
        if (KIND == 0)
            stage_tile_tma<NT, KIND, PLM>(&I->mapA, &I->mapA, I->B, g, ph, c1, c2, c3, tm, I->rows,
                                          bx, by, (unsigned)I->tiles, dyn, dyn + kRing * 4 * NT,
                                          sm, seq, seq0);
        else
            stage_tile_tma<NT, KIND, PLM>(&I->mapB, &I->mapA, I->A, g, ph, c1, c2, c3, tm, I->rows,
                                          bx, by, (unsigned)I->tiles, dyn, dyn + kRing * 4 * NT,
                                          sm, seq, seq0);
    }
}

// Ghost fill of every instance: blockIdx.z = instance, blockIdx.y = side
// (x left, x right, y left, y right); which = 0 fills A, 1 fills B.
__global__ void k_ens_bc(const gk::EnsInst* __restrict__ inst, int which) {
    const gk::EnsInst* I = inst + blockIdx.z;
    if (!I->tm->active) return;
    const int dir = blockIdx.y >> 1, side = blockIdx.y & 1;
    const Geom& g = I->g;
    const long long count = (long long)g.ng * (dir == 0 ? g.ny : g.nx);
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= count) return;
    bc_fill_one(which ? I->B : I->A, g, I->ph, dir, side, id);
}

// begin_one (sim.cpp:70-72, 77-81) for every instance of an ensemble.
__global__ void k_ens_begin(const gk::EnsInst* __restrict__ inst, int n, double dtoutput,
                            int steps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) begin_one(inst[i].tm, inst[i].g, inst[i].ph, dtoutput, steps);
}

// ------------------------------------------------------------ launchers
#include "gk_stage3d.cuh"

static inline dim3 cell_grid(const Geom& g, int threads) {
    return dim3((g.nx + threads - 1) / threads, g.ny, g.nz);
}

void launch_bc(const Ctx& c, double* u, cudaStream_t s) {
    const Geom& g = c.g;
    // size the grid for the directions that are filled only
    long long m = 0;
    if (g.nx > 1) m = max(m, (long long)g.ng * g.ny * g.nz);
    if (g.ny > 1) m = max(m, (long long)g.ng * g.nx * g.nz);
    if (g.nz > 1 && c.ph.fill_z) m = max(m, (long long)g.ng * g.nx * g.ny);
    if (m == 0) return;
    const int sides = (g.nz > 1 && c.ph.fill_z) ? 6 : 4;
    dim3 grid((unsigned)((m + 127) / 128), sides);
    k_bc<<<grid, 128, 0, s>>>(u, g, c.ph, c.tm);
    if (c.ph.nshell > 0 && c.ph.shells)
        k_immersed<<<(c.ph.nshell + 127) / 128, 128, 0, s>>>(u, g, c.ph, c.tm);
    if (c.ph.fix_inner && c.ph.inner[1] > c.ph.inner[0] && c.ph.inner[3] > c.ph.inner[2]) {
        dim3 gi((c.ph.inner[1] - c.ph.inner[0] + 127) / 128, c.ph.inner[3] - c.ph.inner[2], g.nz);
        k_fix_inner<<<gi, 128, 0, s>>>(u, g, c.ph, c.tm);
    }
}

void launch_c2p(const Ctx& c, const double* u, double* w, cudaStream_t s) {
    const Geom& g = c.g;
    dim3 grid((g.lenx + 127) / 128, g.leny, g.nzs);
    k_c2p<<<grid, 128, 0, s>>>(u, w, g, c.ph, c.tm);
}

void launch_flux(const Ctx& c, int dir, const double* w, double* F, cudaStream_t s) {
    const Geom& g = c.g;
    int na = dir == 0 ? g.nx + 1 : g.nx;
    int nb = dir == 1 ? g.ny + 1 : g.ny;
    int nc = dir == 2 ? g.nz + 1 : g.nz;
    dim3 grid((na + 127) / 128, nb, nc);
    k_flux<<<grid, 128, 0, s>>>(w, F, g, c.ph, dir, c.tm);
}

void launch_update(const Ctx& c, const double* u0, const double* uc, double* out,
                   const double* F1, const double* F2, const double* F3, int three, double c1,
                   double c2, double c3, cudaStream_t s) {
    k_update<<<cell_grid(c.g, 128), 128, 0, s>>>(u0, uc, out, F1, F2, F3, c.g, c.ph, three, c1, c2,
                                                 c3, c.tm);
}

// 3D stage: rows per CTA segment and the CTA width (64, 96 or 128 threads,
// whichever wastes the fewest lanes on the last strip of columns).
static inline int stage3d_rows(const Geom& g) { return g.ny < 16 ? g.ny : 16; }
static inline int stage3d_nt(const Geom& g) {
    int best = 128;
    long long best_lanes = 1LL << 62;
    for (int nt : {128, 96, 64}) {
        const long long lanes = (long long)((g.nx + nt - 5) / (nt - 4)) * nt;
        if (lanes < best_lanes) {
            best_lanes = lanes;
            best = nt;
        }
    }
    return best;
}

void launch_zflux(const Ctx& c, const double* u, double* F3, cudaStream_t s) {
    const Geom& g = c.g;
    constexpr int zseg = 32;  // faces per thread; nz + 1 faces in all
    dim3 grid((g.nx + kZX - 1) / kZX, (g.ny + kZY - 1) / kZY, (g.nz + 1 + zseg - 1) / zseg);
    if (c.ph.plm) k_zflux<true><<<grid, 128, 0, s>>>(u, F3, g, c.ph, c.tm, zseg);
    else k_zflux<false><<<grid, 128, 0, s>>>(u, F3, g, c.ph, c.tm, zseg);
}

template <int NT>
static void launch_stage3d_nt(const Ctx& c, const double* uc, const double* u0, double* out,
                              const double* F3, int three, double c1, double c2, double c3,
                              cudaStream_t s) {
    const Geom& g = c.g;
    const int rows = stage3d_rows(g);
    dim3 grid((g.nx + NT - 5) / (NT - 4), (g.ny + rows - 1) / rows, g.nz);
#define GK_S3(TH, PL, LA) \
    k_stage3d<NT, TH, PL, LA><<<grid, NT, 0, s>>>(uc, u0, out, F3, g, c.ph, c1, c2, c3, c.tm, rows)
    if (three == 2) {
        if (c.ph.plm) GK_S3(true, true, true);
        else GK_S3(true, false, true);
    } else if (three) {
        if (c.ph.plm) GK_S3(true, true, false);
        else GK_S3(true, false, false);
    } else {
        if (c.ph.plm) GK_S3(false, true, false);
        else GK_S3(false, false, false);
    }
#undef GK_S3
}

void launch_stage3d(const Ctx& c, const double* uc, const double* u0, double* out, const double* F3,
                    int three, double c1, double c2, double c3, cudaStream_t s) {
    switch (stage3d_nt(c.g)) {
        case 64: launch_stage3d_nt<64>(c, uc, u0, out, F3, three, c1, c2, c3, s); break;
        case 96: launch_stage3d_nt<96>(c, uc, u0, out, F3, three, c1, c2, c3, s); break;
        default: launch_stage3d_nt<128>(c, uc, u0, out, F3, three, c1, c2, c3, s); break;
    }
}

void launch_kick(const Ctx& c, double* u, int which, cudaStream_t s) {
    k_kick<<<cell_grid(c.g, 128), 128, 0, s>>>(u, c.g, c.ph, c.tm, which);
}

// Shared memory of k_run1d: primitives and x fluxes of the row.
static size_t run1d_smem(const Geom& g) { return (size_t)(5 * g.lenx + 5 * (g.nx + 1)) * sizeof(double); }

void launch_run1d(const Ctx& c, double* A, double* B, int nsteps, cudaStream_t s) {
    const Geom& g = c.g;
    const int nt = (g.lenx + 31) / 32 * 32;
    const size_t smem = run1d_smem(g);
    static std::atomic<unsigned long long> attr_set{0};
    if (gk::first_on_device(attr_set)) {  // the largest row: lenx 1024
        const int most = (int)((5 * 1024 + 5 * 1021) * sizeof(double));
        cudaFuncSetAttribute(k_run1d<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        cudaFuncSetAttribute(k_run1d<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
    }
    if (c.has_vz) k_run1d<true><<<1, nt, smem, s>>>(A, B, g, c.ph, c.tm, nsteps);
    else k_run1d<false><<<1, nt, smem, s>>>(A, B, g, c.ph, c.tm, nsteps);
}

void launch_cfl(const Ctx& c, const double* u, int epilogue, cudaStream_t s) {
    const Geom& g = c.g;
    long long ncell = (long long)g.nx * g.ny * g.nz;
    int blocks = (int)min((ncell + 255) / 256, (long long)148 * 8);
    if (c.has_vz || g.ndim == 3)
        k_cfl<true><<<blocks, 256, 0, s>>>(u, g, c.ph, c.tm, epilogue);
    else
        k_cfl<false><<<blocks, 256, 0, s>>>(u, g, c.ph, c.tm, epilogue);
}

template <int NT, int KIND, bool PLM>
static void launch_stage2d_tma(const Ctx& c, const CUtensorMap& mc, const CUtensorMap& m0,
                               double* out, double c1, double c2, double c3, cudaStream_t s) {
    const Geom& g = c.g;
    const int rows = c.h2d_rows;
    dim3 grid((g.nx + NT - 5) / (NT - 4), (g.ny + rows - 1) / rows);
    const size_t dyn = stage_dyn_bytes<NT, (KIND >= 1)>();
    static std::atomic<unsigned long long> attr_set{0};
    if (gk::first_on_device(attr_set))
        cudaFuncSetAttribute(k_stage2d_tma<NT, KIND, PLM>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    k_stage2d_tma<NT, KIND, PLM><<<grid, NT, dyn, s>>>(mc, m0, out, g, c.ph, c1, c2, c3, c.tm, rows);
}

template <int NT>
static void launch_stage2d_tma_nt(const Ctx& c, const CUtensorMap& mc, const CUtensorMap& m0,
                                  double* out, int kind, double c1, double c2, double c3,
                                  cudaStream_t s) {
    if (c.ph.plm) {
        if (kind == 0) launch_stage2d_tma<NT, 0, true>(c, mc, m0, out, c1, c2, c3, s);
        else if (kind == 1) launch_stage2d_tma<NT, 1, true>(c, mc, m0, out, c1, c2, c3, s);
        else launch_stage2d_tma<NT, 2, true>(c, mc, m0, out, c1, c2, c3, s);
    } else {
        if (kind == 0) launch_stage2d_tma<NT, 0, false>(c, mc, m0, out, c1, c2, c3, s);
        else if (kind == 1) launch_stage2d_tma<NT, 1, false>(c, mc, m0, out, c1, c2, c3, s);
        else launch_stage2d_tma<NT, 2, false>(c, mc, m0, out, c1, c2, c3, s);
    }
}

template <int NT, int KIND, bool PLM>
static void launch_stage2d_learn_k(const Ctx& c, const CUtensorMap& mc, const CUtensorMap& m0,
                                   double* out, double c1, double c2, double c3, const float* model,
                                   const gk::FluxGate& gate, unsigned* fired, cudaStream_t s) {
    const Geom& g = c.g;
    const int rows = c.learn_rows > 0 ? c.learn_rows : c.h2d_rows;
    dim3 grid((g.nx + NT - 5) / (NT - 4), (g.ny + rows - 1) / rows);
    const size_t dyn = learn_dyn_bytes<NT, (KIND >= 1)>();
    static std::atomic<unsigned long long> attr_set{0};
    if (gk::first_on_device(attr_set))
        cudaFuncSetAttribute(k_stage2d_learn<NT, KIND, PLM>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    k_stage2d_learn<NT, KIND, PLM><<<grid, NT, dyn, s>>>(mc, m0, out, g, c.ph, c1, c2, c3, c.tm, rows,
                                                         model, gate, fired);
}

template <int NT>
static void launch_stage2d_learn_nt(const Ctx& c, const CUtensorMap& mc, const CUtensorMap& m0,
                                    double* out, int kind, double c1, double c2, double c3,
                                    const float* model, const gk::FluxGate& gate, unsigned* fired,
                                    cudaStream_t s) {
#define GK_SL(K, PL) launch_stage2d_learn_k<NT, K, PL>(c, mc, m0, out, c1, c2, c3, model, gate, fired, s)
    if (c.ph.plm) {
        if (kind == 0) GK_SL(0, true);
        else if (kind == 1) GK_SL(1, true);
        else GK_SL(2, true);
    } else {
        if (kind == 0) GK_SL(0, false);
        else if (kind == 1) GK_SL(1, false);
        else GK_SL(2, false);
    }
#undef GK_SL
}

// Adds status bits to the device clock, in stream order (no reference
// counterpart: the reference throws).
__global__ void k_or_status(DevTime* tm, int bits) { tm->status |= bits; }

// The fused stage with the learned correction (TMA rows only; CTAs of 64 or
// 128 threads).  A tensor map that cannot be encoded sets STATUS_NO_MAP:
// the step does not run silently without its correction.
void launch_stage2d_learn(const Ctx& c, const double* uc, const double* u0, double* out, int kind,
                          double c1, double c2, double c3, const float* model,
                          const gk::FluxGate& gate, unsigned* fired, cudaStream_t s) {
    const int nt = c.stage_threads == 64 ? 64 : 128;
    CUtensorMap mc, m0;
    if (!gk::encode_rows_map(&mc, uc, c.g, nt) || !gk::encode_rows_map(&m0, u0 ? u0 : uc, c.g, nt)) {
        std::fprintf(stderr, "gaukuk: tensor map encoding failed for the learned stage\n");
        k_or_status<<<1, 1, 0, s>>>(c.tm, gk::STATUS_NO_MAP);
        return;
    }
    if (nt == 64) launch_stage2d_learn_nt<64>(c, mc, m0, out, kind, c1, c2, c3, model, gate, fired, s);
    else launch_stage2d_learn_nt<128>(c, mc, m0, out, kind, c1, c2, c3, model, gate, fired, s);
}

void launch_stage2d(const Ctx& c, const double* uc, const double* u0, double* out, int kind,
                    double c1, double c2, double c3, cudaStream_t s) {
    const Geom& g = c.g;
    const int rows = c.h2d_rows;
    if (c.use_tma) {
        const int nt = c.stage_threads;
        CUtensorMap mc, m0;
        if (gk::encode_rows_map(&mc, uc, g, nt) && gk::encode_rows_map(&m0, u0 ? u0 : uc, g, nt)) {
            if (nt == 64) launch_stage2d_tma_nt<64>(c, mc, m0, out, kind, c1, c2, c3, s);
            else if (nt == 256) launch_stage2d_tma_nt<256>(c, mc, m0, out, kind, c1, c2, c3, s);
            else launch_stage2d_tma_nt<128>(c, mc, m0, out, kind, c1, c2, c3, s);
            return;
        }
        std::fprintf(stderr, "gaukuk: tensor map encoding failed; using register-staged rows\n");
    }
    dim3 grid((g.nx + kStageCols - 1) / kStageCols, (g.ny + rows - 1) / rows);
#define GK_STAGE(K, PL) k_stage2d<K, PL><<<grid, kStageThreads, 0, s>>>(uc, u0, out, g, c.ph, c1, c2, c3, c.tm, rows)
    if (c.ph.plm) {
        if (kind == 0) GK_STAGE(0, true);
        else if (kind == 1) GK_STAGE(1, true);
        else GK_STAGE(2, true);
    } else {
        if (kind == 0) GK_STAGE(0, false);
        else if (kind == 1) GK_STAGE(1, false);
        else GK_STAGE(2, false);
    }
#undef GK_STAGE
}

template <int NT, int KIND, bool PLM>
static void launch_ens_stage_k(const gk::EnsInst* inst, const int2* tiles, int ntiles,
                               unsigned* counter, double c1, double c2, double c3, int ctas,
                               cudaStream_t s) {
    const size_t dyn = stage_dyn_bytes<NT, (KIND >= 1)>();
    static std::atomic<unsigned long long> attr_set{0};
    if (gk::first_on_device(attr_set))
        cudaFuncSetAttribute(k_ens_stage<NT, KIND, PLM>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    k_ens_stage<NT, KIND, PLM><<<ctas, NT, dyn, s>>>(inst, tiles, ntiles, counter, c1, c2, c3);
}

template <int NT>
static void launch_ens_stage_nt(int kind, int plm, const gk::EnsInst* inst, const int2* tiles,
                                int ntiles, unsigned* counter, double c1, double c2, double c3,
                                cudaStream_t s) {
    const int ctas = std::min(ntiles, 148 * (512 / NT));
    if (plm) {
        if (kind == 0) launch_ens_stage_k<NT, 0, true>(inst, tiles, ntiles, counter, c1, c2, c3, ctas, s);
        else launch_ens_stage_k<NT, 2, true>(inst, tiles, ntiles, counter, c1, c2, c3, ctas, s);
    } else {
        if (kind == 0) launch_ens_stage_k<NT, 0, false>(inst, tiles, ntiles, counter, c1, c2, c3, ctas, s);
        else launch_ens_stage_k<NT, 2, false>(inst, tiles, ntiles, counter, c1, c2, c3, ctas, s);
    }
}

void launch_ens_stage(int threads, int kind, int plm, const gk::EnsInst* inst, const int2* tiles,
                      int ntiles, unsigned* counter, double c1, double c2, double c3,
                      cudaStream_t s) {
    if (threads == 64) launch_ens_stage_nt<64>(kind, plm, inst, tiles, ntiles, counter, c1, c2, c3, s);
    else if (threads == 256) launch_ens_stage_nt<256>(kind, plm, inst, tiles, ntiles, counter, c1, c2, c3, s);
    else launch_ens_stage_nt<128>(kind, plm, inst, tiles, ntiles, counter, c1, c2, c3, s);
}

void launch_ens_bc(const gk::EnsInst* inst, int n, int which, int max_count, cudaStream_t s) {
    dim3 grid((max_count + 127) / 128, 4, n);
    k_ens_bc<<<grid, 128, 0, s>>>(inst, which);
}

void launch_ens_begin(const gk::EnsInst* inst, int n, double dtoutput, int steps, cudaStream_t s) {
    k_ens_begin<<<(n + 63) / 64, 64, 0, s>>>(inst, n, dtoutput, steps);
}

void launch_epilogue(const Ctx& c, cudaStream_t s) { k_epilogue<<<1, 1, 0, s>>>(c.tm, c.g, c.ph); }

void launch_begin(const Ctx& c, double dtoutput, int steps, cudaStream_t s) {
    k_begin<<<1, 1, 0, s>>>(c.tm, c.g, c.ph, dtoutput, steps);
}

void launch_mtz_check(const Ctx& c, const double* u, int* flag, cudaStream_t s) {
    const Geom& g = c.g;
    long long ncell = (long long)g.nx * g.ny * g.nz;
    int blocks = (int)min((ncell + 255) / 256, (long long)148 * 8);
    k_mtz_check<<<blocks, 256, 0, s>>>(u, g, flag);
}

}  // namespace GK_NS
