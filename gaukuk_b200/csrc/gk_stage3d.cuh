// gk_stage3d.cuh -- the 3D RK stage in two kernels (included by
// gk_kernels.cuh inside the mode namespace).
//
// k_zflux: the z-face fluxes of a state into F3.  The reference forms the
// z-face states with ReconstructYZPLM, whose slope is along y
// (recon_piecewise_linear.cpp:29-50): the left state of face (k-1|k) is the
// upper y state of cell (k-1, j), the right state the lower y state of cell
// (k, j).  A thread owns a column (i, j) and marches up a segment of faces,
// converting each plane's three rows to primitives (ConsToPrim,
// adiabatic.cpp:18-61) and sloping them once for the two faces the cell
// touches.
//
// k_stage3d: one z-plane of the stage, as the fused 2D stage does it --
// a CTA owns NT-4 columns plus a 2-cell halo, marches up a segment of rows,
// exchanges x neighbours through shared memory and solves each x and y face
// once -- with all five variables, and adds the z-flux divergence from F3.
// Face states, Riemann solver, flux divergence, RK combine and floors are the
// generic path's expressions (k_c2p, k_flux, k_update), so both paths give
// the same bits.
#pragma once

// PLM face states of one variable from three cells, as k_flux forms them.
__device__ __forceinline__ double plm_up(double a, double b, double c) {
#if GK_FASTMATH
    return b + vanleer_half(b - a, c - b);
#else
    return b + 0.5 * vanleer(b - a, c - b);
#endif
}
__device__ __forceinline__ double plm_down(double a, double b, double c) {
#if GK_FASTMATH
    return b - vanleer_half(b - a, c - b);
#else
    return b - 0.5 * vanleer(b - a, c - b);
#endif
}

struct W5 {
    double v[5];  // primitive slots: rho, vx, vy, p, vz
};

__device__ __forceinline__ W5 c2p_at(const double* __restrict__ u, const Geom& g, const Phys& ph,
                                     long long c) {
    W5 w;
    cons_to_prim5(u[gk::S_DEN * g.vstride + c], u[gk::S_MTX * g.vstride + c],
                  u[gk::S_MTY * g.vstride + c], u[gk::S_MTZ * g.vstride + c],
                  u[gk::S_ENG * g.vstride + c], ph, w.v);
    return w;
}

// Raw conserved values of one cell (slot order), loaded ahead of their use
// so that the loads of the next row are in flight while this row computes.
struct Q5 {
    double q[5];
};
__device__ __forceinline__ Q5 load5(const double* __restrict__ u, const Geom& g, long long c) {
    Q5 r;
#pragma unroll
    for (int v = 0; v < 5; ++v) r.q[v] = __ldg(u + v * g.vstride + c);
    return r;
}
__device__ __forceinline__ W5 c2p_q(const Q5& a, const Phys& ph) {
    W5 w;
    cons_to_prim5(a.q[gk::S_DEN], a.q[gk::S_MTX], a.q[gk::S_MTY], a.q[gk::S_MTZ], a.q[gk::S_ENG], ph,
                  w.v);
    return w;
}

// Riemann problem of an x face (vx | vy, vz) and a y face (vy | vz, vx),
// hllc.cpp:25-27; the fluxes land in slot order (DEN, MTX, MTY, ENG, MTZ).
__device__ __forceinline__ void hllc5_x(const double (&l)[5], const double (&r)[5], const Phys& ph,
                                        double (&F)[5]) {
    Flux5 f;
    hllc<true, kSel>(l[gk::P_RHO], l[gk::P_VX], l[gk::P_VY], l[gk::P_VZ], l[gk::P_PRE], r[gk::P_RHO],
                     r[gk::P_VX], r[gk::P_VY], r[gk::P_VZ], r[gk::P_PRE], ph, f);
    F[gk::S_DEN] = f.d;
    F[gk::S_MTX] = f.n;
    F[gk::S_MTY] = f.t1;
    F[gk::S_MTZ] = f.t2;
    F[gk::S_ENG] = f.e;
}
__device__ __forceinline__ void hllc5_y(const double (&l)[5], const double (&r)[5], const Phys& ph,
                                        double (&F)[5]) {
    Flux5 f;
    hllc<true, kSel>(l[gk::P_RHO], l[gk::P_VY], l[gk::P_VZ], l[gk::P_VX], l[gk::P_PRE], r[gk::P_RHO],
                     r[gk::P_VY], r[gk::P_VZ], r[gk::P_VX], r[gk::P_PRE], ph, f);
    F[gk::S_DEN] = f.d;
    F[gk::S_MTY] = f.n;
    F[gk::S_MTZ] = f.t1;
    F[gk::S_MTX] = f.t2;
    F[gk::S_ENG] = f.e;
}

// ------------------------------------------------------------ z faces
// Flux::CalFlux's z sweep (cal_flux.cpp:140-156; first order 72-87): PLM states and HLLC at
// every z face.  A CTA of 128 threads owns a tile of 32 columns x 4 rows of z faces and
// marches up a segment of zseg faces; a thread owns column (i, j) of the
// tile.  Per plane the CTA converts the tile's 6 rows (the 4 rows and one
// halo row below and above) once, 1.5 cells per face instead of the 3 a
// thread converting its own rows j-1, j, j+1 would, into a double-buffered
// shared array; the raw values of the next plane are in flight while a face
// is solved.  The y-slope of cell (k, j) gives both its lower state (the
// right state of face k-1|k) and its upper state (the left state of face
// k|k+1).  The expressions are plm_up / plm_down's, so the fluxes are the
// same bits.
constexpr int kZX = 32, kZY = 4, kZRows = kZY + 2, kZCells = kZX * kZRows;

template <bool PLM>
__global__ void __launch_bounds__(128)
    k_zflux(const double* __restrict__ u, double* __restrict__ F3, Geom g, Phys ph,
            const DevTime* __restrict__ tm, int zseg) {
    if (!tm->active) return;
    __shared__ double sW[2][kZRows][5][kZX];
    const int t = threadIdx.x, tx = t & (kZX - 1), ty = t / kZX;
    const int i = g.ib + blockIdx.x * kZX + tx;
    const int j = g.jb + blockIdx.y * kZY + ty;
    const bool mine = i < g.ie && j < g.je;
    const int k0 = g.kb + blockIdx.z * zseg;    // first face (k0-1 | k0)
    const int k1 = min(k0 + zseg, g.ke + 1);    // one past the last face
    // the cells this thread loads: m = t and m = t + 128 (< 192) of the tile's
    // 6 x 32 cells, rows j0-1 .. j0+4 (clamped into the array: rows and
    // columns past the grid feed no face of this tile)
    const int j0 = g.jb + blockIdx.y * kZY;
    auto cell_of = [&](int m) {
        const int row = min(j0 - 1 + m / kZX, g.leny - 1);
        const int col = min(g.ib + blockIdx.x * kZX + (m % kZX), g.lenx - 1);
        return sidx(g, g.kb, row, col) - sidx(g, g.kb, 0, 0);  // offset within a plane
    };
    const long long off0 = cell_of(t);
    const bool two = t + 128 < kZCells;
    const long long off1 = two ? cell_of(t + 128) : off0;
    auto load = [&](int k, Q5& a, Q5& b) {
        const long long base = sidx(g, k, 0, 0);
        a = load5(u, g, base + off0);
        if (two) b = load5(u, g, base + off1);
    };
    auto put = [&](int buf, int m, const Q5& q) {
        const W5 w = c2p_q(q, ph);
#pragma unroll
        for (int v = 0; v < 5; ++v) sW[buf][m / kZX][v][m % kZX] = w.v[v];
    };
    // states of cell (k, j) from the tile's rows ty, ty+1, ty+2 (= j-1, j, j+1)
    auto states = [&](int buf, double (&lo)[5], double (&up)[5]) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double b = sW[buf][ty + 1][v][tx];
            if (PLM) {
                const double a = sW[buf][ty][v][tx], c = sW[buf][ty + 2][v][tx];
#if GK_FASTMATH
                const double h = vanleer_half(b - a, c - b);
#else
                const double h = 0.5 * vanleer(b - a, c - b);
#endif
                lo[v] = b - h;
                up[v] = b + h;
            } else {
                lo[v] = up[v] = b;
            }
        }
    };
    Q5 qa, qb;
    double wl[5], wr[5], nu[5];
    load(k0 - 1, qa, qb);
    put(0, t, qa);
    if (two) put(0, t + 128, qb);
    load(k0, qa, qb);
    __syncthreads();
    states(0, wr, wl);  // the upper state of plane k0-1 is the first face's left state
    int buf = 1;
    for (int k = k0; k < k1; ++k) {
        put(buf, t, qa);
        if (two) put(buf, t + 128, qb);
        if (k + 1 < k1) load(k + 1, qa, qb);
        __syncthreads();  // plane k in sW[buf]; sW[buf ^ 1] is free for plane k+1
        states(buf, wr, nu);
        if (mine) {
            // z face: (vz | vx, vy)
            Flux5 f;
            hllc<true, kSel>(wl[gk::P_RHO], wl[gk::P_VZ], wl[gk::P_VX], wl[gk::P_VY],
                             wl[gk::P_PRE], wr[gk::P_RHO], wr[gk::P_VZ], wr[gk::P_VX],
                             wr[gk::P_VY], wr[gk::P_PRE], ph, f);
            const long long c = fidx(g, k, j, i);
            F3[gk::S_DEN * g.fvstride + c] = f.d;
            F3[gk::S_MTZ * g.fvstride + c] = f.n;
            F3[gk::S_MTX * g.fvstride + c] = f.t1;
            F3[gk::S_MTY * g.fvstride + c] = f.t2;
            F3[gk::S_ENG * g.fvstride + c] = f.e;
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) wl[v] = nu[v];
        buf ^= 1;
    }
}

// ------------------------------------------------------------ x-y plane stage
// THREE = false: out = c1*uc - c2*dF (stage 1); true: out = c1*u0 + c2*uc -
// c3*dF.  out never aliases uc (neighbours of uc are read while out is
// written); u0 may alias out (read pointwise, before the write).  LAST: the
// step's last stage also reduces the CFL speed of the new state (CalCmax,
// adiabatic.cpp:115-160, on the values it writes) and its last CTA runs the
// step epilogue, as k_cfl would after it.
// Resident threads per SM: 384 in fast mode (up to 168 registers each), 512
// in parity mode (128 registers, with 16-72 bytes of spills).  At 256^3 (CTAs of 96) parity
// mode went from 5.39 to 5.13 ms per step with the extra warps, while fast
// mode, whose early row loads need the registers, went from 2.28 to 2.42.
constexpr int kStage3dThreadsPerSM = GK_FASTMATH ? 384 : 512;
template <int NT, bool THREE, bool PLM, bool LAST>
__global__ void __launch_bounds__(NT, kStage3dThreadsPerSM / NT)
    k_stage3d(const double* __restrict__ uc, const double* u0, double* out,
              const double* __restrict__ F3, Geom g, Phys ph, double c1, double c2, double c3,
              DevTime* tm, int rows) {
    if (!tm->active) return;
    unsigned long long cbest = 0ull;  // CFL speed of this thread's cells (bit pattern)
    __shared__ double sP[5][NT];
    __shared__ double sXL[5][NT];
    __shared__ double sF[5][NT];
    const double dt = tm->dt;
    const double dtdx = dt * g.dxRec, dtdy = dt * g.dyRec, dtdz = dt * g.dzRec;
    const int t = threadIdx.x;
    const int tl = t > 0 ? t - 1 : 0;
    const int tr = t < NT - 1 ? t + 1 : t;
    const int xi = g.ib - 2 + blockIdx.x * (NT - 4) + t;
    const int xl = xi < g.lenx ? xi : g.lenx - 1;  // clamped load column
    const bool do_cell = t >= 2 && t <= NT - 3 && xi < g.ie;
    const int k = g.kb + blockIdx.z;
    const int y0 = g.jb + blockIdx.y * rows;
    const int y1 = min(y0 + rows, g.je);
    auto at = [&](int j) { return sidx(g, k, j, xl); };

    // primitives of rows y0-2, y0-1, y0 and y0+1
    const W5 Pm2 = c2p_at(uc, g, ph, at(y0 - 2));
    W5 Pm1 = c2p_at(uc, g, ph, at(y0 - 1));
    W5 P0 = c2p_at(uc, g, ph, at(y0));
    double wlNext[5], fyPrev[5];
    // lower state of y face y0 (upper y state of cell y0-1), then that face
    {
        const W5 P1 = c2p_at(uc, g, ph, at(y0 + 1));
        double wr[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            wlNext[v] = PLM ? plm_up(Pm2.v[v], Pm1.v[v], P0.v[v]) : Pm1.v[v];
            wr[v] = PLM ? plm_down(Pm1.v[v], P0.v[v], P1.v[v]) : P0.v[v];
        }
        hllc5_y(wlNext, wr, ph, fyPrev);
#pragma unroll
        for (int v = 0; v < 5; ++v) wlNext[v] = PLM ? plm_up(Pm1.v[v], P0.v[v], P1.v[v]) : P0.v[v];
        Pm1 = P0;
        P0 = P1;
    }
    // row f: the x faces of cell row f-1 and the y face f above it; update row f-1.
    // The raw row f+2 is loaded one row ahead of its conversion.
    Q5 Qn = load5(uc, g, at(y0 + 2));
    for (int f = y0 + 1; f <= y1; ++f) {
        const Q5 Q1 = Qn;
        if (f + 2 <= y1 + 1) Qn = load5(uc, g, at(f + 2));
        // fast mode: the z fluxes below and above cell row f-1, and its base
        // state, are loaded here so that they arrive while the row's Riemann
        // problems are solved (parity mode's longer IEEE sequences leave no
        // registers for them: it loads them where they are used)
        double zlo[5], zhi[5], b0[5];
        constexpr bool kEarly = GK_FASTMATH;
        auto load_row_inputs = [&]() {
            const long long fc = fidx(g, k, f - 1, xi);
            const long long c = at(f - 1);
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                zlo[v] = __ldg(F3 + v * g.fvstride + fc);
                zhi[v] = __ldg(F3 + v * g.fvstride + fc + g.fkstride);
                b0[v] = THREE ? u0[v * g.vstride + c] : uc[v * g.vstride + c];
            }
        };
        if (kEarly && do_cell) load_row_inputs();
        const W5 P1 = c2p_q(Q1, ph);
#pragma unroll
        for (int v = 0; v < 5; ++v) sP[v][t] = Pm1.v[v];
        __syncthreads();
        double xr[5], wr[5], wlNew[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double a = sP[v][tl], c = sP[v][tr];
            if (PLM) {
                sXL[v][t] = plm_up(a, Pm1.v[v], c);
                xr[v] = plm_down(a, Pm1.v[v], c);
                wr[v] = plm_down(Pm1.v[v], P0.v[v], P1.v[v]);
                wlNew[v] = plm_up(Pm1.v[v], P0.v[v], P1.v[v]);
            } else {
                sXL[v][t] = Pm1.v[v];
                xr[v] = Pm1.v[v];
                wr[v] = P0.v[v];
                wlNew[v] = P0.v[v];
            }
        }
        __syncthreads();
        double xlst[5], fx[5], fy[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) xlst[v] = sXL[v][tl];
        hllc5_x(xlst, xr, ph, fx);
        hllc5_y(wlNext, wr, ph, fy);
#pragma unroll
        for (int v = 0; v < 5; ++v) sF[v][t] = fx[v];
        __syncthreads();
        if (do_cell) {
            // update_cons.cpp (3D): (Fx(i+1)-Fx(i))*dtdx + (Fy(j+1)-Fy(j))*dtdy + (Fz(k+1)-Fz(k))*dtdz
            if (!kEarly) load_row_inputs();
            const long long c = at(f - 1);
            double r[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                double dF = (sF[v][tr] - fx[v]) * dtdx;
                dF = dF + (fy[v] - fyPrev[v]) * dtdy + (zhi[v] - zlo[v]) * dtdz;
                if (THREE) r[v] = c1 * b0[v] + c2 * uc[v * g.vstride + c] - c3 * dF;
                else r[v] = c1 * b0[v] - c2 * dF;
            }
            floors5(r, ph, tm);
            if (LAST) {
                const double local = cell_cmax(r[gk::S_DEN], r[gk::S_MTX], r[gk::S_MTY],
                                               r[gk::S_MTZ], r[gk::S_ENG], ph, true);
                const unsigned long long b = (unsigned long long)__double_as_longlong(local);
                cbest = b > cbest ? b : cbest;
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) out[v * g.vstride + c] = r[v];
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            fyPrev[v] = fy[v];
            wlNext[v] = wlNew[v];
        }
        Pm1 = P0;
        P0 = P1;
    }    if (LAST) {
        __shared__ unsigned long long wmax[NT / 32];
        __shared__ int last;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, cbest, o);
            cbest = x > cbest ? x : cbest;
        }
        if ((t & 31) == 0) wmax[t >> 5] = cbest;
        __syncthreads();
        if (t == 0) {
            unsigned long long m = wmax[0];
            for (int w = 1; w < NT / 32; ++w) m = wmax[w] > m ? wmax[w] : m;
            atomicMax(&tm->cmax_acc, m);
            __threadfence();
            const unsigned total = gridDim.x * gridDim.y * gridDim.z;
            last = atomicAdd(&tm->done_ctas, 1u) == total - 1;
        }
        __syncthreads();
        if (last && t == 0) {
            __threadfence();
            step_epilogue(tm, g, ph, 1);
        }
    }
}
