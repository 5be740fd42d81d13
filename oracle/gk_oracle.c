/*
 * gk_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the Gaukuk
 * finite-volume update: a plain-C restatement of the reference algorithm,
 * function by function, in the reference's own operation order so that a
 * build with strict IEEE flags (-ffp-contract=off, no -ffast-math) gives the
 * same bits as the reference built with the same flags.
 *
 * Each function cites the reference file:line it restates (paths relative to
 * the ShunqH/Gaukuk project root).  The checker role is documented in
 * gk_oracle.h; the restatement is pinned against the reference build
 * (oracle/_ref) and the golden vectors under tests/golden/.
 *
 * Scope: 1D/2D/3D, boundary types 0-3, Euler/RK2/RK3, first order and PLM,
 * constant gravity.  Fixed (type 4) boundaries, point/binary gravity and the
 * immersed body are not restated (the CUDA path does not implement them).
 */
#include "gk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { DEN = 0, MTX = 1, MTY = 2, MTZ = 3, ENG = 4 };
enum { VLX = 1, VLY = 2, VLZ = 3, PRE = 4 };
#define NVAR 5

/* libstdc++ std::max / std::min as the reference calls them (adiabatic.cpp:49,
 * 153-156; sim.cpp:35): max(a,b) = (a<b)?b:a, min(a,b) = (b<a)?b:a */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }

struct gko_sim {
    gko_params p;
    int lenx, leny, lenz;
    int ib, ie, jb, je, kb, ke;
    double dx, dy, dz, dxRec, dyRec, dzRec, drmin;
    double gm1Rec;
    double *cons, *consTemp, *prim, *flx1, *flx2, *flx3;
    int step, isContinue, has_src;
    double t, dt, dtUntilOutput, cmax;
    /* a y-slab of a split grid (gko_advance_split): fills the type-5 sides */
    gko_halo_fn halo;
    void* halo_user;
};

/* TArray index (template_array.hpp:67-72) for dims (NVAR, n3, n2, n1). */
static inline size_t ix4(int n1, int n2, int n3, int n, int k, int j, int i) {
    return (size_t)i + (size_t)n1 * ((size_t)j + (size_t)n2 * ((size_t)k + (size_t)n3 * (size_t)n));
}
#define C(a, n, k, j, i) (a)[ix4(s->lenx, s->leny, s->lenz, (n), (k), (j), (i))]
#define F1(n, k, j, i) s->flx1[ix4(s->lenx + 1, s->leny, s->lenz, (n), (k), (j), (i))]
#define F2(n, k, j, i) s->flx2[ix4(s->lenx, s->leny + 1, s->lenz, (n), (k), (j), (i))]
#define F3(n, k, j, i) s->flx3[ix4(s->lenx, s->leny, s->lenz + 1, (n), (k), (j), (i))]

long long gko_state_size(const gko_sim* s) {
    return (long long)NVAR * s->lenx * s->leny * s->lenz;
}

/* Grid (grid.hpp:18-41), Domain (sim.cpp:16-42), Sim::Sim (sim.cpp:45-67). */
gko_sim* gko_create(const gko_params* p) {
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->ng < 2) return NULL;
    for (int b = 0; b < 6; ++b)
        if (p->bc[b] == 4) return NULL; /* fixed boundaries are not restated */
    gko_sim* s = (gko_sim*)calloc(1, sizeof(gko_sim));
    s->p = *p;
    s->lenx = p->nx + 2 * p->ng;
    s->leny = p->ny + 2 * p->ng;
    s->lenz = p->nz + 2 * p->ng;
    s->ib = p->ng; s->ie = s->ib + p->nx;
    s->jb = p->ng; s->je = s->jb + p->ny;
    s->kb = p->ng; s->ke = s->kb + p->nz;
    s->dx = (p->xmax - p->xmin) / p->nx;
    s->dy = (p->ymax - p->ymin) / p->ny;
    s->dz = (p->zmax - p->zmin) / p->nz;
    s->dxRec = 1. / s->dx;
    s->dyRec = 1. / s->dy;
    s->dzRec = 1. / s->dz;
    if (p->ny <= 1) s->dyRec = 0;
    if (p->nz <= 1) s->dzRec = 0;
    s->drmin = smin(smin(s->dx, s->dy), s->dz);
    s->gm1Rec = 1.0 / (p->gamma - 1.0);
    size_t n = (size_t)gko_state_size(s);
    s->cons = (double*)calloc(n, sizeof(double));
    s->consTemp = (double*)calloc(n, sizeof(double));
    s->prim = (double*)calloc(n, sizeof(double));
    s->flx1 = (double*)calloc((size_t)NVAR * (s->lenx + 1) * s->leny * s->lenz, sizeof(double));
    s->flx2 = (double*)calloc((size_t)NVAR * s->lenx * (s->leny + 1) * s->lenz, sizeof(double));
    s->flx3 = (double*)calloc((size_t)NVAR * s->lenx * s->leny * (s->lenz + 1), sizeof(double));
    s->isContinue = 1;
    s->step = 0;
    s->t = 0;
    s->dt = 1e10;
    s->dtUntilOutput = 1e10;
    s->cmax = 1e-16;
    /* SourceTerm::EnrollConstGravityVector (source.cpp:23-31) */
    s->has_src = (p->grav[0] != 0 || p->grav[1] != 0 || p->grav[2] != 0);
    return s;
}

/* Sim's arrays freed (~TArray, template_array.hpp:89-91). */
void gko_destroy(gko_sim* s) {
    if (!s) return;
    free(s->cons); free(s->consTemp); free(s->prim);
    free(s->flx1); free(s->flx2); free(s->flx3);
    free(s);
}

/* Sim::cons as a setup hook leaves it (main.cpp:25-30), and as Sim::WriteData
 * reads it (write_sim.cpp:14-58); the clock as Sim::GetTime / Getdt / GetStep
 * and isContinue give it (sim.hpp:26, 43-45).  gko_set_time has no reference
 * counterpart (t and step are private, sim.hpp:48-49): restarts use it. */
void gko_set_cons(gko_sim* s, const double* cons) {
    memcpy(s->cons, cons, sizeof(double) * (size_t)gko_state_size(s));
}
void gko_get_cons(const gko_sim* s, double* cons) {
    memcpy(cons, s->cons, sizeof(double) * (size_t)gko_state_size(s));
}
double gko_time(const gko_sim* s) { return s->t; }
double gko_dt(const gko_sim* s) { return s->dt; }
int gko_step(const gko_sim* s) { return s->step; }
int gko_is_continue(const gko_sim* s) { return s->isContinue; }
void gko_set_time(gko_sim* s, double t, int step) { s->t = t; s->step = step; }

/* ---------------------------------------------------------------- EOS --- */

/* EquationOfState::ConsToPrim (adiabatic.cpp:18-61): all i,j (ghosts too),
 * active k only when nz == 1. */
static void cons_to_prim(gko_sim* s, const double* u) {
    int kl = 0, kr = s->lenz;
    if (s->p.nz == 1) { kl = s->kb; kr = s->ke; }
    const double gm1 = s->p.gamma - 1.0;
    const double dmin = s->p.dfloor, pmin = s->p.pfloor;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = kl; k < kr; k++)
        for (int j = 0; j < s->leny; j++)
            for (int i = 0; i < s->lenx; i++) {
                double d = C(u, DEN, k, j, i);
                double mx = C(u, MTX, k, j, i);
                double my = C(u, MTY, k, j, i);
                double mz = C(u, MTZ, k, j, i);
                double e = C(u, ENG, k, j, i);
                d = smax(d, dmin);
                C(s->prim, DEN, k, j, i) = d;
                double denInv = 1.0 / d;
                C(s->prim, VLX, k, j, i) = mx * denInv;
                C(s->prim, VLY, k, j, i) = my * denInv;
                C(s->prim, VLZ, k, j, i) = mz * denInv;
                double engKin = 0.5 * denInv * (mx * mx + my * my + mz * mz);
                double pre = gm1 * (e - engKin);
                C(s->prim, PRE, k, j, i) = (pre > pmin) ? pre : pmin;
            }
}

/* EquationOfState::CalCmax (adiabatic.cpp:115-160), seeded with 1e-16 as
 * Sim::Advance does (sim.cpp:77).  Max is order independent, so the OpenMP
 * reduction is exact. */
double gko_cmax(const gko_sim* s) {
    const double gm1 = s->p.gamma - 1.0;
    const double gamma = s->p.gamma;
    const double dmin = s->p.dfloor, pmin = s->p.pfloor;
    double cmax = 1e-16;
    const double* u = s->cons;
    #pragma omp parallel for collapse(2) reduction(max : cmax) schedule(static)
    for (int k = s->kb; k < s->ke; k++)
        for (int j = s->jb; j < s->je; j++)
            for (int i = s->ib; i < s->ie; i++) {
                double d = C(u, DEN, k, j, i);
                double mx = C(u, MTX, k, j, i);
                double my = C(u, MTY, k, j, i);
                double mz = C(u, MTZ, k, j, i);
                double e = C(u, ENG, k, j, i);
                d = smax(d, dmin);
                double denInv = 1.0 / d;
                double vx = mx * denInv, vy = my * denInv, vz = mz * denInv;
                double engKin = 0.5 * (vx * mx + vy * my + vz * mz);
                double pres = gm1 * (e - engKin);
                pres = (pres > pmin) ? pres : pmin;
                double cs = sqrt(gamma * pres * denInv);
                double local = fabs(vx) + cs;
                local = smax(local, fabs(vy) + cs);
                local = smax(local, fabs(vz) + cs);
                cmax = smax(cmax, local);
            }
    return cmax;
}

/* The per-cell body of EquationOfState::ConsToPrim (adiabatic.cpp:49-57) over
 * n cells of planar arrays, for tests of single cells. */
void gko_cons_to_prim_batch(int n, const double* cons, double gamma,
                            double dfloor, double pfloor, double* prim) {
    const double gm1 = gamma - 1.0;
    for (int c = 0; c < n; ++c) {
        double d = cons[0 * n + c], mx = cons[1 * n + c], my = cons[2 * n + c];
        double mz = cons[3 * n + c], e = cons[4 * n + c];
        d = smax(d, dfloor);
        prim[0 * n + c] = d;
        double denInv = 1.0 / d;
        prim[1 * n + c] = mx * denInv;
        prim[2 * n + c] = my * denInv;
        prim[3 * n + c] = mz * denInv;
        double engKin = 0.5 * denInv * (mx * mx + my * my + mz * mz);
        double pre = gm1 * (e - engKin);
        prim[4 * n + c] = (pre > pfloor) ? pre : pfloor;
    }
}

/* ------------------------------------------------------ reconstruction --- */

/* Reconstruction::VanLeer (reconstruction.hpp:36-42). */
static inline double vanleer(double a, double b) {
    double multi = a * b;
    double sigma = 2.0 * multi / (a + b);
    return (multi <= 0.0) ? 0.0 : sigma;
}

/* Reconstruction::VanLeer (reconstruction.hpp:36-42) over n slope pairs. */
void gko_vanleer_batch(int n, const double* a, const double* b, double* out) {
    for (int c = 0; c < n; ++c) out[c] = vanleer(a[c], b[c]);
}

/* ------------------------------------------------------------- HLLC ----- */

/* Flux::RiemannSolver for one interface (hllc.cpp:22-101).  wl/wr hold
 * DEN,VLX,VLY,VLZ,PRE; dir is VLX/VLY/VLZ.  f receives the flux in the
 * reference's slots DEN, IVLX, IVLY, IVLZ, ENG (hllc.cpp:95-99). */
static inline void hllc(const double wl[5], const double wr[5], int dir,
                        double gamma, double gm1Rec, double f[5]) {
    const int IVLX = VLX + (dir - VLX + 0) % 3;
    const int IVLY = VLX + (dir - VLX + 1) % 3;
    const int IVLZ = VLX + (dir - VLX + 2) % 3;
    const double gmRec = 1.0 / gamma;

    double denl = wl[DEN], vxl = wl[IVLX], vyl = wl[IVLY], vzl = wl[IVLZ], prel = wl[PRE];
    double denr = wr[DEN], vxr = wr[IVLX], vyr = wr[IVLY], vzr = wr[IVLZ], prer = wr[PRE];

    /* EquationOfState::SoundSpeed (eos.hpp:27-29) */
    double al = sqrt(gamma * prel / denl);
    double ar = sqrt(gamma * prer / denr);
    double prePVRS = 0.5 * (prel + prer) - 0.125 * (vxr - vxl) * (denl + denr) * (al + ar);
    prePVRS = smax(prePVRS, 0.0);

    double temp = smax(prePVRS / prel - 1, 0.0);
    double ql = sqrt(1 + 0.5 * (1 + gmRec) * temp);
    temp = smax(prePVRS / prer - 1, 0.0);
    double qr = sqrt(1 + 0.5 * (1 + gmRec) * temp);

    double sl = vxl - al * ql;
    double sr = vxr + ar * qr;
    double ss = (prer - prel + denl * vxl * (sl - vxl) - denr * vxr * (sr - vxr)) /
                (denl * (sl - vxl) - denr * (sr - vxr));

    /* EquationOfState::EGas (eos.hpp:30-32) */
    double el = prel * gm1Rec + 0.5 * denl * (vxl * vxl + vyl * vyl + vzl * vzl);
    double er = prer * gm1Rec + 0.5 * denr * (vxr * vxr + vyr * vyr + vzr * vzr);

    double cl = smin(0.0, sl) * (ss - vxl) / (sl - ss);
    double cr = smax(0.0, sr) * (ss - vxr) / (sr - ss);
    double selectl = (ss >= 0) ? 1.0 : 0.0;
    double selectr = 1.0 - selectl;

    double fl1 = denl * (vxl + cl);
    double fl2 = denl * (vxl * vxl + cl * sl) + prel;
    double fl3 = fl1 * vyl;
    double fl4 = fl1 * vzl;
    double fl5 = (el + prel) * (vxl + cl) + denl * cl * ss * (sl - vxl);

    double fr1 = denr * (vxr + cr);
    double fr2 = denr * (vxr * vxr + cr * sr) + prer;
    double fr3 = fr1 * vyr;
    double fr4 = fr1 * vzr;
    double fr5 = (er + prer) * (vxr + cr) + denr * cr * ss * (sr - vxr);

    f[DEN] = selectl * fl1 + selectr * fr1;
    f[IVLX] = selectl * fl2 + selectr * fr2;
    f[IVLY] = selectl * fl3 + selectr * fr3;
    f[IVLZ] = selectl * fl4 + selectr * fr4;
    f[ENG] = selectl * fl5 + selectr * fr5;
}

/* Flux::RiemannSolver (hllc.cpp:22-101) over n interfaces of planar states. */
void gko_hllc_batch(int n, const double* wl, const double* wr, int dir,
                    double gamma, double* flux) {
    const double gm1Rec = 1.0 / (gamma - 1.0);
    for (int c = 0; c < n; ++c) {
        double l[5], r[5], f[5];
        for (int v = 0; v < 5; ++v) { l[v] = wl[v * n + c]; r[v] = wr[v * n + c]; }
        hllc(l, r, dir, gamma, gm1Rec, f);
        for (int v = 0; v < 5; ++v) flux[v * n + c] = f[v];
    }
}

/* Face states at the face between cells (m) and (p) along one direction,
 * given the four prims around it.  PLM: Reconstruction::ReconstructXPLM /
 * ReconstructYZPLM (recon_piecewise_linear.cpp:8-50): ul = u2 + 0.5*sigma of
 * the left cell, ur = u2 - 0.5*sigma of the right cell.  First order:
 * recon_first_order.cpp:8-28. */
static inline void face_states(const gko_sim* s, int plm,
                               const double* q0, const double* q1,
                               const double* q2, const double* q3,
                               double wl[5], double wr[5]) {
    (void)s;
    for (int n = 0; n < NVAR; ++n) {
        if (plm) {
            double sl = vanleer(q1[n] - q0[n], q2[n] - q1[n]);
            double sr = vanleer(q2[n] - q1[n], q3[n] - q2[n]);
            wl[n] = q1[n] + 0.5 * sl;
            wr[n] = q2[n] - 0.5 * sr;
        } else {
            wl[n] = q1[n];
            wr[n] = q2[n];
        }
    }
}

/* Flux::CalFlux (cal_flux.cpp:13-160).  Only the faces that UpdateCons reads
 * are evaluated; each one sees exactly the reference's inputs. */
static void cal_flux(gko_sim* s) {
    const int plm = (s->p.rc_order != 1);
    const double gamma = s->p.gamma, gm1Rec = s->gm1Rec;
    const double* P = s->prim;
    /* x sweep: active rows, faces ib..ie (cal_flux.cpp:89-101) */
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = s->kb; k < s->ke; k++)
        for (int j = s->jb; j < s->je; j++)
            for (int i = s->ib; i <= s->ie; i++) {
                double q[4][5], wl[5], wr[5], f[5];
                for (int c = 0; c < 4; ++c)
                    for (int n = 0; n < NVAR; ++n) q[c][n] = C(P, n, k, j, i - 2 + c);
                face_states(s, plm, q[0], q[1], q[2], q[3], wl, wr);
                hllc(wl, wr, VLX, gamma, gm1Rec, f);
                for (int n = 0; n < NVAR; ++n) F1(n, k, j, i) = f[n];
            }
    /* y sweep: faces jb..je on active columns (cal_flux.cpp:103-139) */
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = s->kb; k < s->ke; k++)
        for (int j = s->jb; j <= s->je; j++)
            for (int i = s->ib; i < s->ie; i++) {
                double q[4][5], wl[5], wr[5], f[5];
                for (int c = 0; c < 4; ++c)
                    for (int n = 0; n < NVAR; ++n) q[c][n] = C(P, n, k, j - 2 + c, i);
                face_states(s, plm, q[0], q[1], q[2], q[3], wl, wr);
                hllc(wl, wr, VLY, gamma, gm1Rec, f);
                for (int n = 0; n < NVAR; ++n) F2(n, k, j, i) = f[n];
            }
    if (s->p.nz == 1) return;
    /* z sweep (3D only): faces kb..ke on active (j,i) (cal_flux.cpp:140-156).
     * The reference builds the z-face states with ReconstructYZPLM, whose
     * stencil is j-1, j, j+1 at fixed k (recon_piecewise_linear.cpp:29-50):
     * the left state is P(k-1,j) + 0.5*sigma_y(k-1,j) and the right state
     * P(k,j) - 0.5*sigma_y(k,j).  That y-slope is restated as is. */
    #pragma omp parallel for collapse(2) schedule(static)
    for (int j = s->jb; j < s->je; j++)
        for (int k = s->kb; k <= s->ke; k++)
            for (int i = s->ib; i < s->ie; i++) {
                double wl[5], wr[5], f[5];
                for (int n = 0; n < NVAR; ++n) {
                    double l1 = C(P, n, k - 1, j - 1, i), l2 = C(P, n, k - 1, j, i);
                    double l3 = C(P, n, k - 1, j + 1, i);
                    double r1 = C(P, n, k, j - 1, i), r2 = C(P, n, k, j, i);
                    double r3 = C(P, n, k, j + 1, i);
                    if (plm) {
                        wl[n] = l2 + 0.5 * vanleer(l2 - l1, l3 - l2);
                        wr[n] = r2 - 0.5 * vanleer(r2 - r1, r3 - r2);
                    } else {
                        wl[n] = l2;
                        wr[n] = r2;
                    }
                }
                hllc(wl, wr, VLZ, gamma, gm1Rec, f);
                for (int n = 0; n < NVAR; ++n) F3(n, k, j, i) = f[n];
            }
}

/* ------------------------------------------------------------- update --- */

/* Sim::UpdateCons, both overloads (update_cons.cpp:11-133 and 135-269).
 * three_coef = 0: out = c1*u - c2*dF; three_coef = 1: out = c1*u + c2*out - c3*dF. */
static void update_cons(gko_sim* s, const double* u, double* ut, int three_coef,
                        double c1, double c2, double c3) {
    const double dtdx = s->dt * s->dxRec;
    const double dtdy = s->dt * s->dyRec;
    const double dtdz = s->dt * s->dzRec;
    const double dmin = s->p.dfloor, pmin = s->p.pfloor;
    const double gm1 = s->p.gamma - 1;
    const int is3d = (s->p.nz != 1);
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = s->kb; k < s->ke; k++)
        for (int j = s->jb; j < s->je; j++)
            for (int i = s->ib; i < s->ie; i++) {
                double r[NVAR];
                for (int n = 0; n < NVAR; ++n) {
                    double dF;
                    if (!is3d)
                        dF = (F1(n, k, j, i + 1) - F1(n, k, j, i)) * dtdx
                           + (F2(n, k, j + 1, i) - F2(n, k, j, i)) * dtdy;
                    else
                        dF = (F1(n, k, j, i + 1) - F1(n, k, j, i)) * dtdx
                           + (F2(n, k, j + 1, i) - F2(n, k, j, i)) * dtdy
                           + (F3(n, k + 1, j, i) - F3(n, k, j, i)) * dtdz;
                    if (three_coef)
                        r[n] = c1 * C(u, n, k, j, i) + c2 * C(ut, n, k, j, i) - c3 * dF;
                    else
                        r[n] = c1 * C(u, n, k, j, i) - c2 * dF;
                }
                if (r[DEN] < dmin) {
                    r[DEN] = dmin;
                    r[MTX] = 0.0;
                    r[MTY] = 0.0;
                    r[MTZ] = 0.0;
                    r[ENG] = pmin / gm1 + 0.0;
                } else {
                    double inv_den = 1.0 / r[DEN];
                    double ke = 0.5 * inv_den * (r[MTX] * r[MTX] + r[MTY] * r[MTY] + r[MTZ] * r[MTZ]);
                    double press = gm1 * (r[ENG] - ke);
                    if (press < pmin) r[ENG] = pmin / gm1 + ke;
                }
                for (int n = 0; n < NVAR; ++n) C(ut, n, k, j, i) = r[n];
            }
}

/* ----------------------------------------------------------- boundary --- */

/* One ghost-fill routine of boundary/{outflow_copy,periodic,reflective,
 * outflow}.cpp for direction d (0 x, 1 y, 2 z), side (0 left, 1 right) and
 * type (0 copy, 1 periodic, 2 reflective, 3 outflow): OutflowCopyXL..ZR
 * (outflow_copy.cpp:16-182), PeriodicXL..ZR (periodic.cpp:19-191),
 * ReflectiveXL..ZR (reflective.cpp:19-244), OutflowXL..ZR (outflow.cpp:20-312).  Ghosts are filled on
 * active rows/columns only; corners are never touched.  Loop order follows
 * the reference so the in-place semantics match even when n < nGhost. */
static void bc_fill(gko_sim* s, double* u, int d, int side, int type) {
    const int len[3] = {s->lenx, s->leny, s->lenz};
    const int nact[3] = {s->p.nx, s->p.ny, s->p.nz};
    const int b = s->p.ng, e = s->p.ng + nact[d];
    const int gl = side == 0 ? 0 : e, gr = side == 0 ? b : len[d];
    /* transverse active ranges */
    int lo[3] = {s->ib, s->jb, s->kb}, hi[3] = {s->ie, s->je, s->ke};
    lo[d] = gl; hi[d] = gr;
    const int mom = MTX + d;
    const double dmin = s->p.dfloor;
    #define AT(n, c) C(u, (n), (c)[2], (c)[1], (c)[0])
    if (type == 0 || type == 1) {
        /* outflow_copy.cpp:16-182 / periodic.cpp:19-191: ivar, k, j, i loops */
        for (int n = DEN; n <= ENG; n++)
            for (int k = lo[2]; k < hi[2]; k++)
                for (int j = lo[1]; j < hi[1]; j++)
                    for (int i = lo[0]; i < hi[0]; i++) {
                        int c[3] = {i, j, k}, t[3] = {i, j, k};
                        int g = c[d];
                        if (type == 0) t[d] = side == 0 ? b : e - 1;
                        else t[d] = side == 0 ? g + nact[d] : g - nact[d];
                        AT(n, c) = AT(n, t);
                    }
    } else {
        /* reflective.cpp:19-244 / outflow.cpp:20-310: k, j, i loops */
        for (int k = lo[2]; k < hi[2]; k++)
            for (int j = lo[1]; j < hi[1]; j++)
                for (int i = lo[0]; i < hi[0]; i++) {
                    int c[3] = {i, j, k}, t[3] = {i, j, k};
                    int g = c[d];
                    t[d] = side == 0 ? (b + b - g - 1) : (e + e - g - 1);
                    double q[NVAR];
                    for (int n = 0; n < NVAR; ++n) q[n] = AT(n, t);
                    if (type == 2) {
                        q[mom] = -q[mom];
                    } else {
                        double mt = q[mom];
                        double mc = side == 0 ? smin(mt, 0.0) : smax(mt, 0.0);
                        double rho = smax(q[DEN], dmin);
                        double rhoInv = 1.0 / rho;
                        double keOld = 0.5 * rhoInv * mt * mt;
                        double keNew = 0.5 * rhoInv * mc * mc;
                        double eint = q[ENG] - keOld;
                        eint = smax(eint, 1e-16);
                        q[DEN] = rho;
                        q[mom] = mc;
                        q[ENG] = eint + keNew;
                    }
                    for (int n = 0; n < NVAR; ++n) AT(n, c) = q[n];
                }
    }
    #undef AT
}

/* Boundary::Boundary type selection (boundary.cpp:13-125) and
 * Boundary::UpdateBD ordering (boundary.cpp:127-142).  Types other than 0-4
 * fall back to copy; z-side copy maps to the *y* copy routine
 * (boundary.cpp:92,104,109,121). */
static void update_bd(gko_sim* s, double* u) {
    for (int d = 0; d < 3; ++d) {
        if (d == 2 && s->p.nz <= 1) break;
        for (int side = 0; side < 2; ++side) {
            int type = s->p.bc[2 * d + side];
            if (type == 5) continue; /* a side between slabs: gko_advance_split's halo */
            if (type < 0 || type > 3) type = 0;
            if (d == 2 && type == 0) bc_fill(s, u, 1, side, 0);
            else bc_fill(s, u, d, side, type);
        }
    }
}

/* Boundary::UpdateBD on Sim::cons (boundary.cpp:127-142), for tests. */
void gko_update_bd(gko_sim* s) { update_bd(s, s->cons); }

/* ------------------------------------------------------------- source --- */

/* SourceTerm::ConstGravity (const_gravity.cpp:10-69): E first, then m. */
static void const_gravity(gko_sim* s, double* u, double dt) {
    for (int d = 0; d < 3; ++d) {
        double g = s->p.grav[d];
        if (g == 0) continue;
        int mom = MTX + d;
        #pragma omp parallel for collapse(2) schedule(static)
        for (int k = s->kb; k < s->ke; k++)
            for (int j = s->jb; j < s->je; j++)
                for (int i = s->ib; i < s->ie; i++) {
                    C(u, ENG, k, j, i) += C(u, mom, k, j, i) * g * dt;
                    C(u, mom, k, j, i) += C(u, DEN, k, j, i) * g * dt;
                }
    }
}

/* ---------------------------------------------------------- integrate --- */

/* cons.Swap(consTemp), the integrators' last line (forward_euler.cpp:16,
 * rk2.cpp:21, rk3.cpp:27). */
static void swap_state(gko_sim* s) {
    double* t = s->cons; s->cons = s->consTemp; s->consTemp = t;
}

/* The ghost fill of a stage: UpdateBD (rk2.cpp:12, 17; rk3.cpp:12, 17, 22),
 * then (a slab of a split grid) the rows between slabs from the neighbours. */
static void fill_ghosts(gko_sim* s, double* u) {
    update_bd(s, u);
    if (s->halo) s->halo(s->halo_user, u);
}

/* Sim::ForwardEuler_ / RK2_ / RK3_ (forward_euler.cpp:11-18, rk2.cpp:11-23,
 * rk3.cpp:11-29). */
static void integrate(gko_sim* s) {
    fill_ghosts(s, s->cons);
    cons_to_prim(s, s->cons);
    cal_flux(s);
    update_cons(s, s->cons, s->consTemp, 0, 1.0, 1.0, 0.0);
    if (s->p.integrator == 1) { swap_state(s); return; }
    fill_ghosts(s, s->consTemp);
    cons_to_prim(s, s->consTemp);
    cal_flux(s);
    if (s->p.integrator != 3) {
        update_cons(s, s->cons, s->consTemp, 1, 0.5, 0.5, 0.5);
        swap_state(s);
        return;
    }
    update_cons(s, s->cons, s->consTemp, 1, 0.75, 0.25, 0.25);
    fill_ghosts(s, s->consTemp);
    cons_to_prim(s, s->consTemp);
    cal_flux(s);
    double frac13 = 1.0 / 3.0;
    update_cons(s, s->cons, s->consTemp, 1, frac13, 2 * frac13, 2 * frac13);
    swap_state(s);
}

/* Sim::Advance (sim.cpp:69-117). */
int gko_advance(gko_sim* s, double dtoutput, double* dtlog, int cap) {
    int nsteps = 0;
    double tNext = s->t + dtoutput;
    s->dtUntilOutput = dtoutput;
    while (fabs(tNext - s->t) > 1e-12 && s->isContinue) {
        s->cmax = gko_cmax(s);
        s->dt = s->p.cfl * s->drmin / s->cmax;
        s->dt = smin(s->dt, s->dtUntilOutput);
        if (s->has_src) const_gravity(s, s->cons, 0.5 * s->dt);
        integrate(s);
        if (s->has_src) const_gravity(s, s->cons, 0.5 * s->dt);
        s->t += s->dt;
        s->step++;
        s->dtUntilOutput = tNext - s->t;
        if (s->p.stepmax > 0 && s->step >= s->p.stepmax) s->isContinue = 0;
        if (dtlog && nsteps < cap) dtlog[nsteps] = s->dt;
        nsteps++;
    }
    return nsteps;
}

/* ------------------------------------------------------- y-slab split --- */

/* A slab's spacings set to the whole grid's, as Sim forms them (sim.cpp:26-35:
 * dxRec, dyRec = 0 for one row, drmin); the slab's own extent would round
 * differently. */
void gko_set_spacing(gko_sim* s, double dx, double dy, double dz) {
    s->dx = dx;
    s->dy = dy;
    s->dz = dz;
    s->dxRec = 1. / dx;
    s->dyRec = s->p.ny <= 1 ? 0 : 1. / dy;
    s->dzRec = s->p.nz <= 1 ? 0 : 1. / dz;
    s->drmin = smin(smin(dx, dy), dz);
}

/* Sim::Advance (sim.cpp:69-117) on a y-slab of a split grid, at most nsteps
 * steps: the loop of gko_advance with the CFL maximum taken over all slabs
 * (reduce) and the slab's type-5 y sides filled by halo after each stage's
 * UpdateBD.  No counterpart in the reference, which runs one grid whole. */
int gko_advance_split(gko_sim* s, double dtoutput, int nsteps, gko_halo_fn halo,
                      gko_max_fn reduce, void* user, double* dtlog, int cap) {
    int n = 0;
    double tNext = s->t + dtoutput;
    s->dtUntilOutput = dtoutput;
    s->halo = halo;
    s->halo_user = user;
    while (fabs(tNext - s->t) > 1e-12 && s->isContinue && n < nsteps) {
        const double local = gko_cmax(s);
        s->cmax = reduce ? reduce(user, local) : local;
        s->dt = s->p.cfl * s->drmin / s->cmax;
        s->dt = smin(s->dt, s->dtUntilOutput);
        if (s->has_src) const_gravity(s, s->cons, 0.5 * s->dt);
        integrate(s);
        if (s->has_src) const_gravity(s, s->cons, 0.5 * s->dt);
        s->t += s->dt;
        s->step++;
        s->dtUntilOutput = tNext - s->t;
        if (s->p.stepmax > 0 && s->step >= s->p.stepmax) s->isContinue = 0;
        if (dtlog && n < cap) dtlog[n] = s->dt;
        n++;
    }
    s->halo = NULL;
    s->halo_user = NULL;
    return n;
}
