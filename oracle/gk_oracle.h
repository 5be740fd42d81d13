/*
 * gk_oracle.h -- CPU oracle for the Gaukuk finite-volume update.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (ShunqH/Gaukuk, src/) used as the checker for the CUDA path.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it; the product path never does.
 *
 * Parity pin: the restatement is checked bit-for-bit against the reference
 * itself, built from its own sources by oracle/Makefile into oracle/_ref/
 * with strict IEEE flags, and against golden vectors in tests/golden/ that
 * were produced by that build (tests/golden/make_golden.py).
 *
 * Memory layout is the reference's TArray layout (template_array.hpp:67-72):
 * cons[n][k][j][i], n in [0,5) = DEN,MTX,MTY,MTZ,ENG, i fastest, with
 * lenx = nx + 2*ng (grid.hpp:26-28).  In 2D the reference still allocates
 * lenz = 1 + 2*ng planes (sim.cpp:49-54); the same is done here.
 */
#ifndef GK_ORACLE_H
#define GK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gko_params {
    int nx, ny, nz, ng;                 /* NX, NY, NZ, NGhost */
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double gamma, cfl;                  /* gamma, CFL */
    int integrator;                     /* 1 Euler, 2 RK2, 3 RK3 (sim.cpp:56-66) */
    int rc_order;                       /* 1 first order, anything else PLM (cal_flux.cpp:24) */
    int bc[6];                          /* xleft xright yleft yright zleft zright */
    double grav[3];                     /* const gravity vector; all 0 = no source */
    double dfloor, pfloor;              /* GAUKUK_DENSITY_FLOOR / GAUKUK_PRESSURE_FLOOR */
    int stepmax;                        /* <=0 unlimited (sim.cpp:58,95-97) */
} gko_params;

typedef struct gko_sim gko_sim;

/* The y-slab split (gko_advance_split): fills the y ghost rows of state u
 * that come from the neighbouring slabs; the maximum over all slabs. */
typedef void (*gko_halo_fn)(void* user, double* u);
typedef double (*gko_max_fn)(void* user, double local);

/* Sim::Sim (sim.cpp:45-67).  Returns NULL on invalid parameters. */
gko_sim* gko_create(const gko_params* p);
void gko_destroy(gko_sim* s);

/* Number of doubles in one reference-layout state array: 5*lenz*leny*lenx. */
long long gko_state_size(const gko_sim* s);

/* Copy a reference-layout state in / out. */
void gko_set_cons(gko_sim* s, const double* cons);
void gko_get_cons(const gko_sim* s, double* cons);

/* Boundary::UpdateBD (boundary.cpp:127-142) on the current state. */
void gko_update_bd(gko_sim* s);

/* EquationOfState::CalCmax over active cells, starting from 1e-16
 * (sim.cpp:77-78, adiabatic.cpp:115-160). */
double gko_cmax(const gko_sim* s);

/* Sim::Advance (sim.cpp:69-117).  Appends each step's dt to dtlog (if not
 * NULL, up to cap entries) and returns the number of steps taken. */
int gko_advance(gko_sim* s, double dtoutput, double* dtlog, int cap);

/* A y-slab of a grid split across ranks (the multi-GPU decomposition of
 * gk_slabs_*, restated): the whole grid's spacings, then Sim::Advance with
 * the CFL maximum over all slabs (reduce) and the y sides of type 5 (between
 * slabs) filled by halo after every stage's UpdateBD, at most nsteps
 * steps.  The slabs' states are the undivided grid's bits. */
void gko_set_spacing(gko_sim* s, double dx, double dy, double dz);
int gko_advance_split(gko_sim* s, double dtoutput, int nsteps, gko_halo_fn halo,
                      gko_max_fn reduce, void* user, double* dtlog, int cap);

double gko_time(const gko_sim* s);
double gko_dt(const gko_sim* s);
int gko_step(const gko_sim* s);
int gko_is_continue(const gko_sim* s);
void gko_set_time(gko_sim* s, double t, int step);

/* Unit-level restatements, batched over n interfaces / cells. */
/* Flux::RiemannSolver (hllc.cpp:22-101).  wl, wr: 5*n primitives laid out
 * [var][n] (DEN,VLX,VLY,VLZ,PRE); dir: 1=x, 2=y, 3=z (the VLX/VLY/VLZ ids);
 * flux: 5*n conserved fluxes [var][n] in DEN,MTX,MTY,MTZ,ENG slots. */
void gko_hllc_batch(int n, const double* wl, const double* wr, int dir,
                    double gamma, double* flux);
/* Reconstruction::VanLeer (reconstruction.hpp:36-42). */
void gko_vanleer_batch(int n, const double* a, const double* b, double* out);
/* EquationOfState::ConsToPrim pointwise (adiabatic.cpp:41-57). */
void gko_cons_to_prim_batch(int n, const double* cons, double gamma,
                            double dfloor, double pfloor, double* prim);

#ifdef __cplusplus
}
#endif
#endif
