/*
 * gaukuk_cuda.h -- C ABI of the B200 finite-volume update (libgk_cuda.so).
 *
 * The reference (ShunqH/Gaukuk) is a C++ source-level API: a problem hook
 * fills Sim::cons on the host and Sim::Advance runs the time loop.  This
 * library takes over that loop.  The C++ host layer (gaukuk_b200/src) keeps
 * the reference's classes and calls these entry points; Python reaches them
 * through ctypes (gaukuk_b200/_lib.py).  Plain pointers and sizes only.
 *
 * Host arrays use the reference's TArray layout (template_array.hpp:67-72):
 * cons[n][k][j][i], n = DEN,MTX,MTY,MTZ,ENG, lenx = nx + 2*nghost
 * (grid.hpp:26-28), and lenz = nz + 2*nghost planes even in 2D (sim.cpp:49).
 *
 * Every function returns GK_OK (0) or a negative GK_ERR_* code; the text of
 * the last failure on a handle is available from gk_last_error().
 * One host thread per handle; work is ordered on the handle's CUDA stream and
 * every entry point returns after that stream has synchronised, except where
 * stated.
 */
#ifndef GAUKUK_CUDA_H
#define GAUKUK_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define GK_ABI_VERSION 1

enum gk_status {
    GK_OK = 0,
    GK_ERR_INVALID = -1,     /* bad argument or configuration */
    GK_ERR_CUDA = -2,        /* a CUDA runtime call failed */
    GK_ERR_NONFINITE = -3,   /* the CFL reduction met a non-finite state */
    GK_ERR_UNSUPPORTED = -4, /* valid for the reference, not implemented here */
    GK_ERR_STATE = -5        /* call order (e.g. advance before upload) */
};

/* Arithmetic modes.  PARITY evaluates every expression in the reference's
 * order with no FMA contraction: results are bit-identical to the reference
 * compiled with strict IEEE flags (-ffp-contract=off, no -ffast-math),
 * including the dt sequence.  FAST lets the compiler contract to FMA and
 * evaluates only the selected HLLC side; it stays within 1e-12 relative of
 * the reference over 100 steps. */
enum gk_mode { GK_MODE_PARITY = 0, GK_MODE_FAST = 1 };

/* Boundary types, as read from xleft..zright (boundary.cpp:13-125). */
enum gk_bc { GK_BC_COPY = 0, GK_BC_PERIODIC = 1, GK_BC_REFLECTIVE = 2, GK_BC_OUTFLOW = 3,
             GK_BC_FIXED = 4 };

/* Grid + Domain: grid.hpp:18-41 and sim.cpp:16-42 (NX, NY, NZ, NGhost,
 * xmin..zmax from the .in file). */
typedef struct gk_grid_desc {
    int nx, ny, nz, nghost;
    double xmin, xmax, ymin, ymax, zmin, zmax;
} gk_grid_desc;

/* Everything else Sim::Sim reads (sim.cpp:45-67, adiabatic.cpp:12-16,
 * boundary.cpp:13-20), the gravity vector a setup hook enrolls
 * (SourceTerm::EnrollConstGravityVector, source.cpp:23-31) and the floors
 * fixed at build time (gaukuk.hpp:11-21, Makefile:47-48). */
typedef struct gk_phys_desc {
    double gamma;       /* adiabatic index */
    double cfl;         /* CFL */
    int integrator;     /* 1 Euler, 3 RK3, anything else RK2 (sim.cpp:59-66) */
    int rc_order;       /* 1 first order, anything else PLM (cal_flux.cpp:24) */
    int bc[6];          /* xleft xright yleft yright zleft zright */
    double grav[3];     /* constant gravity; all zero = no source term */
    double dfloor;      /* density floor (1e-16 in the reference build) */
    double pfloor;      /* pressure floor (1e-16) */
    int stepmax;        /* <= 0: unlimited (sim.cpp:58, 95-97) */
    int mode;           /* enum gk_mode */
    int device;         /* CUDA device ordinal */
} gk_phys_desc;

typedef struct gk_handle gk_handle;

/* Replaces Sim::Sim (sim.cpp:45-67) with Boundary::Boundary (boundary.cpp:13-125)
 * and EquationOfState::EquationOfState (adiabatic.cpp:12-16): validates the
 * configuration and allocates the device state.  Time starts at t = 0,
 * step = 0 (sim.cpp:45-46). */
int gk_create(const gk_grid_desc* grid, const gk_phys_desc* phys, gk_handle** out);

/* Releases the handle, its stream, graphs and device memory: the end of a
 * Sim's lifetime, where the reference's TArray members free their arrays
 * (~TArray, template_array.hpp:89-91). */
void gk_destroy(gk_handle* h);

/* Fixed (type 4) boundaries: Boundary::EnrollFixedBoundaryData
 * (fixed.cpp:226-268) and FixedBD* (fixed.cpp:16-176).  `snapshot` is the
 * reference-layout state at enrollment; every ghost cell of a type-4 side
 * then gets its value from it at each ghost fill.  fix_inner != 0 also runs
 * Boundary::FixedBDInner (fixed.cpp:180-206) after the sides: in the central
 * index box, cells with x^2 + y^2 + z^2 < 0.25 get back their snapshot
 * values.  NULL removes the data.  A run with a type-4 side refuses to
 * advance until the data are set. */
int gk_set_fixed_boundary(gk_handle* h, const double* snapshot, int fix_inner);

/* A self-defined side whose ghost values depend on the state
 * (Boundary::EnrollSelfDefineBD*, boundary.hpp:28-45; the copy template of
 * setup_example.cpp:120-140): a host routine fills it at every ghost fill.
 * side 0..5 = x left, x right, y left, y right, z left, z right.  cons: the
 * caller's reference-layout array the routine works on (NVar x lenz x leny x
 * lenx, host).  Before each call the library copies into `cons` the side's
 * ghost strip and the `depth` cell layers next to it (depth >= n + nghost:
 * the whole extent), across the whole transverse extent and every variable;
 * fn(user, cons) then fills the strip (ghost layers, active transverse
 * cells), which is copied back.  fn returns 0, or non-zero to stop the run
 * (the advance then returns GK_ERR_INVALID).  The device fills the other
 * sides first.  A handle with host sides runs its steps without a CUDA
 * graph, returning to the host at every ghost fill.  fn = NULL removes the
 * side's routine.  Not for ensembles. */
typedef int (*gk_host_fill_fn)(void* user, double* cons);
int gk_set_host_fill(gk_handle* h, int side, int depth, gk_host_fill_fn fn, void* user,
                     double* cons);

/* Point masses: SourceTerm::EnrollPointGravity (source.cpp:33-68) as the
 * Strang half kicks of PointGravity (point_gravity.cpp:11-92, n = 1) or
 * BinaryGravity (binary_gravity.cpp, n = 2), after the constant gravity.
 * params: gm0, x0, y0, z0, rs0 (n = 1); then gm1, z1, rs1, omega, ab,
 * theta1 (n = 2; the second mass sits at ab (cos, sin)(omega t + theta1), z1),
 * with omega, ab and theta1 as EnrollPointGravity computes them.  n = 0
 * removes them.  Runs with point masses take the generic path. */
int gk_set_point_gravity(gk_handle* h, int n, const double* params);

/* Immersed solid body: the table Boundary::SetupImmersedShell builds
 * (immersed.cpp:89-241), applied as Boundary::ImmersedReflective
 * (immersed.cpp:243-303) at every ghost fill, after the sides and before
 * the inner reset (boundary.cpp:127-142).  The arrays are the reference's
 * own, for n shell cells (nTarMax = 8):
 *   ids  int[3 * n * 9]   shellIDs(3, nShell, 9): ids[(c*n + s)*9 + t] is
 *                         coordinate c (i, j, k; reference indices) of shell
 *                         cell s (t = 0) and of its targets t = 1..ntar[s]
 *   ntar int[n]           nTars
 *   dir  double[4 * n]    shellDirection(4, nShell): cos(phi), sin(phi),
 *                         cos(theta), sin(theta) at dir[c*n + s]
 *   w    double[n * 9]    disGamma(nShell, 9)
 * Every cell named must be active (GK_ERR_INVALID otherwise); n = 0 removes
 * the body.  Needs nx > 1 and ny > 1; runs with a body take the generic
 * path in 2D. */
int gk_set_immersed(gk_handle* h, int n, const int* ids, const int* ntar, const double* dir,
                    const double* w);

/* Number of doubles in one reference-layout state, the size of Sim::cons
 * (cons.NewArray(NVar, lenz, leny, lenx), sim.cpp:49): 5*lenz*leny*lenx. */
long long gk_state_size(const gk_handle* h);

/* Loads Sim::cons from the host after the setup hook ran (main.cpp:25-30):
 * the whole array, ghosts included, is copied to the device (the host array
 * is not retained), the dt log is cleared and the CFL reduction of
 * EquationOfState::CalCmax (adiabatic.cpp:115-160) is evaluated so that the
 * next step's dt is ready.  In 1D/2D a z-momentum plane that is +0.0 in every
 * stored cell (checked on the host while the other planes copy) is cleared
 * on the device instead of copied. */
int gk_upload_cons(gk_handle* h, const double* cons);

/* Copies the device state back into a reference-layout host array, as
 * Sim::WriteData reads it (write_sim.cpp:14-58).  Active cells are exactly
 * the reference's.  In 1D/2D the planes k != nghost are written as zero.
 * Ghost cells hold the boundary fill of the current state. */
int gk_download_cons(gk_handle* h, double* cons);

/* As gk_download_cons, but writes only the planes the device holds (in 1D/2D
 * the active plane k = nghost) and leaves the caller's other planes as they
 * are -- the copy Sim::WriteData needs when Sim::cons is reused between
 * frames, since the reference never writes those planes.  When the fused 2D
 * path runs (gk_path = 1), the z-momentum plane was +0.0 everywhere at upload
 * and no fixed data are set, nothing on the device writes that plane and it
 * is left as it is in `cons` too: a caller that uploaded from the same array
 * has the same bits there. */
int gk_download_planes(gk_handle* h, double* cons);

/* Cells the floors repaired since the last upload (Sim::UpdateCons,
 * update_cons.cpp:55-68): density below the floor (the cell is reset to
 * vacuum) and pressure below it (the energy is reset).  The reference
 * repairs silently; these count every stage's repairs.  Either pointer may
 * be NULL. */
int gk_floor_hits(gk_handle* h, unsigned long long* density, unsigned long long* pressure);

/* Bytes the last gk_upload_cons and the last download moved across the bus
 * (either pointer may be NULL).  No counterpart in the reference, whose state
 * never leaves host memory. */
int gk_io_bytes(const gk_handle* h, long long* upload, long long* download);

/* Replaces Sim::Advance (sim.cpp:69-117, sim.hpp:39): runs time steps on the
 * device until the output time t + dtoutput is reached (tolerance 1e-12),
 * stepmax is hit, or the CFL reduction fails.  Each step: cmax -> dt =
 * min(CFL*drmin/cmax, dtUntilOutput) -> gravity half kick -> integrator ->
 * gravity half kick -> t += dt.  Outputs (any may be NULL): time, step count
 * and the isContinue flag after the call. */
int gk_advance(gk_handle* h, double dtoutput, double* t, int* step, int* is_continue);

/* Runs exactly nsteps steps (fewer if stepmax stops the run, sim.cpp:96-97)
 * with no output time to clamp dt, i.e. Sim::Advance (sim.cpp:69-117) with an
 * infinite dtoutput.  Returns after the stream synchronises; *done receives
 * the steps taken. */
int gk_run_steps(gk_handle* h, int nsteps, int* done);

/* As gk_run_steps, but only enqueues the work on the handle's stream and
 * returns at once: the steps beyond the run's end are no-ops on the device.
 * Used to time a device-resident loop with events on gk_stream(). */
int gk_enqueue_steps(gk_handle* h, int nsteps);

/* Sim::GetTime / Getdt / GetStep and Sim::isContinue (sim.hpp:26, 43-45). */
int gk_get_time(gk_handle* h, double* t, double* dt, int* step, int* is_continue);

/* Sets the simulation clock, for a restart from a written frame (the frame
 * holds t, write_sim.cpp:33).  The reference has no setter: t and step are
 * private members of Sim (sim.hpp:48-49). */
int gk_set_time(gk_handle* h, double t, int step);

/* The dt of every step since the last upload, at full precision: the values
 * Sim::Advance prints with 6 digits (sim.cpp:100-103).  Copies up to cap
 * entries; *n receives the total count. */
int gk_dt_log(gk_handle* h, double* buf, int cap, int* n);

/* EquationOfState::CalCmax seeded with 1e-16 (sim.cpp:77-78) on the current
 * device state. */
int gk_cmax(gk_handle* h, double* cmax);

/* The handle's CUDA stream (a cudaStream_t), for callers that time or order
 * work around the library's launches.  No counterpart in the reference (CPU
 * only). */
int gk_stream(gk_handle* h, void** stream);

/* Which device implementation the handle selected: 0 generic (unfused
 * per-phase kernels, any dimension), 1 fused 2D stage kernel, 2 3D stage
 * (z fluxes and a fused x-y stage per plane), 3 a 1D run in one CTA (up to
 * 1024 cells per row, many steps per launch).  No counterpart in the
 * reference, which has one CPU path for every dimension. */
int gk_path(gk_handle* h, int* path);

/* Launch accounting: whole time steps per graph launch, and kernel launches
 * per time step on the selected path.  No counterpart in the reference. */
int gk_graph_info(gk_handle* h, int* steps_per_graph, int* launches_per_step);

/* Device time of each kernel class over `nsteps` un-graphed steps, measured
 * with CUDA events on the handle's stream: names (';'-separated, into
 * `names`, size `names_cap`), per-class total milliseconds and launch counts
 * (arrays of `cap` entries).  *n receives the number of classes.  The
 * reference times only the whole run (main.cpp:42-43, 54-58). */
int gk_profile_steps(gk_handle* h, int nsteps, char* names, int names_cap,
                     double* total_ms, int* launches, int cap, int* n);

/* Tile shape of the fused 2D stage kernel: threads per CTA (64, 128 or 256;
 * each CTA updates threads-4 columns) and rows per CTA segment.  Takes effect
 * from the next run; the project's autotuner (gaukuk_b200/autotune.py) picks
 * it by measurement. */
int gk_set_tiling(gk_handle* h, int threads, int rows);

/* Ensembles: independent 2D problems (fused path: vz = 0, RK2, same mode
 * and device) advanced together.  Every RK stage of every instance is one
 * persistent launch over a tile table and every ghost fill one launch, held
 * in a CUDA graph of whole steps; each instance keeps its own handle, clock
 * and dt, and its results equal those of running it alone.  The handles
 * stay valid for upload, download and time queries; they must outlive the
 * ensemble.  A handle with a fixed (type 4) side must have its data set
 * (gk_set_fixed_boundary) before it joins: GK_ERR_STATE otherwise.  No
 * counterpart in the reference, which runs one problem per process. */
typedef struct gk_ensemble gk_ensemble;
int gk_ens_create(gk_handle* const* handles, int n, gk_ensemble** out);
void gk_ens_destroy(gk_ensemble* e);
/* threads per CTA (64, 128, 256) for all instances; rows: one entry per
 * instance, or NULL to keep the current ones (default 16). */
int gk_ens_set_tiling(gk_ensemble* e, int threads, const int* rows);
/* Sim::Advance(dtoutput) on every instance, each from its own time. */
int gk_ens_advance(gk_ensemble* e, double dtoutput);
/* nsteps steps of every instance (no output time); the enqueue form returns
 * at once, for timing with events on the ensemble's stream. */
int gk_ens_run_steps(gk_ensemble* e, int nsteps);
int gk_ens_enqueue_steps(gk_ensemble* e, int nsteps);
/* Number of tiles, threads per CTA and the ensemble's CUDA stream. */
int gk_ens_info(gk_ensemble* e, int* ntiles, int* threads, void** stream);
const char* gk_ens_last_error(const gk_ensemble* e);

/* ---- Learned flux correction (no counterpart in the reference) ----
 * A 16 -> 64 -> 64 -> 4 MLP with GELU predicts a correction to each face's
 * HLLC flux on a coarse grid from the 4-cell stencil of primitives across
 * the face; it is trained to the restricted fluxes of a finer run.  Model
 * blob (gk_mlp_nmodel() floats): W1[64][16] b1[64] W2[64][64] b2[64]
 * W3[4][64] b3[4] (gk_mlp_nparams() parameters), then the input means[16],
 * input deviations[16], output means[4], output deviations[4].  Training and
 * inference run in BF16 on the tensor cores with FP32 accumulation
 * (gaukuk_b200/csrc/gk_mlp.cu); the correction is added to the FP64 flux. */
typedef struct gk_mlp gk_mlp;
int gk_mlp_nparams(void);
int gk_mlp_nmodel(void);
int gk_mlp_create(const float* model_host, gk_mlp** out);
void gk_mlp_destroy(gk_mlp* m);
int gk_mlp_get(gk_mlp* m, float* model_host);
/* Loss of the training calls.  w < 0 (the default): the squared error of
 * each sample summed over the outputs.  0 <= w <= 1: the samples come in
 * pairs (2m, 2m + 1) of neighbouring faces and each pair's loss per output
 * is (1 - w)(e0^2 + e1^2) + w (e1 - e0)^2, the last term being the error of
 * the update of the cell between the two faces; n must then be even. */
int gk_mlp_set_pair_loss(gk_mlp* m, float w);
/* Summed gradient of the first `batch` samples (no update).  X: n x 16 BF16
 * and T: n x 4 FP32 (standardised), on the device. */
int gk_mlp_grad(gk_mlp* m, const void* X, const float* T, long long n, int batch,
                float* grad_host, float* loss_host);
/* `steps` Adam steps (b1 0.9, b2 0.999, eps 1e-8) on batches drawn with
 * replacement; *loss_host: mean squared error of the last batch. */
int gk_mlp_train(gk_mlp* m, const void* X, const float* T, long long n, int batch, int steps,
                 float lr, unsigned long long seed, float* loss_host);
/* Standardised outputs of n samples (device X, device Y n x 4). */
int gk_mlp_forward(gk_mlp* m, const void* X, long long n, float* Y);

/* Installs (model_host != NULL) or removes the correction on a 2D handle:
 * every stage then adds the network's correction to each face flux, except
 * where the detector fires -- a pressure ratio above 1 + shock_jump over the
 * stencil, or a correction moving more than pos_frac of an adjacent cell's
 * mass or internal energy in one step -- which keeps plain HLLC there, and
 * except in smooth flow: faces whose stencil total variation (the sum of
 * |differences| of neighbouring cells' normalised features) is below tv_min
 * keep plain HLLC too, without counting as a detector firing.  Each
 * component of a correction is clipped to diss_frac times the face's HLL
 * dissipation (1/2) max(|vn| + c) |U_R - U_L| of its PLM face states, so the
 * corrected flux keeps part of the scheme's dissipation; diss_frac < 0
 * disables the clip. */
int gk_set_flux_model(gk_handle* h, const float* model_host, int nmodel, float shock_jump,
                      float pos_frac, float tv_min, float diss_frac);
/* Where the correction runs (pattern 4's inference; no counterpart in the
 * reference).  fused = 1 (the default): inside the fused 2D stage, at the
 * face where its HLLC flux is formed (hllc.cpp:90-95 within
 * cal_flux.cpp:89-121), for runs the fused stage takes (2D RK2/RK3, vz = 0,
 * TMA rows); fused = 0: on the generic path, as a pass over the face fluxes
 * of each direction.  In parity mode the two give the same bits; the
 * detector counts the same faces. */
int gk_set_flux_model_fused(gk_handle* h, int fused);
/* Faces where the detector has fired since the model was installed. */
int gk_flux_model_fired(gk_handle* h, unsigned* fired);

/* Training data: the HLLC face fluxes of the current state (2D; DEN, MTX,
 * MTY, ENG planes; x faces [4][ny][nx+1], y faces [4][ny+1][nx], host).  An
 * installed flux model corrects them (its shock detector, smoothness gate
 * and dissipation clip apply; the positivity detector, which needs a step
 * size, does not). */
int gk_face_fluxes(gk_handle* h, double* fx, double* fy);
/* Advances a 2D RK2 run by nsub steps of fixed dt_sub and returns the
 * fluxes through the faces of the grid coarsened by `ratio`, averaged over
 * the fine faces of each coarse face, the two RK stages and the steps:
 * fx_acc, fy_acc [4][ny/ratio][nx/ratio] (left / lower face of each coarse
 * cell), host.  An installed flux model corrects the tapped fluxes. */
int gk_tap_substeps(gk_handle* h, int nsub, double dt_sub, int ratio, double* fx_acc,
                    double* fy_acc);

/* Diagnostic of the FAST mode arithmetic: the largest error, in ulp of the
 * IEEE result, of its refined reciprocal, square root and reciprocal square
 * root against CUDA's IEEE division and sqrt, over n arguments spread over
 * [2^-60, 2^60] (worst3 = {reciprocal, sqrt, rsqrt}).  Runs on the current
 * device.  No counterpart in the reference, whose arithmetic is the host
 * compiler's. */
int gk_fastmath_check(int n, unsigned long long seed, double* worst3);


/* The bounds-checked build (lib/checked/libgk_cuda.so, compiled with
 * GK_CHECKED; no counterpart in the reference, whose only sanitizer is a
 * commented-out AddressSanitizer line, Makefile:43-44): the number of cell,
 * face, stage-row and TMA-row coordinates found outside their arrays since
 * the library loaded (each was clamped into its array or not issued, so no
 * access left a buffer), and the first one: site << 48 | coordinate << 24 |
 * bound (sites: 1-3 state k, j, i; 4-6 face k, j, i; 7 stage store row;
 * 8 TMA row).  GK_ERR_UNSUPPORTED in the normal build. */
int gk_checked_report(unsigned long long* count, unsigned long long* first);

/* One RK2 time step of a 2D problem (vz = 0, gz = 0) on a caller-owned
 * device state, for callers that cannot allocate device memory while they
 * run: their memory comes from their own pool or arena, or their budget is
 * fixed at start-up.  No counterpart in the reference; the arithmetic is
 * that of gk_run_steps with one step (constant gravity included: both half
 * kicks).  Nothing is allocated: the intermediate stage state (all five
 * planes, since the ghost fill writes every plane's ghosts) and the device
 * clock live in one fixed 64 MiB array inside the library, held by every GPU
 * that loads it until the process exits, so grids whose stage state exceeds
 * it (5 * leny * pitch > 2^23 doubles: more than about 1290 x 1290 cells)
 * are rejected with GK_ERR_INVALID.  Fixed (type 4) sides need the state at
 * enrollment that only a handle holds: GK_ERR_UNSUPPORTED.
 *
 * state: the device layout of the library -- five planes DEN, MTX, MTY, ENG,
 * MTZ, each leny rows of `pitch` doubles (lenx rounded up to a multiple of
 * 16), ghost columns and rows included; MTZ must be zero.  It is updated in
 * place; its ghost cells are overwritten by the boundary fill.  A state
 * aligned to 16 bytes (any cudaMalloc'd or pool block) is staged into the
 * stage kernel by TMA; the tensor map cannot describe a less aligned one, and
 * the call then runs the register-staged form of the stage (same results)
 * after a line on stderr.
 * dt = min(CFL*drmin/cmax(state), dtmax) as in Sim::Advance (sim.cpp:77-81);
 * *dt_used (host, may be NULL) receives it.  stream: a cudaStream_t or NULL;
 * the call returns after that stream synchronises.
 *
 * The first call on a device looks up the array's device address; make it
 * before any stream capture.  The array is shared by every call and keeps the
 * last call's contents (the clock is reset on entry): calls whose work
 * overlaps on one GPU race on it. */
int gk_rk2_step_noalloc(const gk_grid_desc* grid, const gk_phys_desc* phys, double* state,
                        double dtmax, double* dt_used, void* stream);

/* ---- One 2D grid split into y-slabs (scale-out of Sim::Advance) ----
 * No counterpart in the reference, which runs one grid in one process
 * (sim.cpp:69-117); the arithmetic is Sim::Advance's over the whole grid.
 * The ny active rows are split into nslab slabs of ny/nslab rows (the first
 * ny % nslab take one more).  Per RK stage every slab's two ghost rows on
 * each side come from its neighbours' active rows (a ring under periodic y);
 * per step the CFL maximum is taken over all slabs, so every slab takes the
 * whole grid's dt.  Results (state and dt sequence) equal the undivided
 * grid's bit for bit.  Needs the fused 2D path: 2D, RK2 or RK3, vz = 0,
 * gz = 0, no point masses, immersed body, fixed sides or flux model; a
 * periodic y side needs a periodic partner; every slab needs >= 2 rows. */
typedef struct gk_slabs gk_slabs;

/* Rows and neighbours of slab k of nslab over ny active rows: first active
 * row j0 (0-based), row count, lower and upper neighbour slab (-1: a side of
 * the grid, filled by the ghost fill).  Host only. */
int gk_slab_layout(int ny, int nslab, int k, int periodic, int* j0, int* rows, int* lower,
                   int* upper);
/* The NCCL calls of one halo exchange of slab k, in the order the library
 * makes them: nops pairs {kind, peer} in ops8, kind 0 send the top rows,
 * 1 receive the lower ghost rows, 2 send the bottom rows, 3 receive the
 * upper ghost rows (rows going up first, then down: between two ranks the
 * k-th send matches the k-th receive).  Host only. */
int gk_slab_exchange_plan(int nslab, int k, int periodic, int* ops8, int* nops);
/* nslab slabs in this process, on phys->device, exchanging through device
 * copies on one stream (a grid emulated as slabs on one GPU, or slabs that
 * share a GPU). */
int gk_slabs_create(const gk_grid_desc* grid, const gk_phys_desc* phys, int nslab, gk_slabs** out);
/* One slab per process (rank of nranks, slab index = rank) on phys->device,
 * exchanging through NCCL (libnccl.so.2, loaded at the first call): the
 * rows are sent and received once per stage, the CFL speed is all-reduced
 * (max) once per step.  id128: a 128-byte NCCL unique id made by one process
 * with gk_slabs_nccl_id and passed to all.  Every process must make the same
 * calls in the same order (they take part in the same collectives).  The
 * library's NCCL calls have no timeout: a process that fails or leaves
 * between steps leaves the others waiting in their next exchange, and the
 * job's launcher must end them, as for any NCCL job.  A failure that every
 * process sees (a non-finite state, a timed-out row load) stops all of them
 * together: the status word is part of the per-step all-reduce. */
int gk_slabs_nccl_id(void* id128);
int gk_slabs_create_nccl(const gk_grid_desc* grid, const gk_phys_desc* phys, int nranks, int rank,
                         const void* id128, gk_slabs** out);
void gk_slabs_destroy(gk_slabs* s);
/* The whole grid's state in the reference layout (NVar x lenz x (ny+4) x
 * lenx): each slab of this process takes its rows.  Download writes this
 * process's active rows (and the grid's own ghost rows where its slabs end
 * the grid) and leaves the other rows of `cons` as they are. */
int gk_slabs_upload_cons(gk_slabs* s, const double* cons);
int gk_slabs_download_cons(gk_slabs* s, double* cons);
/* Sim::Advance(dtoutput) of the whole grid, and a fixed step count. */
int gk_slabs_advance(gk_slabs* s, double dtoutput, double* t, int* step, int* is_continue);
int gk_slabs_run_steps(gk_slabs* s, int nsteps, int* done);
/* The whole grid's dt sequence (every slab takes the same steps). */
int gk_slabs_dt_log(gk_slabs* s, double* buf, int cap, int* n);
/* This process's slabs: count, index of the first, its first row and rows. */
int gk_slabs_info(gk_slabs* s, int* nslab_local, int* first, int* j0, int* rows);
const char* gk_slabs_last_error(const gk_slabs* s);

/* Text for a status code, and the last failure message on a handle.  The
 * reference throws instead (grid.hpp:24, read_config.cpp:22,
 * write_sim.cpp:25) and main does not catch. */
const char* gk_strerror(int status);
const char* gk_last_error(const gk_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* GAUKUK_CUDA_H */
