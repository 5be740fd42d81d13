// gk_internal.h -- types shared by the C-ABI layer and the kernel units.
//
// Device state layout (one allocation per state buffer): five variable
// planes in slot order DEN, MTX, MTY, ENG, MTZ, so that the four variables a
// 2D run evolves are contiguous and MTZ is last.  Each plane holds `nzs`
// z-planes (1 in 1D/2D, lenz in 3D) of `leny` rows with a row pitch of
// `pitch` doubles (lenx rounded up to 16 doubles = 128 bytes).  Column i and
// row j are the reference's own indices (ghosts at 0..nghost-1), so ghost
// fills and face indices read exactly like the reference loops.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>

namespace gk {

// True the first time it is called for the current device with this mask:
// kernel attributes (dynamic shared memory above 48 KB) are per device, so a
// process that drives several GPUs sets them on each.
inline bool first_on_device(std::atomic<unsigned long long>& mask) {
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    return (mask.fetch_or(bit) & bit) == 0;
}

// Device variable slots.
enum Slot { S_DEN = 0, S_MTX = 1, S_MTY = 2, S_ENG = 3, S_MTZ = 4 };
// Primitive slots use the same positions: rho, vx, vy, p, vz.
enum PSlot { P_RHO = 0, P_VX = 1, P_VY = 2, P_PRE = 3, P_VZ = 4 };

struct Geom {
    int nx, ny, nz, ng;
    int lenx, leny, lenz;
    int ib, ie, jb, je, kb, ke;
    int ndim;            // 1, 2 or 3
    int pitch;           // doubles per row
    int nzs;             // stored z-planes
    int kofs;            // reference k of stored plane 0
    long long kstride;   // doubles per stored z-plane (pitch*leny)
    long long vstride;   // doubles per variable slot (kstride*nzs)
    // face arrays (generic path): rows leny+1, planes nzs+1
    int fpitch;
    long long fkstride, fvstride;
    double dx, dy, dz, dxRec, dyRec, dzRec, drmin;
    double xmin, ymin, zmin;  // cell centres: xmin - ng*dx + 0.5*dx + i*dx (sim.cpp:36-41)
};

// One shell cell of an immersed body (Boundary::SetupImmersedShell,
// immersed.cpp:89-241), indices in device layout: the cell, its image-point
// targets tgt[0..ntar), the direction cosines cos(phi), sin(phi),
// cos(theta), sin(theta) and the weights disGamma(s, 0..8).
struct Shell {
    long long cell;
    long long tgt[8];
    double dir[4];
    double w[9];
    int ntar;
};

struct Phys {
    double gamma, gm1, gm1Rec, gmRec, cq;  // cq = 0.5*(1+1/gamma) (hllc.cpp:55-58)
    double gm1Rec1;                        // gm1Rec + 1: fast mode's E + p = p*gm1Rec1 + rho k/2
    double gcq;                            // gamma*cq: fast mode's gamma X = gamma p + gcq max(p* - p, 0)
    double hgm1;                           // (gamma-1)/2: fast mode's conversion
    double cfl, dmin, pmin;
    double grav[3];
    int has_grav;
    int integrator;   // 1, 2, 3
    int plm;          // 1 = PLM, 0 = first order
    int bc[6];        // effective ghost-fill type per side (after the z->y copy mapping)
    int fill_z;       // 3D only: whether z sides are filled (per side bit 0/1)
    int stepmax;
    // Fixed (type 4) sides and the inner reset (fixed.cpp): the state at
    // enrollment in device layout (null when none), and the index box
    // [inner[0], inner[1]) x [inner[2], inner[3]) of FixedBDInner.
    const double* fixed_bd;
    int fix_inner;
    int inner[4];
    // Point masses (point_gravity.cpp, binary_gravity.cpp): npoint 0, 1 or
    // 2; pm = gm0, x0, y0, z0, rs0, gm1, z1, rs1, omega, ab, theta1.
    int npoint;
    double pm[11];
    // Immersed body (immersed.cpp): nshell shell cells (0 = none).
    const Shell* shells;
    int nshell;
    // A slab of a grid split in y: the last stage leaves the step epilogue
    // to launch_epilogue, which runs after the CFL maximum over all slabs.
    int defer_epilogue;
    // The fused 2D stage writes the periodic ghost images of the cells it
    // updates (a grid periodic on all four sides, no source term): the
    // steps skip the ghost fill.
    int periodic_images;
};

// Device-resident clock of Sim::Advance (sim.cpp:69-117).  Written by the
// step epilogue (the last CTA of the CFL kernel) and by the begin kernel.
struct DevTime {
    double t, dt, tNext, dtUntilOutput;
    double cmax_last;                 // CalCmax of the current state
    unsigned long long cmax_acc;      // running max (bit pattern; values >= 0)
    unsigned int done_ctas;           // last-CTA detection counter
    int step;
    int is_continue;                  // Sim::isContinue
    int active;                       // the loop condition of the running call
    int status;                       // error bits (STATUS_*)
    int steps_left;                   // step budget (-1 = none)
    int nlog, log_cap;
    double* log;                      // dt of each step
    // cells the floors repaired since the last upload (update_cons.cpp:55-68):
    // density below the floor (vacuum reset), pressure below it (energy reset)
    unsigned long long floor_den, floor_pre;
};

enum { STATUS_NONFINITE = 1, STATUS_TMA_TIMEOUT = 2, STATUS_NO_MAP = 4 };

struct Ctx {
    Geom g;
    Phys ph;
    DevTime* tm;
    int has_vz;      // 2D: MTZ not identically zero -> generic path
    int h2d_rows;       // fused 2D kernel: rows per CTA segment
    int use_tma;        // fused 2D kernel: rows staged in shared memory by TMA
    int stage_threads;  // fused 2D kernel (TMA): threads per CTA, 64 / 128 / 256
    int learn_rows;     // the fused stage with the learned correction: rows per
                        // segment (0: h2d_rows)
};

// One instance of an ensemble, as the persistent stage kernel reads it from
// global memory: tensor maps of its two state buffers, the buffers, its
// clock, its tiling and geometry.
struct alignas(64) EnsInst {
    CUtensorMap mapA;
    CUtensorMap mapB;
    double* A;
    double* B;
    DevTime* tm;
    int rows, tiles_x, tiles;
    Geom g;
    Phys ph;
};

// Tensor map of the four evolved planes of a state buffer: dims (pitch, leny,
// 4) doubles, box (nt, 1, 4), no swizzle, zero fill out of bounds (gk_api.cu).
bool encode_rows_map(CUtensorMap* map, const double* base, const Geom& g, int nt);

// Where and how far the learned flux correction applies.  A face keeps its
// plain HLLC flux when max(p)/min(p) over its stencil exceeds 1 + shock_jump,
// or when the correction would move more than pos_frac of an adjacent cell's
// mass or internal energy through it in one step (both counted as detector
// firings), or when the total variation of its stencil's features is below
// tv_min (smooth flow, where the plain method is accurate; not counted).
// Each component of a correction is clipped to diss_frac times the face's
// HLL dissipation (1/2) max(|vn| + c) |U_R - U_L| of the PLM face states, so
// the corrected flux keeps part of the scheme's own dissipation
// (diss_frac < 0: no clip).
struct FluxGate {
    float shock_jump = 0.5f;
    float pos_frac = 0.02f;
    float tv_min = 0.0f;
    float diss_frac = -1.0f;
};

// The learned flux correction of one direction of a generic-path stage
// (gk_mlp.cu).
void launch_flux_correct(const float* model, const double* W, double* F, const Geom& g,
                         const Phys& ph, const DevTime* tm, int dir, const FluxGate& gate,
                         unsigned* fired, cudaStream_t s);

// One slab of a grid split into y-slabs, as the halo and reduction kernels
// of gk_slab.cu read it: its three state buffers (A, B, C; C null without
// RK3), its clock, its row range and its neighbours (slab indices, -1 where
// the side is a physical boundary filled by the ghost fill).
struct SlabDev {
    double* buf[3];
    DevTime* tm;
    long long vstride;
    int jb, je;          // active rows [jb, je) in the slab's own indices
    int lower, upper;
};

// Halo exchange between the slabs of one process (same device): the two
// ghost rows below and above every slab, all five planes, active columns,
// copied from its neighbours' active rows in buffer `role` (0 A, 1 B, 2 C).
void launch_slab_halo(const SlabDev* sd, int n, int role, const Geom& g, cudaStream_t s);
// The CFL maximum over slabs: which = 0 the running maximum of a step
// (cmax_acc, before the deferred epilogue), 1 the maximum of the uploaded
// states (cmax_last, before a run begins); status words are combined.
void launch_slab_reduce(const SlabDev* sd, int n, int which, cudaStream_t s);
// Across processes: the rows a slab sends down (its first two active rows)
// and up (its last two) packed into two buffers of 5 x 2 x nx doubles, the
// rows it receives unpacked into its ghost rows (null: a physical side).
void launch_slab_pack(const double* u, double* send_lo, double* send_hi, const Geom& g,
                      const DevTime* tm, cudaStream_t s);
void launch_slab_unpack(double* u, const double* recv_lo, const double* recv_hi, const Geom& g,
                        const DevTime* tm, cudaStream_t s);
// {CFL maximum bits, status} of one slab to and from the all-reduce buffer.
void launch_slab_red_pack(const DevTime* tm, unsigned long long* red, int which, cudaStream_t s);
void launch_slab_red_unpack(DevTime* tm, const unsigned long long* red, int which,
                            cudaStream_t s);

// Kernel classes, for per-kernel profiling.
enum KClass { K_BC = 0, K_C2P, K_FLUX, K_UPDATE, K_KICK, K_CFL, K_STAGE, K_BEGIN, K_NCLASS };
static const char* const kClassNames[K_NCLASS] = {
    "ghost_fill", "cons_to_prim", "flux", "update", "gravity_kick", "cfl_reduce",
    "stage2d", "begin"};

}  // namespace gk

// One set of launchers per arithmetic mode (gk_kernels_parity.cu,
// gk_kernels_fast.cu).  Same signatures, different namespaces.
#define GK_DECLARE_KERNEL_SET(NS)                                                              \
    namespace NS {                                                                             \
    void launch_bc(const gk::Ctx& c, double* u, cudaStream_t s);                               \
    void launch_c2p(const gk::Ctx& c, const double* u, double* prim, cudaStream_t s);          \
    void launch_flux(const gk::Ctx& c, int dir, const double* prim, double* F, cudaStream_t s); \
    void launch_update(const gk::Ctx& c, const double* u0, const double* uc, double* out,      \
                       const double* F1, const double* F2, const double* F3, int three,        \
                       double c1, double c2, double c3, cudaStream_t s);                       \
    void launch_kick(const gk::Ctx& c, double* u, int which, cudaStream_t s);                  \
    void launch_zflux(const gk::Ctx& c, const double* u, double* F3, cudaStream_t s);          \
    void launch_stage3d(const gk::Ctx& c, const double* uc, const double* u0, double* out,     \
                        const double* F3, int three, double c1, double c2, double c3,          \
                        cudaStream_t s);                                                       \
    void launch_cfl(const gk::Ctx& c, const double* u, int epilogue, cudaStream_t s);          \
    void launch_run1d(const gk::Ctx& c, double* A, double* B, int nsteps, cudaStream_t s);     \
    void launch_stage2d(const gk::Ctx& c, const double* uc, const double* u0, double* out,     \
                        int kind, double c1, double c2, double c3, cudaStream_t s);            \
    void launch_stage2d_learn(const gk::Ctx& c, const double* uc, const double* u0,           \
                              double* out, int kind, double c1, double c2, double c3,          \
                              const float* model, const gk::FluxGate& gate, unsigned* fired,   \
                              cudaStream_t s);                                                 \
    void launch_begin(const gk::Ctx& c, double dtoutput, int steps, cudaStream_t s);           \
    void launch_epilogue(const gk::Ctx& c, cudaStream_t s);                                    \
    int checked_report(unsigned long long* count, unsigned long long* first);                  \
    void launch_mtz_check(const gk::Ctx& c, const double* u, int* flag, cudaStream_t s);       \
    void launch_ens_stage(int threads, int kind, int plm, const gk::EnsInst* inst,             \
                          const int2* tiles, int ntiles, unsigned* counter, double c1,          \
                          double c2, double c3, cudaStream_t s);                                \
    void launch_ens_bc(const gk::EnsInst* inst, int n, int which, int max_count,               \
                       cudaStream_t s);                                                        \
    void launch_ens_begin(const gk::EnsInst* inst, int n, double dtoutput, int steps,          \
                          cudaStream_t s);                                                     \
    }

GK_DECLARE_KERNEL_SET(gk_parity)
GK_DECLARE_KERNEL_SET(gk_fast)
