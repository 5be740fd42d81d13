// gk_api.cu -- the C ABI of include/gaukuk_cuda.h.
//
// A handle owns: three state buffers (A holds the state between steps; B and
// C are the RK stage results), the generic path's primitive and face-flux
// buffers (allocated only if that path runs), the device clock (DevTime) with
// its dt log, a stream, and a CUDA graph holding a fixed number of whole time
// steps.  Sim::Advance's loop runs on the device: every kernel of a step
// first reads DevTime::active, which the step epilogue (last CTA of the CFL
// kernel) clears once the output time, stepmax or an error ends the call.
// The host launches the graph repeatedly and only looks at `active` between
// batches, so surplus launches cost one no-op kernel each.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>

#include "gaukuk_cuda.h"
#include "gk_internal.h"

namespace gk_fast {
int fastmath_check(int n, unsigned long long seed, double* host_worst3);
}

namespace gk {

bool encode_rows_map(CUtensorMap* map, const double* base, const Geom& g, int nt) {
    // resolved through the runtime so the library has no link-time dependency
    // on the driver library
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    cuuint64_t dims[3] = {(cuuint64_t)g.pitch, (cuuint64_t)g.leny, 4};
    cuuint64_t strides[2] = {(cuuint64_t)g.pitch * sizeof(double),
                             (cuuint64_t)g.vstride * sizeof(double)};
    cuuint32_t box[3] = {(cuuint32_t)nt, 1, 4};
    cuuint32_t estr[3] = {1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace gk

namespace {

struct KernelSet {
    decltype(&gk_parity::launch_bc) bc;
    decltype(&gk_parity::launch_c2p) c2p;
    decltype(&gk_parity::launch_flux) flux;
    decltype(&gk_parity::launch_update) update;
    decltype(&gk_parity::launch_kick) kick;
    decltype(&gk_parity::launch_cfl) cfl;
    decltype(&gk_parity::launch_stage2d) stage2d;
    decltype(&gk_parity::launch_begin) begin;
    decltype(&gk_parity::launch_mtz_check) mtz_check;
    decltype(&gk_parity::launch_ens_stage) ens_stage;
    decltype(&gk_parity::launch_ens_bc) ens_bc;
    decltype(&gk_parity::launch_ens_begin) ens_begin;
    decltype(&gk_parity::launch_zflux) zflux;
    decltype(&gk_parity::launch_stage3d) stage3d;
    decltype(&gk_parity::launch_epilogue) epilogue;
    decltype(&gk_parity::launch_stage2d_learn) stage2d_learn;
    decltype(&gk_parity::launch_run1d) run1d;
};

const KernelSet kParity = {gk_parity::launch_bc,     gk_parity::launch_c2p,
                           gk_parity::launch_flux,   gk_parity::launch_update,
                           gk_parity::launch_kick,   gk_parity::launch_cfl,
                           gk_parity::launch_stage2d, gk_parity::launch_begin,
                           gk_parity::launch_mtz_check, gk_parity::launch_ens_stage,
                           gk_parity::launch_ens_bc,  gk_parity::launch_ens_begin,
                           gk_parity::launch_zflux,   gk_parity::launch_stage3d,
                           gk_parity::launch_epilogue, gk_parity::launch_stage2d_learn,
                           gk_parity::launch_run1d};
const KernelSet kFast = {gk_fast::launch_bc,     gk_fast::launch_c2p,     gk_fast::launch_flux,
                         gk_fast::launch_update, gk_fast::launch_kick,    gk_fast::launch_cfl,
                         gk_fast::launch_stage2d, gk_fast::launch_begin,  gk_fast::launch_mtz_check,
                         gk_fast::launch_ens_stage, gk_fast::launch_ens_bc, gk_fast::launch_ens_begin,
                         gk_fast::launch_zflux, gk_fast::launch_stage3d, gk_fast::launch_epilogue,
                         gk_fast::launch_stage2d_learn, gk_fast::launch_run1d};

constexpr int kLogCap = 1 << 20;

inline double smin(double a, double b) { return (b < a) ? b : a; }

// Reference var index (DEN,MTX,MTY,MTZ,ENG) -> device slot.
constexpr int kSlotOf[5] = {gk::S_DEN, gk::S_MTX, gk::S_MTY, gk::S_MTZ, gk::S_ENG};

// Optional per-launch event recording (gk_profile_steps).
struct Profiler {
    std::vector<int> cls;
    std::vector<cudaEvent_t> ev;  // pairs
};

}  // namespace

struct gk_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    gk_grid_desc gd{};
    gk_phys_desc pd{};
    gk::Ctx ctx{};
    const KernelSet* ks = nullptr;
    double *A = nullptr, *B = nullptr, *C = nullptr;
    double *W = nullptr, *F1 = nullptr, *F2 = nullptr, *F3 = nullptr;
    gk::DevTime* tm = nullptr;
    gk::DevTime* htm = nullptr;  // pinned mirror
    double* dlog = nullptr;
    int* dflag = nullptr;
    int path = 0;  // 0 generic, 1 fused 2D
    bool uploaded = false;
    int upload_step = 0;  // clock step at the last upload
    bool tiling_set = false;  // gk_set_tiling overrides the default tiling
    float* model = nullptr;   // learned flux correction (device), or null
    gk::FluxGate gate;
    int learn_fused = 1;      // the correction runs inside the fused 2D stage where it can
    // With periodic images (Phys::periodic_images) the steps fill no ghosts:
    // A's ghosts must be filled once after anything that leaves them stale
    // (an upload, a change of path or physics, an ensemble run).
    bool ghosts_dirty = true;
    double* fixed = nullptr;  // state at enrollment of fixed boundaries (device layout)
    gk::Shell* shells = nullptr;  // immersed body's shell table (device)
    int shell_cap = 0;
    bool mtz_plane_zero = false;  // 1D/2D: every stored MTZ value was +0.0 at upload
    long long io_up = 0, io_down = 0;  // bytes the last upload / download moved
    unsigned* fired = nullptr;  // faces where the detector kept plain HLLC
    int tiling_rows = 0;
    cudaGraphExec_t gexec = nullptr;
    int graph_steps = 0;
    int graph_path = -1;
    // sides whose ghost fill is a host routine (gk_set_host_fill)
    struct HostFill {
        int side, depth;
        gk_host_fill_fn fn;
        void* user;
        double* cons;
    };
    std::vector<HostFill> host_fills;
    int host_fill_rc = GK_OK;  // first failure inside a host fill, reported by the run
    std::string err;
};

namespace {

// An NVTX range over a public call (visible in Nsight timelines; free when
// no tool is attached).
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

int fail(gk_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

#define GK_CUDA(h, call)                                                                    \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail((h), GK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

long long round_up(long long a, long long b) { return (a + b - 1) / b * b; }

int build_ctx(gk_handle* h) {
    const gk_grid_desc& gd = h->gd;
    const gk_phys_desc& pd = h->pd;
    gk::Geom& g = h->ctx.g;
    gk::Phys& ph = h->ctx.ph;
    if (gd.nx <= 0 || gd.ny <= 0 || gd.nz <= 0 || gd.nghost < 0)
        return fail(h, GK_ERR_INVALID, "Invalid grid parameters from config");
    if (gd.nghost != 2)
        return fail(h, GK_ERR_UNSUPPORTED, "the device path is built for NGhost = 2");
    if ((gd.nx > 1 && gd.nx < gd.nghost) || (gd.ny > 1 && gd.ny < gd.nghost) ||
        (gd.nz > 1 && gd.nz < gd.nghost))
        return fail(h, GK_ERR_UNSUPPORTED, "a direction with more than one cell needs at least NGhost cells");
    if (gd.nx == 1 && (gd.ny > 1 || gd.nz > 1))
        return fail(h, GK_ERR_UNSUPPORTED, "x must be the first active direction");
    if (!(pd.gamma > 1.0)) return fail(h, GK_ERR_INVALID, "gamma must exceed 1");
    if (!(pd.cfl > 0.0)) return fail(h, GK_ERR_INVALID, "CFL must be positive");
    if (pd.mode != GK_MODE_PARITY && pd.mode != GK_MODE_FAST)
        return fail(h, GK_ERR_INVALID, "unknown arithmetic mode");
    if (pd.mode == GK_MODE_FAST && !(pd.dfloor > 0.0 && pd.pfloor > 0.0))
        return fail(h, GK_ERR_UNSUPPORTED, "fast mode needs positive density and pressure floors");
    g.nx = gd.nx; g.ny = gd.ny; g.nz = gd.nz; g.ng = gd.nghost;
    g.lenx = g.nx + 2 * g.ng; g.leny = g.ny + 2 * g.ng; g.lenz = g.nz + 2 * g.ng;
    g.ib = g.ng; g.ie = g.ib + g.nx;
    g.jb = g.ng; g.je = g.jb + g.ny;
    g.kb = g.ng; g.ke = g.kb + g.nz;
    g.ndim = g.nz > 1 ? 3 : (g.ny > 1 ? 2 : 1);
    g.pitch = (int)round_up(g.lenx, 16);
    g.nzs = g.nz > 1 ? g.lenz : 1;
    g.kofs = g.nz > 1 ? 0 : g.kb;
    g.kstride = (long long)g.pitch * g.leny;
    g.vstride = g.kstride * g.nzs;
    g.fpitch = (int)round_up(g.lenx + 1, 16);
    g.fkstride = (long long)g.fpitch * (g.leny + 1);
    g.fvstride = g.fkstride * (g.nzs + 1);
    // Domain (sim.cpp:16-36)
    g.dx = (gd.xmax - gd.xmin) / gd.nx;
    g.dy = (gd.ymax - gd.ymin) / gd.ny;
    g.dz = (gd.zmax - gd.zmin) / gd.nz;
    g.dxRec = 1. / g.dx;
    g.dyRec = 1. / g.dy;
    g.dzRec = 1. / g.dz;
    if (gd.ny <= 1) g.dyRec = 0;
    if (gd.nz <= 1) g.dzRec = 0;
    g.drmin = smin(smin(g.dx, g.dy), g.dz);
    g.xmin = gd.xmin;
    g.ymin = gd.ymin;
    g.zmin = gd.zmin;
    // EquationOfState (adiabatic.cpp:12-16), hllc.cpp:28-29
    ph.gamma = pd.gamma;
    ph.gm1 = pd.gamma - 1.0;
    ph.gm1Rec = 1.0 / (pd.gamma - 1.0);
    ph.gmRec = 1.0 / pd.gamma;
    ph.cq = 0.5 * (1 + ph.gmRec);
    ph.gm1Rec1 = ph.gm1Rec + 1.0;
    ph.gcq = ph.gamma * ph.cq;
    ph.hgm1 = 0.5 * ph.gm1;
    ph.cfl = pd.cfl;
    ph.dmin = pd.dfloor;
    ph.pmin = pd.pfloor;
    for (int d = 0; d < 3; ++d) ph.grav[d] = pd.grav[d];
    ph.has_grav = (pd.grav[0] != 0 || pd.grav[1] != 0 || pd.grav[2] != 0);
    ph.integrator = pd.integrator == 1 ? 1 : (pd.integrator == 3 ? 3 : 2);
    ph.plm = pd.rc_order != 1;
    ph.stepmax = pd.stepmax;
    // Boundary::Boundary (boundary.cpp:13-125): unknown ids copy; type 4
    // (fixed) takes the data given by gk_set_fixed_boundary.
    for (int s = 0; s < 6; ++s) {
        int t = pd.bc[s];
        if (t < 0 || t > 4) t = 0;
        ph.bc[s] = t;
    }
    ph.fixed_bd = nullptr;
    ph.fix_inner = 0;
    ph.npoint = 0;
    ph.shells = nullptr;
    ph.nshell = 0;
    ph.defer_epilogue = 0;
    ph.fill_z = 0;
    if (g.ndim == 3) {
        // z sides of type 0 run OutflowCopyYL/YR after the y fill
        // (boundary.cpp:92,104,109,121, 127-142): the y ghosts end as copies
        // and those z ghosts are never filled.
        for (int side = 0; side < 2; ++side) {
            if (ph.bc[4 + side] == 0) ph.bc[2 + side] = 0;
            else ph.fill_z |= 1 << side;
        }
    }
    h->ctx.has_vz = 1;
    return GK_OK;
}

int alloc_state(gk_handle* h) {
    const gk::Geom& g = h->ctx.g;
    size_t bytes = sizeof(double) * 5 * (size_t)g.vstride;
    GK_CUDA(h, cudaMalloc(&h->A, bytes));
    GK_CUDA(h, cudaMalloc(&h->B, bytes));
    GK_CUDA(h, cudaMemsetAsync(h->A, 0, bytes, h->stream));
    GK_CUDA(h, cudaMemsetAsync(h->B, 0, bytes, h->stream));
    if (h->ctx.ph.integrator == 3) {
        GK_CUDA(h, cudaMalloc(&h->C, bytes));
        GK_CUDA(h, cudaMemsetAsync(h->C, 0, bytes, h->stream));
    }
    GK_CUDA(h, cudaMalloc(&h->tm, sizeof(gk::DevTime)));
    GK_CUDA(h, cudaMalloc(&h->dlog, sizeof(double) * kLogCap));
    GK_CUDA(h, cudaMalloc(&h->dflag, sizeof(int)));
    GK_CUDA(h, cudaMallocHost(&h->htm, sizeof(gk::DevTime)));
    gk::DevTime t{};
    t.t = 0; t.dt = 1e10; t.tNext = 0; t.dtUntilOutput = 1e10;  // sim.cpp:45-46
    t.cmax_last = 1e-16;
    double seed = 1e-16;
    std::memcpy(&t.cmax_acc, &seed, sizeof(double));
    t.done_ctas = 0; t.step = 0; t.is_continue = 1; t.active = 0; t.status = 0;
    t.steps_left = -1; t.nlog = 0; t.log_cap = kLogCap; t.log = h->dlog;
    *h->htm = t;
    GK_CUDA(h, cudaMemcpyAsync(h->tm, h->htm, sizeof(gk::DevTime), cudaMemcpyHostToDevice, h->stream));
    GK_CUDA(h, cudaStreamSynchronize(h->stream));
    h->ctx.tm = h->tm;
    return GK_OK;
}

int alloc_generic(gk_handle* h) {
    if (h->W) return GK_OK;
    const gk::Geom& g = h->ctx.g;
    size_t sb = sizeof(double) * 5 * (size_t)g.vstride;
    size_t fb = sizeof(double) * 5 * (size_t)g.fvstride;
    GK_CUDA(h, cudaMalloc(&h->W, sb));
    GK_CUDA(h, cudaMalloc(&h->F1, fb));
    GK_CUDA(h, cudaMalloc(&h->F2, fb));
    GK_CUDA(h, cudaMalloc(&h->F3, fb));
    GK_CUDA(h, cudaMemsetAsync(h->W, 0, sb, h->stream));
    GK_CUDA(h, cudaMemsetAsync(h->F1, 0, fb, h->stream));
    GK_CUDA(h, cudaMemsetAsync(h->F2, 0, fb, h->stream));
    GK_CUDA(h, cudaMemsetAsync(h->F3, 0, fb, h->stream));
    return GK_OK;
}

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

// Tile shape of the fused 2D stage (threads per CTA, rows per tile), from the
// grid: enough tiles for every resident CTA slot (148 SMs x 512/threads), at
// most 24 rows.  Each tile repeats a 4-row prologue, so longer tiles do less
// work; but few waves of tiles leave a tail, and a small grid needs short
// tiles and narrow CTAs for every SM to get work.  Measured:
//   KH 4096^2, 128 threads, G zone-updates/s at 16 / 24 / 32 rows: fast
//   17.6 / 17.8 / 17.8, parity 7.37 / 7.40 / 7.31;
//   RT 1024x3072 (9 strips), same: fast 9.10 / 9.10 / 9.04, parity 4.09 /
//   4.01 / 3.45 (1.5 waves at 32 rows);
//   KH 256^2, us per step, 128 threads x 4 rows -> 64 x 2: fast 24.2 -> 20.7,
//   parity 52.8 -> 38.3; KH 512^2, 128 x 4 -> 64 x 4: fast 37.9 -> 33.4,
//   parity 92.7 -> 63.4.
// Parity mode's heavier cells want more waves of long tiles where a grid has
// more than one wave at 24 rows: it then aims at 4 waves with at least 12
// rows.  Parity, us per step at the rows chosen (12 / 16 / 24 rows):
// RT 1024x3072 761 (761 / 772 / 788), KH 2048^2 621 at 15 (625 / 631 / 666),
// KH 4096^2 2267 at 24.  Smaller grids keep the one-wave rule, which a tail
// wave would cost more than short tiles save: KH 1024^2 at 16 rows is one
// wave of 576 tiles, 189 us (12 rows: 234).
// GK_STAGE_THREADS / GK_STAGE_ROWS override (tuning).
int stage_threads_for(const gk::Geom& g) {
    const int v = env_int("GK_STAGE_THREADS", 0);
    if (v == 64 || v == 128 || v == 256) return v;
    const long long strips = (g.nx + 123) / 124;
    return (long long)g.ny * strips / (148 * 4) < 8 ? 64 : 128;
}

// The stage with the learned correction holds 256 threads per SM (its
// registers and shared memory), and a tile's time is about its rows plus
// half a row (the segment's first y faces).  Rows per segment: the r in
// [2, 24] that minimises waves x (r + 1/2).  KH 256^2 (CTAs of 64): 3 rows,
// one wave of 430 CTAs (the plain rule's 2 rows made two waves); 1024^2
// (CTAs of 128): 16 rows, two waves of 288.
int learn_stage_rows(const gk::Geom& g, int threads) {
    const long long nt = threads == 64 ? 64 : 128;
    const long long strips = (g.nx + nt - 5) / (nt - 4);
    const long long slots = 148LL * (256 / nt);
    int best = 2;
    double best_cost = 1e300;
    for (int r = 2; r <= 24; ++r) {
        const long long tiles = strips * ((g.ny + r - 1) / r);
        const double cost = (double)((tiles + slots - 1) / slots) * (r + 0.5);
        if (cost < best_cost) {
            best_cost = cost;
            best = r;
        }
    }
    return best;
}

int stage_rows(const gk::Geom& g, int threads, bool parity) {
    const int forced = env_int("GK_STAGE_ROWS", 0);
    if (forced > 0) return forced;
    const long long cols = threads - 4;
    const long long strips = (g.nx + cols - 1) / cols;
    const long long tiles = (long long)g.ny * strips, slots = 148LL * (512 / threads);
    const long long per_slot = (tiles + slots - 1) / slots;
    if (!parity || per_slot <= 24) return (int)std::max(2LL, std::min(24LL, per_slot));
    return (int)std::max(12LL, std::min(24LL, (tiles + 4 * slots - 1) / (4 * slots)));
}

// Path 1, the fused 2D stage, applies to 2D RK2/RK3 runs with MTZ
// identically zero, no z gravity (it would make MTZ non-zero) and no point
// masses (their kicks run between the fused stages' CFL reduction and the
// epilogue).  With a learned correction it takes the stage with the network
// at every face (TMA rows; unless gk_set_flux_model_fused turned that off).
// Path 2, the 3D stage (z fluxes, then one fused x-y stage per plane),
// applies to 3D RK2/RK3 runs (forward Euler updates in place, which the
// fused stage cannot).  Path 3, a 1D run in one CTA (k_run1d, many steps
// per launch), applies to 1D runs of up to 1024 cells per row (lenx) with
// the device's own ghost fills (copy, periodic, reflecting, outflow) and no
// source term, learned correction or host routine.  Path 0 is generic.
int choose_path(const gk_handle* h) {
    const gk::Ctx& c = h->ctx;
    if (c.g.ndim == 3 && c.ph.integrator != 1 && env_int("GK_STAGE3D", 1) != 0) return 2;
    if (c.g.ndim == 1) {
        bool own_fills = true;
        for (int s = 0; s < 2; ++s) own_fills = own_fills && c.ph.bc[s] >= 0 && c.ph.bc[s] <= 3;
        return (c.g.lenx <= 1024 && own_fills && !c.ph.has_grav && c.ph.npoint == 0 &&
                c.ph.nshell == 0 && !c.ph.fix_inner && !h->model && h->host_fills.empty() &&
                env_int("GK_RUN1D", 1) != 0) ? 3 : 0;
    }
    if (!(c.g.ndim == 2 && !c.has_vz && c.ph.integrator != 1 && c.ph.grav[2] == 0 &&
          c.ph.npoint == 0))
        return 0;
    if (!h->model) return 1;
    if (!h->learn_fused || !c.use_tma || !h->A) return 0;
    CUtensorMap probe;
    return gk::encode_rows_map(&probe, h->A, c.g, c.stage_threads == 64 ? 64 : 128) ? 1 : 0;
}

// The path, and whether the fused 2D stage writes the periodic ghost images
// itself (Phys::periodic_images): x and y periodic on both sides, no
// gravity kick between the fills and the stages, no host routine, fixed
// side, inner reset or immersed body, and at most 2^21 cells, where the
// ghost fills' launches are a visible part of a step (KH 256^2 fast: 21.0 ->
// 15.9 us per step, 1024^2: 77.5 -> 74.0; at 4096^2 the images cost 1 %).
void set_path(gk_handle* h) {
    h->path = choose_path(h);
    h->ghosts_dirty = true;
    const gk::Phys& ph = h->ctx.ph;
    bool periodic = true;
    for (int s = 0; s < 4; ++s) periodic = periodic && ph.bc[s] == 1;
    const bool small = (long long)h->ctx.g.nx * h->ctx.g.ny <= (1LL << 21);
    h->ctx.ph.periodic_images = (h->path == 1 && periodic && small && !ph.has_grav && ph.npoint == 0 &&
                                 ph.nshell == 0 && !ph.fix_inner && !ph.fixed_bd &&
                                 h->host_fills.empty() && env_int("GK_PERIODIC_IMAGES", 1) != 0)
                                    ? 1
                                    : 0;
}

// Sides filled by host routines (gk_set_host_fill), after the device ghost
// fill of buffer u: the stream is synchronised, the cells each routine may
// read (its ghost strip and `depth` layers next to it, every transverse
// index, every variable) are copied into its host array, the routines run in
// UpdateBD's side order (boundary.cpp:127-142), and each side's ghost strip
// (active transverse cells, as the routine writes it) goes back.  Skipped
// once the run has stopped, like the kernels.
int run_host_fills(gk_handle* h, double* u) {
    const gk::Geom& g = h->ctx.g;
    cudaStream_t s = h->stream;
    GK_CUDA(h, cudaMemcpyAsync(&h->htm->active, &h->tm->active, sizeof(int),
                               cudaMemcpyDeviceToHost, s));
    GK_CUDA(h, cudaStreamSynchronize(s));
    if (!h->htm->active) return GK_OK;
    const int n3[3] = {g.nx, g.ny, g.nz};
    const size_t db = sizeof(double);
    // ranges along each direction: [lo, hi)
    auto region = [&](int side, int depth, bool strip_only, int lo[3], int hi[3]) {
        const int dir = side / 2, sd = side % 2;
        const int len[3] = {g.lenx, g.leny, g.lenz};
        const int beg[3] = {g.ib, g.jb, g.kb}, end[3] = {g.ie, g.je, g.ke};
        for (int d = 0; d < 3; ++d) {
            lo[d] = strip_only ? beg[d] : 0;
            hi[d] = strip_only ? end[d] : len[d];
        }
        // depth >= n + nghost: the whole extent along dir
        const int reach = strip_only ? 0 : std::min(depth, n3[dir] + g.ng);
        lo[dir] = sd == 0 ? 0 : std::max(0, end[dir] - reach);
        hi[dir] = sd == 0 ? std::min(len[dir], g.ng + reach) : len[dir];
    };
    auto copy = [&](const gk_handle::HostFill& f, bool to_host) -> int {
        int lo[3], hi[3];
        region(f.side, f.depth, !to_host, lo, hi);
        for (int n = 0; n < 5; ++n)
            for (int k = std::max(lo[2], g.kofs); k < std::min(hi[2], g.kofs + g.nzs); ++k) {
                double* ref = f.cons + ((size_t)(n * g.lenz + k) * g.leny + lo[1]) * g.lenx + lo[0];
                double* dev = u + (size_t)kSlotOf[n] * g.vstride + (size_t)(k - g.kofs) * g.kstride +
                              (size_t)lo[1] * g.pitch + lo[0];
                const size_t w = db * (hi[0] - lo[0]);
                if (to_host)
                    GK_CUDA(h, cudaMemcpy2DAsync(ref, db * g.lenx, dev, db * g.pitch, w, hi[1] - lo[1],
                                                 cudaMemcpyDeviceToHost, s));
                else
                    GK_CUDA(h, cudaMemcpy2DAsync(dev, db * g.pitch, ref, db * g.lenx, w, hi[1] - lo[1],
                                                 cudaMemcpyHostToDevice, s));
            }
        return GK_OK;
    };
    int rc;
    for (const auto& f : h->host_fills)
        if ((rc = copy(f, true)) != GK_OK) return rc;
    GK_CUDA(h, cudaStreamSynchronize(s));
    for (const auto& f : h->host_fills)
        if (f.fn(f.user, f.cons) != 0)
            return fail(h, GK_ERR_INVALID, "a host boundary routine reported a failure");
    for (const auto& f : h->host_fills)
        if ((rc = copy(f, false)) != GK_OK) return rc;
    // the host arrays are read again by the next fill: let the copies finish
    GK_CUDA(h, cudaStreamSynchronize(s));
    return GK_OK;
}

// One time step.  Kernel order per RK stage follows Sim::RK2_/RK3_/
// ForwardEuler_ (rk2.cpp:11-23, rk3.cpp:11-29, forward_euler.cpp:11-18),
// wrapped in the Strang half kicks of sim.cpp:85-91; the step ends with the
// CFL reduction and epilogue.  The state is in A before and after.
void enqueue_step(gk_handle* h, Profiler* prof) {
    const KernelSet& k = *h->ks;
    const gk::Ctx& c = h->ctx;
    cudaStream_t s = h->stream;
    auto mark = [&](int cls) {
        if (!prof) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        prof->cls.push_back(cls);
        prof->ev.push_back(e);
    };
#define GK_L(cls, stmt) \
    do {                \
        mark(cls);      \
        stmt;           \
        mark(-1);       \
    } while (0)
    // ghost fill of a buffer: the device sides, then any host-routine sides
    auto fill = [&](double* u) {
        k.bc(c, u, s);
        if (!h->host_fills.empty() && h->host_fill_rc == GK_OK) h->host_fill_rc = run_host_fills(h, u);
    };
    double* A = h->A;
    double* B = h->B;
    double* Cb = h->C;
    const int integ = c.ph.integrator;
    const double frac13 = 1.0 / 3.0;
    if (c.ph.has_grav || c.ph.npoint) GK_L(gk::K_KICK, k.kick(c, A, 0, s));
    if (h->path == 3) {
        // the whole step in one launch (ghost fills, stages, CFL, epilogue)
        GK_L(gk::K_STAGE, k.run1d(c, A, B, 1, s));
        return;
    }
    if (h->path == 2) {
        // z fluxes of the stage's state into F3, then the fused x-y stage;
        // without a kick after it the last stage also reduces the CFL speed
        const bool kicks = c.ph.has_grav || c.ph.npoint;
        const int last = kicks ? 1 : 2;
        GK_L(gk::K_BC, fill(A));
        GK_L(gk::K_FLUX, k.zflux(c, A, h->F3, s));
        GK_L(gk::K_STAGE, k.stage3d(c, A, nullptr, B, h->F3, 0, 1.0, 1.0, 0.0, s));
        GK_L(gk::K_BC, fill(B));
        GK_L(gk::K_FLUX, k.zflux(c, B, h->F3, s));
        if (integ == 3) {
            GK_L(gk::K_STAGE, k.stage3d(c, B, A, Cb, h->F3, 1, 0.75, 0.25, 0.25, s));
            GK_L(gk::K_BC, fill(Cb));
            GK_L(gk::K_FLUX, k.zflux(c, Cb, h->F3, s));
            GK_L(gk::K_STAGE, k.stage3d(c, Cb, A, A, h->F3, last, frac13, 2 * frac13, 2 * frac13, s));
        } else {
            GK_L(gk::K_STAGE, k.stage3d(c, B, A, A, h->F3, last, 0.5, 0.5, 0.5, s));
        }
        if (kicks) {
            GK_L(gk::K_KICK, k.kick(c, A, 1, s));
            GK_L(gk::K_CFL, k.cfl(c, A, 1, s));
        }
        return;
    }
    if (h->path == 1) {
        // the last stage also applies the second half kick, the CFL
        // reduction and the step epilogue; with a learned correction the
        // stage applies it at every face
        auto stage = [&](const double* uc, const double* u0, double* out, int kind, double c1,
                         double c2, double c3) {
            if (h->model)
                k.stage2d_learn(c, uc, u0, out, kind, c1, c2, c3, h->model, h->gate, h->fired, s);
            else
                k.stage2d(c, uc, u0, out, kind, c1, c2, c3, s);
        };
        // with periodic images the stages write the ghosts themselves (the
        // run fills A once before its first step)
        const bool fills = !c.ph.periodic_images;
        if (fills) GK_L(gk::K_BC, fill(A));
        GK_L(gk::K_STAGE, stage(A, nullptr, B, 0, 1.0, 1.0, 0.0));
        if (fills) GK_L(gk::K_BC, fill(B));
        if (integ == 3) {
            GK_L(gk::K_STAGE, stage(B, A, Cb, 1, 0.75, 0.25, 0.25));
            if (fills) GK_L(gk::K_BC, fill(Cb));
            GK_L(gk::K_STAGE, stage(Cb, A, A, 2, frac13, 2 * frac13, 2 * frac13));
        } else {
            GK_L(gk::K_STAGE, stage(B, A, A, 2, 0.5, 0.5, 0.5));
        }
        return;
    }
    auto fluxes = [&](const double* u) {
        GK_L(gk::K_C2P, k.c2p(c, u, h->W, s));
        GK_L(gk::K_FLUX, k.flux(c, 0, h->W, h->F1, s));
        if (c.g.ndim >= 2) GK_L(gk::K_FLUX, k.flux(c, 1, h->W, h->F2, s));
        if (c.g.ndim == 3) GK_L(gk::K_FLUX, k.flux(c, 2, h->W, h->F3, s));
        if (h->model) {
            // learned correction of the face fluxes (gk_mlp.cu)
            GK_L(gk::K_FLUX, gk::launch_flux_correct(h->model, h->W, h->F1, c.g, c.ph, c.tm, 0,
                                                     h->gate, h->fired, s));
            GK_L(gk::K_FLUX, gk::launch_flux_correct(h->model, h->W, h->F2, c.g, c.ph, c.tm, 1,
                                                     h->gate, h->fired, s));
        }
    };
    GK_L(gk::K_BC, fill(A));
    fluxes(A);
    if (integ == 1) {
        GK_L(gk::K_UPDATE, k.update(c, nullptr, A, A, h->F1, h->F2, h->F3, 0, 1.0, 1.0, 0.0, s));
    } else {
        GK_L(gk::K_UPDATE, k.update(c, nullptr, A, B, h->F1, h->F2, h->F3, 0, 1.0, 1.0, 0.0, s));
        GK_L(gk::K_BC, fill(B));
        fluxes(B);
        if (integ == 3) {
            GK_L(gk::K_UPDATE, k.update(c, A, B, B, h->F1, h->F2, h->F3, 1, 0.75, 0.25, 0.25, s));
            GK_L(gk::K_BC, fill(B));
            fluxes(B);
            GK_L(gk::K_UPDATE, k.update(c, A, B, A, h->F1, h->F2, h->F3, 1, frac13, 2 * frac13,
                                        2 * frac13, s));
        } else {
            GK_L(gk::K_UPDATE, k.update(c, A, B, A, h->F1, h->F2, h->F3, 1, 0.5, 0.5, 0.5, s));
        }
    }
    if (c.ph.has_grav || c.ph.npoint) GK_L(gk::K_KICK, k.kick(c, A, 1, s));
    GK_L(gk::K_CFL, k.cfl(c, A, 1, s));
#undef GK_L
}

int steps_per_graph_of(const gk::Geom& g) {
    long long cells = (long long)g.nx * g.ny * g.nz;
    if (cells >= (1LL << 22)) return 2;
    if (cells >= (1LL << 18)) return 8;
    return 32;
}

int ensure_graph(gk_handle* h) {
    if (h->gexec && h->graph_path == h->path) return GK_OK;
    if (h->gexec) {
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
    }
    h->graph_steps = steps_per_graph_of(h->ctx.g);
    cudaGraph_t graph;
    GK_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    if (h->path == 3)  // one launch runs the graph's steps
        h->ks->run1d(h->ctx, h->A, h->B, h->graph_steps, h->stream);
    else
        for (int i = 0; i < h->graph_steps; ++i) enqueue_step(h, nullptr);
    GK_CUDA(h, cudaStreamEndCapture(h->stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&h->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(h, GK_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    h->graph_path = h->path;
    return GK_OK;
}

int pull_time(gk_handle* h) {
    GK_CUDA(h, cudaMemcpyAsync(h->htm, h->tm, sizeof(gk::DevTime), cudaMemcpyDeviceToHost, h->stream));
    GK_CUDA(h, cudaStreamSynchronize(h->stream));
    return GK_OK;
}

// A reference-layout host state (NVar x lenz x leny x lenx) into a device
// state buffer (slots DEN, MTX, MTY, ENG, MTZ; stored planes; pitched rows).
// Stored planes of reference variable n (all five when n < 0).
int copy_ref_to_device(gk_handle* h, const double* ref, double* dev, int only = -1) {
    const gk::Geom& g = h->ctx.g;
    for (int n = 0; n < 5; ++n) {
        if (only >= 0 && n != only) continue;
        for (int kk = 0; kk < g.nzs; ++kk) {
            const int k = g.kofs + kk;
            const double* src = ref + ((size_t)(n * g.lenz + k) * g.leny) * g.lenx;
            double* dst = dev + (size_t)kSlotOf[n] * g.vstride + (size_t)kk * g.kstride;
            GK_CUDA(h, cudaMemcpy2DAsync(dst, sizeof(double) * g.pitch, src, sizeof(double) * g.lenx,
                                         sizeof(double) * g.lenx, g.leny, cudaMemcpyHostToDevice,
                                         h->stream));
        }
    }
    return GK_OK;
}

// Whether every one of the n doubles at p has the bit pattern of +0.0; a
// few host threads share the scan (it runs while the other planes copy).
bool host_all_zero(const double* p, size_t n) {
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t parts = std::max<size_t>(1, std::min<size_t>(hw ? hw : 1, 8));
    std::vector<unsigned char> zero(parts, 1);
    auto scan = [&](size_t part) {
        const size_t lo = n * part / parts, hi = n * (part + 1) / parts;
        unsigned long long acc = 0;
        for (size_t i = lo; i < hi; ++i) {
            unsigned long long b;
            std::memcpy(&b, p + i, sizeof b);
            acc |= b;
        }
        zero[part] = acc == 0;
    };
    std::vector<std::thread> pool;
    for (size_t part = 1; part < parts; ++part) pool.emplace_back(scan, part);
    scan(0);
    for (auto& t : pool) t.join();
    for (unsigned char z : zero)
        if (!z) return false;
    return true;
}

// A change of the physics that kernels take by value: the captured graph
// is rebuilt at the next launch, and the path follows.
int physics_changed(gk_handle* h) {
    if (h->ctx.ph.npoint || h->ctx.ph.nshell) h->ctx.has_vz = 1;  // see gk_upload_cons
    if (h->gexec) {
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
        h->graph_steps = 0;
    }
    if (h->uploaded) {
        set_path(h);
        if (h->path != 1) return alloc_generic(h);
    }
    return GK_OK;
}

// The device status word after a run: a TMA row wait that gave up (the
// stage kernel's waits are bounded), or a non-finite CFL reduction.
int status_error(gk_handle* h) {
    const int st = h->htm->status;
    if (st & gk::STATUS_TMA_TIMEOUT)
        return fail(h, GK_ERR_CUDA, "a TMA row load did not complete within the stage kernel's wait limit");
    if (st & gk::STATUS_NO_MAP)
        return fail(h, GK_ERR_CUDA, "the learned stage's tensor map could not be encoded");
    if (st) return fail(h, GK_ERR_NONFINITE, "CFL reduction met a non-finite state");
    return GK_OK;
}

int check_ready(gk_handle* h) {
    if (!h) return GK_ERR_INVALID;
    if (!h->uploaded) return fail(h, GK_ERR_STATE, "no state uploaded");
    for (int s = 0; s < 6; ++s)
        if (h->ctx.ph.bc[s] == 4 && !h->ctx.ph.fixed_bd)
            return fail(h, GK_ERR_STATE, "fixed (type 4) boundary data not set (gk_set_fixed_boundary)");
    GK_CUDA(h, cudaSetDevice(h->device));
    return GK_OK;
}

}  // namespace

extern "C" {

int gk_create(const gk_grid_desc* grid, const gk_phys_desc* phys, gk_handle** out) {
    if (!grid || !phys || !out) return GK_ERR_INVALID;
    *out = nullptr;
    gk_handle* h = new gk_handle();
    h->gd = *grid;
    h->pd = *phys;
    h->device = phys->device;
    int rc = build_ctx(h);
    if (rc != GK_OK) {
        std::fprintf(stderr, "gk_create: %s\n", h->err.c_str());
        delete h;
        return rc;
    }
    h->ks = phys->mode == GK_MODE_FAST ? &kFast : &kParity;
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "gk_create: %s\n", cudaGetErrorString(e));
        delete h;
        return GK_ERR_CUDA;
    }
    rc = alloc_state(h);
    if (rc != GK_OK) {
        std::fprintf(stderr, "gk_create: %s\n", h->err.c_str());
        gk_destroy(h);
        return rc;
    }
    *out = h;
    return GK_OK;
}

void gk_destroy(gk_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    for (double* p : {h->A, h->B, h->C, h->W, h->F1, h->F2, h->F3, h->dlog, h->fixed}) cudaFree(p);
    cudaFree(h->model);
    cudaFree(h->fired);
    cudaFree(h->shells);
    cudaFree(h->tm);
    cudaFree(h->dflag);
    if (h->htm) cudaFreeHost(h->htm);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

long long gk_state_size(const gk_handle* h) {
    if (!h) return 0;
    const gk::Geom& g = h->ctx.g;
    return 5LL * g.lenz * g.leny * g.lenx;
}

int gk_upload_cons(gk_handle* h, const double* cons) {
    Range range("gk_upload_cons");
    if (!h || !cons) return GK_ERR_INVALID;
    GK_CUDA(h, cudaSetDevice(h->device));
    const gk::Geom& g = h->ctx.g;
    const size_t plane_bytes = sizeof(double) * (size_t)g.lenx * g.leny;
    // In 1D/2D the z momentum is usually zero everywhere: the other four
    // variables are copied while the host checks its plane, and a plane that
    // is +0.0 in every stored cell is cleared on the device instead of copied.
    h->mtz_plane_zero = false;
    h->io_up = 5LL * g.nzs * (long long)plane_bytes;
    if (g.ndim <= 2 && g.nzs == 1) {
        for (int n : {0, 1, 2, 4}) {
            int rc = copy_ref_to_device(h, cons, h->A, n);
            if (rc != GK_OK) return rc;
        }
        const double* mz = cons + ((size_t)(3 * g.lenz + g.kofs) * g.leny) * g.lenx;
        if (host_all_zero(mz, (size_t)g.lenx * g.leny)) {
            h->mtz_plane_zero = true;
            h->io_up -= (long long)plane_bytes;
            GK_CUDA(h, cudaMemsetAsync(h->A + (size_t)gk::S_MTZ * g.vstride, 0,
                                       sizeof(double) * (size_t)g.vstride, h->stream));
        } else {
            int rc = copy_ref_to_device(h, cons, h->A, 3);
            if (rc != GK_OK) return rc;
        }
    } else {
        int rc0 = copy_ref_to_device(h, cons, h->A);
        if (rc0 != GK_OK) return rc0;
    }
    // Path: the fused kernel evolves four variables; it applies when the run
    // is 2D and MTZ is zero on every active cell (it then stays zero).
    h->ctx.has_vz = 1;
    if (g.ndim <= 2 && h->mtz_plane_zero) {
        h->ctx.has_vz = 0;
    } else if (g.ndim <= 2) {
        GK_CUDA(h, cudaMemsetAsync(h->dflag, 0, sizeof(int), h->stream));
        h->ks->mtz_check(h->ctx, h->A, h->dflag, h->stream);
        int flag = 0;
        GK_CUDA(h, cudaMemcpyAsync(&flag, h->dflag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        GK_CUDA(h, cudaStreamSynchronize(h->stream));
        h->ctx.has_vz = flag;
    }
    // a point mass off the mid-plane makes MTZ non-zero during the run; an
    // immersed body writes MTZ (signed zeros in 2D) into its shell cells
    if (h->ctx.ph.npoint || h->ctx.ph.nshell) h->ctx.has_vz = 1;
    set_path(h);
    h->ctx.use_tma = env_int("GK_STAGE_TMA", 1) != 0;
    if (!h->tiling_set) {
        h->ctx.stage_threads = stage_threads_for(g);
        h->ctx.h2d_rows = stage_rows(g, h->ctx.stage_threads, h->ks == &kParity);
        h->ctx.learn_rows = learn_stage_rows(g, h->ctx.stage_threads);
    } else {
        h->ctx.h2d_rows = h->tiling_rows;
        h->ctx.learn_rows = 0;
    }
    if (h->path != 1) {
        int rc = alloc_generic(h);
        if (rc != GK_OK) return rc;
    }
    // reset the step machinery; the clock (t, step, isContinue) is kept
    int rc = pull_time(h);
    if (rc != GK_OK) return rc;
    gk::DevTime t = *h->htm;
    double seed = 1e-16;
    std::memcpy(&t.cmax_acc, &seed, sizeof(double));
    t.floor_den = 0;
    t.floor_pre = 0;
    t.done_ctas = 0;
    t.status = 0;
    t.nlog = 0;
    t.active = 0;
    *h->htm = t;
    GK_CUDA(h, cudaMemcpyAsync(h->tm, h->htm, sizeof(gk::DevTime), cudaMemcpyHostToDevice, h->stream));
    h->ks->cfl(h->ctx, h->A, 0, h->stream);
    GK_CUDA(h, cudaGetLastError());
    rc = pull_time(h);
    if (rc != GK_OK) return rc;
    h->uploaded = true;
    h->upload_step = h->htm->step;
    if (h->htm->status) return fail(h, GK_ERR_NONFINITE, "non-finite state in the uploaded array");
    return GK_OK;
}

static int download(gk_handle* h, double* cons, bool zero_other_planes) {
    Range range("gk_download");
    int rc = check_ready(h);
    if (rc != GK_OK) return rc;
    if (!cons) return GK_ERR_INVALID;
    rc = pull_time(h);
    if (rc != GK_OK) return rc;
    const gk::Geom& g = h->ctx.g;
    // The fused 2D path never writes MTZ, so a plane cleared at upload is
    // still +0.0 everywhere (no fixed data can fill its ghosts): a planes-only
    // download leaves the caller's plane as it is.
    const bool skip_mtz = !zero_other_planes && h->mtz_plane_zero && h->path == 1 &&
                          !h->ctx.ph.fixed_bd;
    h->io_down = 0;
    for (int n = 0; n < 5; ++n) {
        if (skip_mtz && n == 3) continue;
        for (int kk = 0; kk < g.nzs; ++kk) {
            const int k = g.kofs + kk;
            double* dst = cons + ((size_t)(n * g.lenz + k) * g.leny) * g.lenx;
            const double* src = h->A + (size_t)kSlotOf[n] * g.vstride + (size_t)kk * g.kstride;
            GK_CUDA(h, cudaMemcpy2DAsync(dst, sizeof(double) * g.lenx, src, sizeof(double) * g.pitch,
                                         sizeof(double) * g.lenx, g.leny, cudaMemcpyDeviceToHost,
                                         h->stream));
            h->io_down += (long long)sizeof(double) * g.lenx * g.leny;
        }
    }
    // Ghost strips as the reference leaves them after a step: Sim's integrators
    // end with cons.Swap(consTemp) (rk2.cpp:21, rk3.cpp:27), so the written
    // array carries the ghost fill of the last intermediate stage state.  That
    // fill sits in the stage buffer (B, or C for the fused RK3 path); the
    // strips of active rows/columns are taken from there.  Euler runs in place
    // and 1D y rows follow the reference's in-place order, so both keep A's.
    const double* donor = nullptr;
    if (h->htm->step > h->upload_step && h->ctx.ph.integrator != 1)
        donor = ((h->path == 1 || h->path == 2) && h->ctx.ph.integrator == 3) ? h->C : h->B;
    if (donor) {
        const size_t rowb = sizeof(double) * g.lenx, prow = sizeof(double) * g.pitch;
        for (int n = 0; n < 5; ++n) {
            if (skip_mtz && n == 3) continue;
            for (int kk = 0; kk < g.nzs; ++kk) {
                const int k = g.kofs + kk;
                if (k < g.kb || k >= g.ke) continue;
                double* dst = cons + ((size_t)(n * g.lenz + k) * g.leny) * g.lenx;
                const double* src = donor + (size_t)kSlotOf[n] * g.vstride + (size_t)kk * g.kstride;
                if (g.nx > 1) {
                    for (int side = 0; side < 2; ++side) {
                        const int i0 = side == 0 ? 0 : g.ie;
                        GK_CUDA(h, cudaMemcpy2DAsync(dst + (size_t)g.jb * g.lenx + i0, rowb,
                                                     src + (size_t)g.jb * g.pitch + i0, prow,
                                                     sizeof(double) * g.ng, g.ny,
                                                     cudaMemcpyDeviceToHost, h->stream));
                        h->io_down += (long long)sizeof(double) * g.ng * g.ny;
                    }
                }
                if (g.ny > 1) {
                    for (int side = 0; side < 2; ++side) {
                        const int j0 = side == 0 ? 0 : g.je;
                        GK_CUDA(h, cudaMemcpy2DAsync(dst + (size_t)j0 * g.lenx + g.ib, rowb,
                                                     src + (size_t)j0 * g.pitch + g.ib, prow,
                                                     sizeof(double) * g.nx, g.ng,
                                                     cudaMemcpyDeviceToHost, h->stream));
                        h->io_down += (long long)sizeof(double) * g.nx * g.ng;
                    }
                }
            }
            if (g.nz > 1) {
                for (int side = 0; side < 2; ++side) {
                    if (!((h->ctx.ph.fill_z >> side) & 1)) continue;
                    for (int gi = 0; gi < g.ng; ++gi) {
                        const int k = side == 0 ? gi : g.ke + gi;
                        double* dst = cons + ((size_t)(n * g.lenz + k) * g.leny) * g.lenx;
                        const double* src = donor + (size_t)kSlotOf[n] * g.vstride +
                                            (size_t)(k - g.kofs) * g.kstride;
                        GK_CUDA(h, cudaMemcpy2DAsync(dst + (size_t)g.jb * g.lenx + g.ib, rowb,
                                                     src + (size_t)g.jb * g.pitch + g.ib, prow,
                                                     sizeof(double) * g.nx, g.ny,
                                                     cudaMemcpyDeviceToHost, h->stream));
                        h->io_down += (long long)sizeof(double) * g.nx * g.ny;
                    }
                }
            }
        }
    }
    if (g.nzs == 1 && zero_other_planes) {
        const size_t plane = (size_t)g.leny * g.lenx;
        for (int n = 0; n < 5; ++n)
            for (int k = 0; k < g.lenz; ++k)
                if (k != g.kofs) std::memset(cons + (size_t)(n * g.lenz + k) * plane, 0, plane * sizeof(double));
    }
    GK_CUDA(h, cudaStreamSynchronize(h->stream));
    return GK_OK;
}

int gk_download_cons(gk_handle* h, double* cons) { return download(h, cons, true); }
int gk_download_planes(gk_handle* h, double* cons) { return download(h, cons, false); }

int gk_floor_hits(gk_handle* h, unsigned long long* density, unsigned long long* pressure) {
    if (!h) return GK_ERR_INVALID;
    int rc = pull_time(h);
    if (rc != GK_OK) return rc;
    if (density) *density = h->htm->floor_den;
    if (pressure) *pressure = h->htm->floor_pre;
    return GK_OK;
}

int gk_io_bytes(const gk_handle* h, long long* upload, long long* download) {
    if (!h) return GK_ERR_INVALID;
    if (upload) *upload = h->io_up;
    if (download) *download = h->io_down;
    return GK_OK;
}

// With periodic images the steps fill no ghosts, so A's are filled before a
// run's first step when they may be stale (after the begin kernel: the fill
// runs only while the run is active).
static void refill_ghosts(gk_handle* h) {
    if (!h->ctx.ph.periodic_images || !h->ghosts_dirty) return;
    h->ks->bc(h->ctx, h->A, h->stream);
    h->ghosts_dirty = false;
}

// Runs with host-routine sides: no graph (each ghost fill returns to the
// host), every step enqueued and finished in turn.
static int run_loop_host(gk_handle* h, double dtoutput, int nsteps) {
    h->host_fill_rc = GK_OK;
    h->ks->begin(h->ctx, dtoutput, nsteps, h->stream);
    GK_CUDA(h, cudaGetLastError());
    for (int i = 0; nsteps <= 0 || i < nsteps; ++i) {
        enqueue_step(h, nullptr);
        if (h->host_fill_rc != GK_OK) return h->host_fill_rc;
        GK_CUDA(h, cudaMemcpyAsync(&h->htm->active, &h->tm->active, sizeof(int),
                                   cudaMemcpyDeviceToHost, h->stream));
        GK_CUDA(h, cudaStreamSynchronize(h->stream));
        if (!h->htm->active) break;
    }
    GK_CUDA(h, cudaGetLastError());
    return pull_time(h);
}

static int run_loop(gk_handle* h, double dtoutput, int nsteps, bool wait) {
    if (!h->host_fills.empty()) return run_loop_host(h, dtoutput, nsteps);
    int rc = ensure_graph(h);
    if (rc != GK_OK) return rc;
    h->ks->begin(h->ctx, dtoutput, nsteps, h->stream);
    refill_ghosts(h);
    GK_CUDA(h, cudaGetLastError());
    if (nsteps > 0) {
        int launches = (nsteps + h->graph_steps - 1) / h->graph_steps;
        for (int i = 0; i < launches; ++i) GK_CUDA(h, cudaGraphLaunch(h->gexec, h->stream));
        if (!wait) return GK_OK;
        return pull_time(h);
    }
    int batch = 1;
    for (;;) {
        for (int i = 0; i < batch; ++i) GK_CUDA(h, cudaGraphLaunch(h->gexec, h->stream));
        GK_CUDA(h, cudaMemcpyAsync(&h->htm->active, &h->tm->active, sizeof(int),
                                   cudaMemcpyDeviceToHost, h->stream));
        GK_CUDA(h, cudaStreamSynchronize(h->stream));
        if (!h->htm->active) break;
        batch = std::min(batch * 2, 64);
    }
    return pull_time(h);
}

int gk_advance(gk_handle* h, double dtoutput, double* t, int* step, int* is_continue) {
    Range range("gk_advance");
    int rc = check_ready(h);
    if (rc != GK_OK) return rc;
    rc = run_loop(h, dtoutput, 0, true);
    if (rc != GK_OK) return rc;
    if (t) *t = h->htm->t;
    if (step) *step = h->htm->step;
    if (is_continue) *is_continue = h->htm->is_continue;
    if (h->htm->status) return status_error(h);
    return GK_OK;
}

int gk_run_steps(gk_handle* h, int nsteps, int* done) {
    Range range("gk_run_steps");
    int rc = check_ready(h);
    if (rc != GK_OK) return rc;
    if (nsteps <= 0) {
        if (done) *done = 0;
        return GK_OK;
    }
    rc = pull_time(h);
    if (rc != GK_OK) return rc;
    const int before = h->htm->step;
    rc = run_loop(h, 0.0, nsteps, true);
    if (rc != GK_OK) return rc;
    if (done) *done = h->htm->step - before;
    if (h->htm->status) return status_error(h);
    return GK_OK;
}

int gk_enqueue_steps(gk_handle* h, int nsteps) {
    Range range("gk_enqueue_steps");
    int rc = check_ready(h);
    if (rc != GK_OK) return rc;
    if (nsteps <= 0) return GK_OK;
    return run_loop(h, 0.0, nsteps, false);
}

int gk_get_time(gk_handle* h, double* t, double* dt, int* step, int* is_continue) {
    if (!h) return GK_ERR_INVALID;
    GK_CUDA(h, cudaSetDevice(h->device));
    int rc = pull_time(h);
    if (rc != GK_OK) return rc;
    if (t) *t = h->htm->t;
    if (dt) *dt = h->htm->dt;
    if (step) *step = h->htm->step;
    if (is_continue) *is_continue = h->htm->is_continue;
    return GK_OK;
}

int gk_set_time(gk_handle* h, double t, int step) {
    if (!h) return GK_ERR_INVALID;
    GK_CUDA(h, cudaSetDevice(h->device));
    int rc = pull_time(h);
    if (rc != GK_OK) return rc;
    h->htm->t = t;
    h->htm->step = step;
    h->htm->is_continue = !(h->ctx.ph.stepmax > 0 && step >= h->ctx.ph.stepmax);
    GK_CUDA(h, cudaMemcpyAsync(h->tm, h->htm, sizeof(gk::DevTime), cudaMemcpyHostToDevice, h->stream));
    GK_CUDA(h, cudaStreamSynchronize(h->stream));
    return GK_OK;
}

int gk_dt_log(gk_handle* h, double* buf, int cap, int* n) {
    if (!h) return GK_ERR_INVALID;
    GK_CUDA(h, cudaSetDevice(h->device));
    int rc = pull_time(h);
    if (rc != GK_OK) return rc;
    int total = h->htm->nlog;
    int avail = std::min(total, kLogCap);
    int m = std::min(avail, cap);
    if (buf && m > 0)
        GK_CUDA(h, cudaMemcpy(buf, h->dlog, sizeof(double) * m, cudaMemcpyDeviceToHost));
    if (n) *n = total;
    return GK_OK;
}

int gk_cmax(gk_handle* h, double* cmax) {
    int rc = check_ready(h);
    if (rc != GK_OK) return rc;
    h->ks->cfl(h->ctx, h->A, 0, h->stream);
    GK_CUDA(h, cudaGetLastError());
    rc = pull_time(h);
    if (rc != GK_OK) return rc;
    if (cmax) *cmax = h->htm->cmax_last;
    return GK_OK;
}

int gk_stream(gk_handle* h, void** stream) {
    if (!h || !stream) return GK_ERR_INVALID;
    *stream = (void*)h->stream;
    return GK_OK;
}

int gk_path(gk_handle* h, int* path) {
    if (!h || !path) return GK_ERR_INVALID;
    *path = h->path;
    return GK_OK;
}

int gk_graph_info(gk_handle* h, int* steps_per_graph, int* launches_per_step) {
    if (!h) return GK_ERR_INVALID;
    const gk::Ctx& c = h->ctx;
    const int stages = c.ph.integrator;  // 1, 2 or 3 stages
    int per;
    // immersed body and inner reset after each ghost fill
    const int inner = (c.ph.fix_inner ? 1 : 0) + (c.ph.nshell > 0 ? 1 : 0);
    if (h->path == 1) {
        // kick, (ghost fill + stage) per stage; with periodic images the stage alone
        per = (c.ph.has_grav ? 1 : 0) + (c.ph.periodic_images ? 1 : 2 + inner) * stages;
    } else if (h->path == 2) {
        per = (c.ph.has_grav || c.ph.npoint ? 3 : 0) + (3 + inner) * stages;
    } else if (h->path == 3) {
        per = 1;  // in a graph, one launch runs all of its steps
    } else {
        per = (c.ph.has_grav || c.ph.npoint ? 2 : 0) + stages * (3 + inner + c.g.ndim) + 1;
    }
    if (steps_per_graph) *steps_per_graph = steps_per_graph_of(c.g);
    if (launches_per_step) *launches_per_step = per;
    return GK_OK;
}

int gk_profile_steps(gk_handle* h, int nsteps, char* names, int names_cap, double* total_ms,
                     int* launches, int cap, int* n) {
    int rc = check_ready(h);
    if (rc != GK_OK) return rc;
    h->ks->begin(h->ctx, 0.0, nsteps, h->stream);
    refill_ghosts(h);
    Profiler prof;
    for (int i = 0; i < nsteps; ++i) enqueue_step(h, &prof);
    GK_CUDA(h, cudaStreamSynchronize(h->stream));
    std::vector<double> ms(gk::K_NCLASS, 0.0);
    std::vector<int> cnt(gk::K_NCLASS, 0);
    for (size_t i = 0; i + 1 < prof.ev.size(); i += 2) {
        float t = 0.f;
        cudaEventElapsedTime(&t, prof.ev[i], prof.ev[i + 1]);
        ms[prof.cls[i]] += t;
        cnt[prof.cls[i]] += 1;
    }
    for (cudaEvent_t e : prof.ev) cudaEventDestroy(e);
    std::string nm;
    int m = 0;
    for (int c = 0; c < gk::K_NCLASS; ++c) {
        if (!cnt[c]) continue;
        if (m < cap) {
            if (total_ms) total_ms[m] = ms[c];
            if (launches) launches[m] = cnt[c];
        }
        nm += (m ? ";" : "");
        nm += gk::kClassNames[c];
        ++m;
    }
    if (names && names_cap > 0) {
        std::strncpy(names, nm.c_str(), names_cap - 1);
        names[names_cap - 1] = 0;
    }
    if (n) *n = m;
    return pull_time(h);
}

int gk_checked_report(unsigned long long* count, unsigned long long* first) {
    if (!count || !first) return GK_ERR_INVALID;
    unsigned long long c[2] = {0, 0}, f[2] = {0, 0};
    const int a = gk_parity::checked_report(&c[0], &f[0]);
    const int b = gk_fast::checked_report(&c[1], &f[1]);
    if (a > 0 || b > 0) return GK_ERR_UNSUPPORTED;
    if (a < 0 || b < 0) return GK_ERR_CUDA;
    *count = c[0] + c[1];
    *first = c[0] ? f[0] : f[1];
    return GK_OK;
}

int gk_fastmath_check(int n, unsigned long long seed, double* worst3) {
    if (n <= 0 || !worst3) return GK_ERR_INVALID;
    return gk_fast::fastmath_check(n, seed, worst3) == 0 ? GK_OK : GK_ERR_CUDA;
}


const char* gk_strerror(int status) {
    switch (status) {
        case GK_OK: return "ok";
        case GK_ERR_INVALID: return "invalid argument or configuration";
        case GK_ERR_CUDA: return "CUDA runtime error";
        case GK_ERR_NONFINITE: return "non-finite state in the CFL reduction";
        case GK_ERR_UNSUPPORTED: return "configuration not supported by the device path";
        case GK_ERR_STATE: return "call out of order";
        default: return "unknown status";
    }
}

const char* gk_last_error(const gk_handle* h) { return h ? h->err.c_str() : ""; }

}  // extern "C"

// Context of a descriptor pair without a handle, for entry points that take
// caller-owned buffers (gk_noalloc.cu).  Returns a GK_* status; *err gets
// the reason on failure.
int gk_internal_build_ctx(const gk_grid_desc* gd, const gk_phys_desc* pd, gk::Ctx* ctx,
                          std::string* err) {
    gk_handle tmp;
    tmp.gd = *gd;
    tmp.pd = *pd;
    const int rc = build_ctx(&tmp);
    if (rc != GK_OK) {
        if (err) *err = tmp.err;
        return rc;
    }
    tmp.ctx.use_tma = env_int("GK_STAGE_TMA", 1) != 0;
    tmp.ctx.stage_threads = stage_threads_for(tmp.ctx.g);
    tmp.ctx.h2d_rows = stage_rows(tmp.ctx.g, tmp.ctx.stage_threads, pd->mode != GK_MODE_FAST);
    *ctx = tmp.ctx;
    return GK_OK;
}

// ------------------------------------------------------------ tiling
extern "C" int gk_set_tiling(gk_handle* h, int threads, int rows) {
    if (!h) return GK_ERR_INVALID;
    if (threads != 64 && threads != 128 && threads != 256)
        return fail(h, GK_ERR_INVALID, "threads per CTA must be 64, 128 or 256");
    if (rows < 1) return fail(h, GK_ERR_INVALID, "rows per segment must be positive");
    h->ctx.stage_threads = threads;
    h->ctx.h2d_rows = rows;
    h->ctx.learn_rows = 0;  // forced rows serve both stages
    h->tiling_set = true;
    h->tiling_rows = rows;
    if (h->gexec) {  // the graph holds the old launch shapes
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
    }
    return GK_OK;
}

// ------------------------------------------------------------ ensembles
// A batch of independent 2D problems advanced together: every stage of every
// instance is one persistent launch over a tile table (k_ens_stage), every
// ghost fill one launch over all instances, and a CUDA graph holds whole
// steps.  Each instance keeps its own handle, buffers and clock, so its dt
// and t follow its own CFL condition exactly as if it ran alone.
struct gk_ensemble {
    std::vector<gk_handle*> h;
    int n = 0, threads = 128, plm = 1, device = 0;
    const KernelSet* ks = nullptr;
    cudaStream_t stream = nullptr;
    gk::EnsInst* dinst = nullptr;
    int2* dtiles = nullptr;
    unsigned* dcount = nullptr;  // work counters of the two stages
    int* dany = nullptr;
    int ntiles = 0, max_bc = 0;
    std::vector<int> rows;
    cudaGraphExec_t gexec = nullptr;
    int graph_steps = 8;
    std::string err;
};

namespace {

int efail(gk_ensemble* e, int code, const std::string& msg) {
    if (e) e->err = msg;
    return code;
}

#define GK_ECUDA(e, call)                                                                       \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return efail((e), GK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Whether any instance of an ensemble is still inside its Sim::Advance loop
// (sim.cpp:72): the host's loop condition for the whole ensemble.
__global__ void k_ens_any_active(const gk::EnsInst* __restrict__ inst, int n, int* any) {
    int a = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a |= inst[i].tm->active;
    a = __syncthreads_or(a);
    if (threadIdx.x == 0) *any = a;
}

int ens_build(gk_ensemble* e) {
    std::vector<gk::EnsInst> inst(e->n);
    std::vector<int2> tiles;
    e->max_bc = 0;
    for (int i = 0; i < e->n; ++i) {
        const gk::Ctx& c = e->h[i]->ctx;
        const gk::Geom& g = c.g;
        gk::EnsInst& I = inst[i];
        std::memset(&I, 0, sizeof(I));
        if (!gk::encode_rows_map(&I.mapA, e->h[i]->A, g, e->threads) ||
            !gk::encode_rows_map(&I.mapB, e->h[i]->B, g, e->threads))
            return efail(e, GK_ERR_CUDA, "tensor map encoding failed");
        I.A = e->h[i]->A;
        I.B = e->h[i]->B;
        I.tm = e->h[i]->tm;
        I.rows = std::max(1, e->rows[i]);
        I.tiles_x = (g.nx + e->threads - 5) / (e->threads - 4);
        I.tiles = I.tiles_x * ((g.ny + I.rows - 1) / I.rows);
        I.g = g;
        I.ph = c.ph;
        I.ph.periodic_images = 0;  // the ensemble fills every instance's ghosts
        for (int t = 0; t < I.tiles; ++t) tiles.push_back(make_int2(i, t));
        e->max_bc = std::max(e->max_bc, g.ng * std::max(g.nx, g.ny));
    }
    cudaFree(e->dinst);
    cudaFree(e->dtiles);
    e->dinst = nullptr;
    e->dtiles = nullptr;
    e->ntiles = (int)tiles.size();
    GK_ECUDA(e, cudaMalloc(&e->dinst, sizeof(gk::EnsInst) * e->n));
    GK_ECUDA(e, cudaMalloc(&e->dtiles, sizeof(int2) * tiles.size()));
    GK_ECUDA(e, cudaMemcpy(e->dinst, inst.data(), sizeof(gk::EnsInst) * e->n,
                           cudaMemcpyHostToDevice));
    GK_ECUDA(e, cudaMemcpy(e->dtiles, tiles.data(), sizeof(int2) * tiles.size(),
                           cudaMemcpyHostToDevice));
    if (e->gexec) {
        cudaGraphExecDestroy(e->gexec);
        e->gexec = nullptr;
    }
    return GK_OK;
}

// One RK2 step of every instance (rk2.cpp:11-23 per instance).
void ens_enqueue_step(gk_ensemble* e) {
    const KernelSet& k = *e->ks;
    cudaStream_t s = e->stream;
    cudaMemsetAsync(e->dcount, 0, 2 * sizeof(unsigned), s);
    k.ens_bc(e->dinst, e->n, 0, e->max_bc, s);
    k.ens_stage(e->threads, 0, e->plm, e->dinst, e->dtiles, e->ntiles, e->dcount, 1.0, 1.0, 0.0, s);
    k.ens_bc(e->dinst, e->n, 1, e->max_bc, s);
    k.ens_stage(e->threads, 2, e->plm, e->dinst, e->dtiles, e->ntiles, e->dcount + 1, 0.5, 0.5,
                0.5, s);
}

int ens_graph(gk_ensemble* e) {
    if (e->gexec) return GK_OK;
    cudaGraph_t graph;
    GK_ECUDA(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < e->graph_steps; ++i) ens_enqueue_step(e);
    GK_ECUDA(e, cudaStreamEndCapture(e->stream, &graph));
    cudaError_t err = cudaGraphInstantiate(&e->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess)
        return efail(e, GK_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(err));
    return GK_OK;
}

int ens_run(gk_ensemble* e, double dtoutput, int nsteps, bool wait) {
    for (gk_handle* h : e->h) h->ghosts_dirty = true;  // the instances' ghosts follow the ensemble's fills
    GK_ECUDA(e, cudaSetDevice(e->device));
    for (gk_handle* h : e->h) GK_ECUDA(e, cudaStreamSynchronize(h->stream));
    int rc = ens_graph(e);
    if (rc != GK_OK) return rc;
    e->ks->ens_begin(e->dinst, e->n, dtoutput, nsteps, e->stream);
    GK_ECUDA(e, cudaGetLastError());
    if (nsteps > 0) {
        const int launches = (nsteps + e->graph_steps - 1) / e->graph_steps;
        for (int i = 0; i < launches; ++i) GK_ECUDA(e, cudaGraphLaunch(e->gexec, e->stream));
        if (wait) GK_ECUDA(e, cudaStreamSynchronize(e->stream));
        return GK_OK;
    }
    int batch = 1, any = 1;
    while (any) {
        for (int i = 0; i < batch; ++i) GK_ECUDA(e, cudaGraphLaunch(e->gexec, e->stream));
        k_ens_any_active<<<1, 128, 0, e->stream>>>(e->dinst, e->n, e->dany);
        GK_ECUDA(e, cudaMemcpyAsync(&any, e->dany, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
        GK_ECUDA(e, cudaStreamSynchronize(e->stream));
        batch = std::min(batch * 2, 64);
    }
    return GK_OK;
}

}  // namespace

extern "C" {

int gk_ens_create(gk_handle* const* handles, int n, gk_ensemble** out) {
    if (!handles || n <= 0 || !out) return GK_ERR_INVALID;
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        gk_handle* h = handles[i];
        if (!h || !h->uploaded) return GK_ERR_STATE;
        if (h->path != 1 || h->ctx.ph.integrator != 2 || h->ctx.ph.fix_inner ||
            !h->host_fills.empty() || h->model)
            return GK_ERR_UNSUPPORTED;
        // an instance's physics is copied here: fixed data must already be set
        for (int s = 0; s < 6; ++s)
            if (h->ctx.ph.bc[s] == 4 && !h->ctx.ph.fixed_bd) return GK_ERR_STATE;
        if (h->ks != handles[0]->ks || h->device != handles[0]->device ||
            h->ctx.ph.plm != handles[0]->ctx.ph.plm)
            return GK_ERR_INVALID;
    }
    gk_ensemble* e = new gk_ensemble();
    e->h.assign(handles, handles + n);
    e->n = n;
    e->ks = handles[0]->ks;
    e->plm = handles[0]->ctx.ph.plm;
    e->device = handles[0]->device;
    e->rows.assign(n, 16);
    cudaError_t ce = cudaSetDevice(e->device);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaMalloc(&e->dcount, 2 * sizeof(unsigned));
    if (ce == cudaSuccess) ce = cudaMalloc(&e->dany, sizeof(int));
    int rc = ce == cudaSuccess ? ens_build(e) : GK_ERR_CUDA;
    if (rc != GK_OK) {
        std::fprintf(stderr, "gk_ens_create: %s\n",
                     ce != cudaSuccess ? cudaGetErrorString(ce) : e->err.c_str());
        gk_ens_destroy(e);
        return rc;
    }
    *out = e;
    return GK_OK;
}

void gk_ens_destroy(gk_ensemble* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    cudaFree(e->dinst);
    cudaFree(e->dtiles);
    cudaFree(e->dcount);
    cudaFree(e->dany);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int gk_ens_set_tiling(gk_ensemble* e, int threads, const int* rows) {
    if (!e) return GK_ERR_INVALID;
    if (threads != 64 && threads != 128 && threads != 256)
        return efail(e, GK_ERR_INVALID, "threads per CTA must be 64, 128 or 256");
    e->threads = threads;
    if (rows)
        for (int i = 0; i < e->n; ++i) e->rows[i] = std::max(1, rows[i]);
    cudaSetDevice(e->device);
    return ens_build(e);
}

int gk_ens_advance(gk_ensemble* e, double dtoutput) {
    Range range("gk_ens_advance");
    if (!e) return GK_ERR_INVALID;
    return ens_run(e, dtoutput, 0, true);
}

int gk_ens_run_steps(gk_ensemble* e, int nsteps) {
    Range range("gk_ens_run_steps");
    if (!e) return GK_ERR_INVALID;
    if (nsteps <= 0) return GK_OK;
    return ens_run(e, 0.0, nsteps, true);
}

int gk_ens_enqueue_steps(gk_ensemble* e, int nsteps) {
    Range range("gk_ens_enqueue_steps");
    if (!e) return GK_ERR_INVALID;
    if (nsteps <= 0) return GK_OK;
    return ens_run(e, 0.0, nsteps, false);
}

int gk_ens_info(gk_ensemble* e, int* ntiles, int* threads, void** stream) {
    if (!e) return GK_ERR_INVALID;
    if (ntiles) *ntiles = e->ntiles;
    if (threads) *threads = e->threads;
    if (stream) *stream = (void*)e->stream;
    return GK_OK;
}

const char* gk_ens_last_error(const gk_ensemble* e) { return e ? e->err.c_str() : ""; }

}  // extern "C"

// ------------------------------------------------------------ flux taps
// Device side of the learned flux correction's data: face fluxes of the
// current state, and restricted fine-grid fluxes over fixed sub-steps.
namespace {

// The clock of a fixed-dt tap: dt set and the run active, so the per-phase
// kernels run (the reference's dt comes from sim.cpp:79-81 instead).
__global__ void k_arm_clock(gk::DevTime* tm, double dt) {
    tm->dt = dt;
    tm->active = 1;
}

// t += dt and step++ for each of n steps (sim.cpp:92-93), then inactive.
__global__ void k_clock_advance(gk::DevTime* tm, double dt, int n) {
    for (int i = 0; i < n; ++i) tm->t += dt;
    tm->step += n;
    tm->active = 0;
}

// acc[v][jc][ic] += w * sum of the `ratio` fine faces making up the left
// (x) or lower (y) face of coarse cell (jc, ic).
__global__ void k_restrict_faces(const double* __restrict__ F, double* __restrict__ acc,
                                 gk::Geom g, int ratio, int nxc, int nyc, int dir, double w) {
    const int ic = blockIdx.x * blockDim.x + threadIdx.x;
    const int jc = blockIdx.y;
    const int v = blockIdx.z;
    if (ic >= nxc) return;
    double s = 0.0;
    for (int k = 0; k < ratio; ++k) {
        const int i = dir == 0 ? g.ib + ratio * ic : g.ib + ratio * ic + k;
        const int j = dir == 0 ? g.jb + ratio * jc + k : g.jb + ratio * jc;
        s += F[v * g.fvstride + (long long)j * g.fpitch + i];
    }
    acc[((long long)v * nyc + jc) * nxc + ic] += w * s;
}

// Face flux arrays keep DEN, MTX, MTY, ENG in slots 0..3 (gk::Slot).
int copy_faces(gk_handle* h, const double* F, int dir, double* out) {
    const gk::Geom& g = h->ctx.g;
    const int nfx = dir == 0 ? g.nx + 1 : g.nx, nfy = dir == 0 ? g.ny : g.ny + 1;
    for (int v = 0; v < 4; ++v) {
        const double* src = F + v * g.fvstride + (long long)g.jb * g.fpitch + g.ib;
        GK_CUDA(h, cudaMemcpy2DAsync(out + (size_t)v * nfx * nfy, sizeof(double) * nfx, src,
                                     sizeof(double) * g.fpitch, sizeof(double) * nfx, nfy,
                                     cudaMemcpyDeviceToHost, h->stream));
    }
    return GK_OK;
}

}  // namespace

extern "C" int gk_face_fluxes(gk_handle* h, double* fx, double* fy) {
    int rc = check_ready(h);
    if (rc != GK_OK) return rc;
    if (h->ctx.g.ndim != 2) return fail(h, GK_ERR_UNSUPPORTED, "face fluxes are provided for 2D runs");
    rc = alloc_generic(h);
    if (rc != GK_OK) return rc;
    const KernelSet& k = *h->ks;
    k_arm_clock<<<1, 1, 0, h->stream>>>(h->tm, 0.0);
    k.bc(h->ctx, h->A, h->stream);
    k.c2p(h->ctx, h->A, h->W, h->stream);
    k.flux(h->ctx, 0, h->W, h->F1, h->stream);
    k.flux(h->ctx, 1, h->W, h->F2, h->stream);
    if (h->model) {  // dt is 0 here, so only the shock detector can veto a face
        gk::launch_flux_correct(h->model, h->W, h->F1, h->ctx.g, h->ctx.ph, h->ctx.tm, 0, h->gate,
                                nullptr, h->stream);
        gk::launch_flux_correct(h->model, h->W, h->F2, h->ctx.g, h->ctx.ph, h->ctx.tm, 1, h->gate,
                                nullptr, h->stream);
    }
    GK_CUDA(h, cudaGetLastError());
    if (fx && (rc = copy_faces(h, h->F1, 0, fx)) != GK_OK) return rc;
    if (fy && (rc = copy_faces(h, h->F2, 1, fy)) != GK_OK) return rc;
    k_clock_advance<<<1, 1, 0, h->stream>>>(h->tm, 0.0, 0);
    GK_CUDA(h, cudaStreamSynchronize(h->stream));
    return GK_OK;
}

extern "C" int gk_tap_substeps(gk_handle* h, int nsub, double dt_sub, int ratio, double* fx_acc,
                               double* fy_acc) {
    int rc = check_ready(h);
    if (rc != GK_OK) return rc;
    const gk::Geom& g = h->ctx.g;
    if (g.ndim != 2 || h->ctx.ph.integrator != 2 || h->ctx.ph.has_grav)
        return fail(h, GK_ERR_UNSUPPORTED, "flux taps need a 2D RK2 run without sources");
    if (ratio < 1 || nsub < 1 || g.nx % ratio || g.ny % ratio || !(dt_sub > 0))
        return fail(h, GK_ERR_INVALID, "ratio must divide the grid; nsub, dt_sub positive");
    rc = alloc_generic(h);
    if (rc != GK_OK) return rc;
    h->ghosts_dirty = true;  // the taps advance A on the generic path
    const int nxc = g.nx / ratio, nyc = g.ny / ratio;
    const size_t nacc = (size_t)4 * nxc * nyc;
    double* acc = nullptr;
    GK_CUDA(h, cudaMallocAsync(&acc, 2 * nacc * sizeof(double), h->stream));
    GK_CUDA(h, cudaMemsetAsync(acc, 0, 2 * nacc * sizeof(double), h->stream));
    const KernelSet& k = *h->ks;
    const gk::Ctx& c = h->ctx;
    cudaStream_t s = h->stream;
    // RK2 stage weight 1/2, time average 1/nsub, face average 1/ratio
    const double w = 0.5 / nsub / ratio;
    const dim3 grid((nxc + 127) / 128, nyc, 4);
    k_arm_clock<<<1, 1, 0, s>>>(h->tm, dt_sub);
    for (int n = 0; n < nsub; ++n) {
        for (int stage = 0; stage < 2; ++stage) {
            double* u = stage == 0 ? h->A : h->B;
            k.bc(c, u, s);
            k.c2p(c, u, h->W, s);
            k.flux(c, 0, h->W, h->F1, s);
            k.flux(c, 1, h->W, h->F2, s);
            if (h->model) {  // an installed correction is part of the tapped flux
                gk::launch_flux_correct(h->model, h->W, h->F1, c.g, c.ph, c.tm, 0, h->gate, h->fired, s);
                gk::launch_flux_correct(h->model, h->W, h->F2, c.g, c.ph, c.tm, 1, h->gate, h->fired, s);
            }
            k_restrict_faces<<<grid, 128, 0, s>>>(h->F1, acc, g, ratio, nxc, nyc, 0, w);
            k_restrict_faces<<<grid, 128, 0, s>>>(h->F2, acc + nacc, g, ratio, nxc, nyc, 1, w);
            if (stage == 0)
                k.update(c, nullptr, h->A, h->B, h->F1, h->F2, h->F3, 0, 1.0, 1.0, 0.0, s);
            else
                k.update(c, h->A, h->B, h->A, h->F1, h->F2, h->F3, 1, 0.5, 0.5, 0.5, s);
        }
    }
    k_clock_advance<<<1, 1, 0, s>>>(h->tm, dt_sub, nsub);
    k.cfl(c, h->A, 0, s);  // cmax of the new state for the next step's dt
    GK_CUDA(h, cudaGetLastError());
    if (fx_acc) GK_CUDA(h, cudaMemcpyAsync(fx_acc, acc, nacc * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (fy_acc)
        GK_CUDA(h, cudaMemcpyAsync(fy_acc, acc + nacc, nacc * sizeof(double), cudaMemcpyDeviceToHost, s));
    GK_CUDA(h, cudaFreeAsync(acc, s));
    GK_CUDA(h, cudaStreamSynchronize(s));
    return pull_time(h);
}

// ------------------------------------------------------------ fixed boundaries, point masses
extern "C" int gk_set_fixed_boundary(gk_handle* h, const double* snapshot, int fix_inner) {
    if (!h) return GK_ERR_INVALID;
    GK_CUDA(h, cudaSetDevice(h->device));
    gk::Phys& ph = h->ctx.ph;
    const gk::Geom& g = h->ctx.g;
    if (!snapshot) {
        ph.fixed_bd = nullptr;
        ph.fix_inner = 0;
        return physics_changed(h);
    }
    if (!h->fixed) {
        const size_t bytes = sizeof(double) * 5 * (size_t)g.vstride;
        GK_CUDA(h, cudaMalloc(&h->fixed, bytes));
        GK_CUDA(h, cudaMemsetAsync(h->fixed, 0, bytes, h->stream));
    }
    int rc = copy_ref_to_device(h, snapshot, h->fixed);
    if (rc != GK_OK) return rc;
    GK_CUDA(h, cudaStreamSynchronize(h->stream));
    ph.fixed_bd = h->fixed;
    ph.fix_inner = fix_inner ? 1 : 0;
    // the index box of Boundary::FixedBDInner (fixed.cpp:182-185)
    ph.inner[0] = static_cast<int>(g.ib + 0.25 * (g.ie - g.ib));
    ph.inner[1] = static_cast<int>(g.ib + 0.75 * (g.ie - g.ib));
    ph.inner[2] = static_cast<int>(g.jb + 0.25 * (g.je - g.jb));
    ph.inner[3] = static_cast<int>(g.jb + 0.75 * (g.je - g.jb));
    return physics_changed(h);
}

extern "C" int gk_set_host_fill(gk_handle* h, int side, int depth, gk_host_fill_fn fn, void* user,
                                double* cons) {
    if (!h || side < 0 || side > 5) return GK_ERR_INVALID;
    gk::Phys& ph = h->ctx.ph;
    const int n3[3] = {h->ctx.g.nx, h->ctx.g.ny, h->ctx.g.nz};
    auto& v = h->host_fills;
    for (size_t i = 0; i < v.size(); ++i)
        if (v[i].side == side) {
            v.erase(v.begin() + i);
            break;
        }
    if (!fn) {
        // back to the side's own ghost fill
        gk_handle fresh;
        fresh.gd = h->gd;
        fresh.pd = h->pd;
        if (build_ctx(&fresh) == GK_OK) ph.bc[side] = fresh.ctx.ph.bc[side];
        return physics_changed(h);
    }
    if (!cons || depth < 1) return fail(h, GK_ERR_INVALID, "a host fill needs its array and depth >= 1");
    if (n3[side / 2] <= 1) return fail(h, GK_ERR_INVALID, "that direction has one cell");
    v.push_back({side, depth, fn, user, cons});
    std::sort(v.begin(), v.end(), [](const gk_handle::HostFill& a, const gk_handle::HostFill& b) {
        return a.side < b.side;
    });
    ph.bc[side] = 5;  // the device ghost fill leaves the side alone
    return physics_changed(h);
}

extern "C" int gk_set_immersed(gk_handle* h, int n, const int* ids, const int* ntar,
                               const double* dir, const double* w) {
    if (!h || n < 0 || (n > 0 && (!ids || !ntar || !dir || !w))) return GK_ERR_INVALID;
    GK_CUDA(h, cudaSetDevice(h->device));
    gk::Phys& ph = h->ctx.ph;
    const gk::Geom& g = h->ctx.g;
    if (n > 0 && (g.nx <= 1 || g.ny <= 1))
        return fail(h, GK_ERR_INVALID, "an immersed body needs a 2D or 3D grid (immersed.cpp:90-92)");
    // The table in device layout.  Every cell must be active: the reference's
    // setup rejects bodies whose search reaches outside (immersed.cpp:201-205),
    // and the kernel relies on it for its indices.
    std::vector<gk::Shell> tab((size_t)n);
    auto id = [&](int c, int s, int t) { return ids[((size_t)c * n + s) * 9 + t]; };
    auto index = [&](int s, int t, long long* out) {
        const int i = id(0, s, t), j = id(1, s, t), k = id(2, s, t);
        if (i < g.ib || i >= g.ie || j < g.jb || j >= g.je || k < g.kb || k >= g.ke) return false;
        *out = (long long)(k - g.kofs) * g.kstride + (long long)j * g.pitch + i;
        return true;
    };
    for (int s = 0; s < n; ++s) {
        gk::Shell& sh = tab[s];
        std::memset(&sh, 0, sizeof(sh));
        sh.ntar = ntar[s];
        if (sh.ntar < 0 || sh.ntar > 8)
            return fail(h, GK_ERR_INVALID, "immersed shell: target count outside [0, 8]");
        if (!index(s, 0, &sh.cell)) return fail(h, GK_ERR_INVALID, "immersed shell cell not active");
        for (int t = 1; t <= sh.ntar; ++t)
            if (!index(s, t, &sh.tgt[t - 1]))
                return fail(h, GK_ERR_INVALID, "immersed shell target not active");
        for (int c = 0; c < 4; ++c) sh.dir[c] = dir[(size_t)c * n + s];
        for (int t = 0; t < 9; ++t) sh.w[t] = w[(size_t)s * 9 + t];
    }
    if (n > h->shell_cap) {
        GK_CUDA(h, cudaStreamSynchronize(h->stream));
        cudaFree(h->shells);
        h->shells = nullptr;
        h->shell_cap = 0;
        GK_CUDA(h, cudaMalloc(&h->shells, sizeof(gk::Shell) * (size_t)n));
        h->shell_cap = n;
    }
    if (n > 0) {
        GK_CUDA(h, cudaMemcpyAsync(h->shells, tab.data(), sizeof(gk::Shell) * (size_t)n,
                                   cudaMemcpyHostToDevice, h->stream));
        GK_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    ph.shells = n > 0 ? h->shells : nullptr;
    ph.nshell = n;
    return physics_changed(h);
}

extern "C" int gk_set_point_gravity(gk_handle* h, int n, const double* params) {
    if (!h || n < 0 || n > 2 || (n > 0 && !params)) return GK_ERR_INVALID;
    gk::Phys& ph = h->ctx.ph;
    ph.npoint = n;
    for (int i = 0; i < 11; ++i) ph.pm[i] = 0.0;
    for (int i = 0; i < (n == 2 ? 11 : (n == 1 ? 5 : 0)); ++i) ph.pm[i] = params[i];
    return physics_changed(h);
}

// ------------------------------------------------------------ learned correction on a handle
extern "C" int gk_set_flux_model(gk_handle* h, const float* model_host, int nmodel,
                                 float shock_jump, float pos_frac, float tv_min,
                                 float diss_frac) {
    if (!h) return GK_ERR_INVALID;
    GK_CUDA(h, cudaSetDevice(h->device));
    if (!model_host) {
        cudaFree(h->model);
        h->model = nullptr;
    } else {
        if (h->ctx.g.ndim != 2) return fail(h, GK_ERR_UNSUPPORTED, "the flux model is for 2D runs");
        if (nmodel != gk_mlp_nmodel()) return fail(h, GK_ERR_INVALID, "model size mismatch");
        if (!h->model) GK_CUDA(h, cudaMalloc(&h->model, sizeof(float) * nmodel));
        if (!h->fired) {
            GK_CUDA(h, cudaMalloc(&h->fired, sizeof(unsigned)));
            GK_CUDA(h, cudaMemset(h->fired, 0, sizeof(unsigned)));
        }
        GK_CUDA(h, cudaMemcpy(h->model, model_host, sizeof(float) * nmodel, cudaMemcpyHostToDevice));
        h->gate.shock_jump = shock_jump;
        h->gate.pos_frac = pos_frac;
        h->gate.tv_min = tv_min;
        h->gate.diss_frac = diss_frac;
        int rc = alloc_generic(h);
        if (rc != GK_OK) return rc;
    }
    // the path and the graph follow the model
    if (h->uploaded) {
        set_path(h);
        if (h->path != 1) {
            int rc = alloc_generic(h);
            if (rc != GK_OK) return rc;
        }
    }
    if (h->gexec) {
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
    }
    return GK_OK;
}

extern "C" int gk_set_flux_model_fused(gk_handle* h, int fused) {
    if (!h || (fused != 0 && fused != 1)) return GK_ERR_INVALID;
    GK_CUDA(h, cudaSetDevice(h->device));
    h->learn_fused = fused;
    if (h->uploaded) {
        set_path(h);
        if (h->path != 1) {
            int rc = alloc_generic(h);
            if (rc != GK_OK) return rc;
        }
    }
    if (h->gexec) {
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
    }
    return GK_OK;
}

extern "C" int gk_flux_model_fired(gk_handle* h, unsigned* fired) {
    if (!h || !fired) return GK_ERR_INVALID;
    *fired = 0;
    if (!h->fired) return GK_OK;
    GK_CUDA(h, cudaMemcpy(fired, h->fired, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return GK_OK;
}

// ------------------------------------------------------------ y-slabs
// One 2D grid split into y-slabs (a scale-out form of Sim::Advance for a grid
// larger than one GPU's share).  Each slab is a fused-2D handle over rows
// [j0, j0 + ny) of the global grid, with the global dx, dy and drmin.  Per RK
// stage, after the ghost fill of the x sides and of any physical y side, the
// two ghost rows on either side of a slab come from its neighbours' active
// rows; with periodic y the slabs form a ring.  The last stage defers the
// step epilogue: the CFL maximum is taken over all slabs first, so every slab
// takes the dt of the whole grid (sim.cpp:77-81) and the results are the
// undivided grid's bit for bit.  Slabs in one process share one device and
// one stream and exchange through a copy kernel; one slab per process
// exchanges through NCCL (send/recv of the packed rows, all-reduce(max) of
// the CFL speed and the status word), loaded at run time so the library does
// not depend on NCCL otherwise.
#include <dlfcn.h>
#include <nccl.h>

namespace {

struct NcclApi {
    ncclResult_t (*GetUniqueId)(ncclUniqueId*);
    ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int);
    ncclResult_t (*CommDestroy)(ncclComm_t);
    ncclResult_t (*GroupStart)();
    ncclResult_t (*GroupEnd)();
    ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t);
    const char* (*GetErrorString)(ncclResult_t);
};

// NCCL, resolved once from the process's libnccl.so.2 (the one a framework in
// the same process already loaded, else the system's).
const NcclApi* nccl_api(std::string* err) {
    static NcclApi api{};
    static bool tried = false, ok = false;
    static std::string why;
    if (!tried) {
        tried = true;
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            why = std::string("cannot load libnccl.so.2: ") + dlerror();
        } else {
            auto sym = [&](const char* name) { return dlsym(h, name); };
            api.GetUniqueId = (decltype(api.GetUniqueId))sym("ncclGetUniqueId");
            api.CommInitRank = (decltype(api.CommInitRank))sym("ncclCommInitRank");
            api.CommDestroy = (decltype(api.CommDestroy))sym("ncclCommDestroy");
            api.GroupStart = (decltype(api.GroupStart))sym("ncclGroupStart");
            api.GroupEnd = (decltype(api.GroupEnd))sym("ncclGroupEnd");
            api.Send = (decltype(api.Send))sym("ncclSend");
            api.Recv = (decltype(api.Recv))sym("ncclRecv");
            api.AllReduce = (decltype(api.AllReduce))sym("ncclAllReduce");
            api.GetErrorString = (decltype(api.GetErrorString))sym("ncclGetErrorString");
            ok = api.GetUniqueId && api.CommInitRank && api.CommDestroy && api.GroupStart &&
                 api.GroupEnd && api.Send && api.Recv && api.AllReduce && api.GetErrorString;
            if (!ok) why = "libnccl.so.2 lacks a needed symbol";
        }
    }
    if (!ok && err) *err = why;
    return ok ? &api : nullptr;
}

// Rows of slab k of n over ny active rows: the first ny % n slabs take one
// row more.
void slab_rows(int ny, int n, int k, int* j0, int* cnt) {
    const int base = ny / n, rem = ny % n;
    *cnt = base + (k < rem ? 1 : 0);
    *j0 = k * base + (k < rem ? k : rem);
}

// The NCCL calls of one halo exchange of slab k of n, in order: rows going
// up first (send the top rows to the upper neighbour, receive the lower
// ghosts from the lower one), then rows going down.  Between any two ranks
// the k-th send then matches the k-th receive, a single ring slab
// exchanging with itself included.  Each op: {kind, peer}, kind 0 send top
// rows, 1 receive lower ghosts, 2 send bottom rows, 3 receive upper ghosts.
int slab_exchange_plan(int n, int k, bool periodic, int (*ops)[2]) {
    int m = 0;
    const int lower = k > 0 ? k - 1 : (periodic ? n - 1 : -1);
    const int upper = k < n - 1 ? k + 1 : (periodic ? 0 : -1);
    if (upper >= 0) { ops[m][0] = 0; ops[m][1] = upper; ++m; }
    if (lower >= 0) { ops[m][0] = 1; ops[m][1] = lower; ++m; }
    if (lower >= 0) { ops[m][0] = 2; ops[m][1] = lower; ++m; }
    if (upper >= 0) { ops[m][0] = 3; ops[m][1] = upper; ++m; }
    return m;
}

// Neighbours of slab k of n: -1 where the y side is the grid's own boundary
// (filled by the ghost fill); with periodic y the first and last slabs are
// each other's neighbours (a single slab is its own).
void slab_neighbors(int n, int k, bool periodic, int* lower, int* upper) {
    *lower = k > 0 ? k - 1 : (periodic ? n - 1 : -1);
    *upper = k < n - 1 ? k + 1 : (periodic ? 0 : -1);
}

}  // namespace

struct gk_slabs {
    gk_grid_desc gd{};        // the whole grid
    gk_phys_desc pd{};
    int nslab = 1;            // slabs of the whole grid
    int first = 0;            // index of this process's first slab
    std::vector<gk_handle*> s;  // this process's slabs
    std::vector<int> j0, ny;  // their first active row (global, 0-based) and row count
    cudaStream_t stream = nullptr;  // the first slab's: every launch of the group
    gk::SlabDev* dsd = nullptr;     // device table of the local slabs
    const NcclApi* nccl = nullptr;
    ncclComm_t comm = nullptr;
    int lower = -1, upper = -1;     // NCCL: neighbour ranks
    double* xbuf = nullptr;         // NCCL: send lo, send hi, recv lo, recv hi
    unsigned long long* red = nullptr;
    std::string err;
};

namespace {

int sfail(gk_slabs* G, int code, const std::string& msg) {
    if (G) G->err = msg;
    return code;
}

#define GK_SCUDA(G, call)                                                                       \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return sfail((G), GK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define GK_SNCCL(G, call)                                                                      \
    do {                                                                                       \
        ncclResult_t r_ = (call);                                                              \
        if (r_ != ncclSuccess)                                                                 \
            return sfail((G), GK_ERR_CUDA, std::string(#call) + ": " + (G)->nccl->GetErrorString(r_)); \
    } while (0)

// Creates this process's slabs (global indices first .. first + count - 1).
int slabs_build(gk_slabs* G, int first, int count) {
    const gk_grid_desc& gd = G->gd;
    const gk_phys_desc& pd = G->pd;
    if (gd.nz != 1 || gd.ny < 2 || gd.nx < 2)
        return sfail(G, GK_ERR_UNSUPPORTED, "y-slabs split 2D grids");
    if (pd.integrator != 2 && pd.integrator != 3)
        return sfail(G, GK_ERR_UNSUPPORTED, "y-slabs run RK2 or RK3 (the fused 2D stage)");
    if (pd.grav[2] != 0)
        return sfail(G, GK_ERR_UNSUPPORTED, "y-slabs need gz = 0 (the fused 2D stage)");
    if (pd.bc[2] == 4 || pd.bc[3] == 4 || pd.bc[0] == 4 || pd.bc[1] == 4)
        return sfail(G, GK_ERR_UNSUPPORTED, "fixed (type 4) sides are not split");
    if (G->nslab < 1 || gd.ny / G->nslab < gd.nghost)
        return sfail(G, GK_ERR_INVALID, "every slab needs at least NGhost rows");
    // the whole grid's spacings (sim.cpp:16-36), which every slab keeps
    gk_handle whole;
    whole.gd = gd;
    whole.pd = pd;
    int rc = build_ctx(&whole);
    if (rc != GK_OK) return sfail(G, rc, whole.err);
    const bool periodic = whole.ctx.ph.bc[2] == 1;
    if (periodic != (whole.ctx.ph.bc[3] == 1))
        return sfail(G, GK_ERR_UNSUPPORTED, "a periodic y side needs a periodic partner");
    for (int k = first; k < first + count; ++k) {
        int j0, cnt, lo, up;
        slab_rows(gd.ny, G->nslab, k, &j0, &cnt);
        slab_neighbors(G->nslab, k, periodic, &lo, &up);
        gk_grid_desc sg = gd;
        sg.ny = cnt;
        gk_handle* h = nullptr;
        rc = gk_create(&sg, &pd, &h);
        if (rc != GK_OK) return sfail(G, rc, "slab creation failed");
        G->s.push_back(h);
        G->j0.push_back(j0);
        G->ny.push_back(cnt);
        gk::Geom& g = h->ctx.g;
        g.dy = whole.ctx.g.dy;
        g.dyRec = whole.ctx.g.dyRec;
        g.drmin = whole.ctx.g.drmin;
        g.ymin = whole.ctx.g.ymin + j0 * whole.ctx.g.dy;  // cell centres, not used by the fused stage
        // sides between slabs (all y sides under periodic y) come from the exchange
        if (lo >= 0) h->ctx.ph.bc[2] = 5;
        if (up >= 0) h->ctx.ph.bc[3] = 5;
        h->ctx.ph.defer_epilogue = 1;
    }
    G->stream = G->s[0]->stream;
    return GK_OK;
}

int slabs_device_table(gk_slabs* G) {
    const int n = (int)G->s.size();
    std::vector<gk::SlabDev> t(n);
    const bool periodic = G->pd.bc[2] == 1;
    for (int k = 0; k < n; ++k) {
        gk_handle* h = G->s[k];
        t[k].buf[0] = h->A;
        t[k].buf[1] = h->B;
        t[k].buf[2] = h->C;
        t[k].tm = h->tm;
        t[k].vstride = h->ctx.g.vstride;
        t[k].jb = h->ctx.g.jb;
        t[k].je = h->ctx.g.je;
        int lo, up;
        slab_neighbors(G->nslab, G->first + k, periodic, &lo, &up);
        // in-process exchange only: neighbours are local slabs
        t[k].lower = lo >= 0 ? lo - G->first : -1;
        t[k].upper = up >= 0 ? up - G->first : -1;
    }
    GK_SCUDA(G, cudaMalloc(&G->dsd, sizeof(gk::SlabDev) * n));
    GK_SCUDA(G, cudaMemcpy(G->dsd, t.data(), sizeof(gk::SlabDev) * n, cudaMemcpyHostToDevice));
    return GK_OK;
}

double* slab_buf(gk_handle* h, int role) { return role == 0 ? h->A : (role == 1 ? h->B : h->C); }

// The two ghost rows on each side of every local slab, in buffer `role`.
int slabs_halo(gk_slabs* G, int role) {
    if (!G->comm) {
        gk::launch_slab_halo(G->dsd, (int)G->s.size(), role, G->s[0]->ctx.g, G->stream);
        return GK_OK;
    }
    gk_handle* h = G->s[0];
    const gk::Geom& g = h->ctx.g;
    const size_t cnt = 10 * (size_t)g.nx;
    double *slo = G->xbuf, *shi = G->xbuf + cnt, *rlo = G->xbuf + 2 * cnt, *rhi = G->xbuf + 3 * cnt;
    double* u = slab_buf(h, role);
    gk::launch_slab_pack(u, slo, shi, g, h->ctx.tm, G->stream);
    int ops[4][2];
    const int nops = slab_exchange_plan(G->nslab, G->first, G->pd.bc[2] == 1, ops);
    double* const bufs[4] = {shi, rlo, slo, rhi};
    GK_SNCCL(G, G->nccl->GroupStart());
    for (int o = 0; o < nops; ++o) {
        double* b = bufs[ops[o][0]];
        if (ops[o][0] == 0 || ops[o][0] == 2)
            GK_SNCCL(G, G->nccl->Send(b, cnt, ncclDouble, ops[o][1], G->comm, G->stream));
        else
            GK_SNCCL(G, G->nccl->Recv(b, cnt, ncclDouble, ops[o][1], G->comm, G->stream));
    }
    GK_SNCCL(G, G->nccl->GroupEnd());
    gk::launch_slab_unpack(u, G->lower >= 0 ? rlo : nullptr, G->upper >= 0 ? rhi : nullptr, g,
                           h->ctx.tm, G->stream);
    return GK_OK;
}

// The CFL maximum (and status) over all slabs into every slab's clock.
int slabs_reduce(gk_slabs* G, int which) {
    if (!G->comm) {
        gk::launch_slab_reduce(G->dsd, (int)G->s.size(), which, G->stream);
        return GK_OK;
    }
    gk_handle* h = G->s[0];
    gk::launch_slab_red_pack(h->tm, G->red, which, G->stream);
    GK_SNCCL(G, G->nccl->AllReduce(G->red, G->red, 2, ncclUint64, ncclMax, G->comm, G->stream));
    gk::launch_slab_red_unpack(h->tm, G->red, which, G->stream);
    return GK_OK;
}

// One time step of the whole grid (Sim::RK2_/RK3_ with the Strang half kicks
// of sim.cpp:85-91), every phase over all local slabs before the next.
int slabs_enqueue_step(gk_slabs* G) {
    const KernelSet& k = *G->s[0]->ks;
    cudaStream_t st = G->stream;
    const bool rk3 = G->s[0]->ctx.ph.integrator == 3;
    const double frac13 = 1.0 / 3.0;
    int rc;
    for (gk_handle* h : G->s)
        if (h->ctx.ph.has_grav) k.kick(h->ctx, h->A, 0, st);
    for (gk_handle* h : G->s) k.bc(h->ctx, h->A, st);
    if ((rc = slabs_halo(G, 0)) != GK_OK) return rc;
    for (gk_handle* h : G->s) k.stage2d(h->ctx, h->A, nullptr, h->B, 0, 1.0, 1.0, 0.0, st);
    for (gk_handle* h : G->s) k.bc(h->ctx, h->B, st);
    if ((rc = slabs_halo(G, 1)) != GK_OK) return rc;
    if (rk3) {
        for (gk_handle* h : G->s) k.stage2d(h->ctx, h->B, h->A, h->C, 1, 0.75, 0.25, 0.25, st);
        for (gk_handle* h : G->s) k.bc(h->ctx, h->C, st);
        if ((rc = slabs_halo(G, 2)) != GK_OK) return rc;
        for (gk_handle* h : G->s)
            k.stage2d(h->ctx, h->C, h->A, h->A, 2, frac13, 2 * frac13, 2 * frac13, st);
    } else {
        for (gk_handle* h : G->s) k.stage2d(h->ctx, h->B, h->A, h->A, 2, 0.5, 0.5, 0.5, st);
    }
    if ((rc = slabs_reduce(G, 0)) != GK_OK) return rc;
    for (gk_handle* h : G->s) k.epilogue(h->ctx, st);
    return GK_OK;
}

int slabs_check_ready(gk_slabs* G) {
    if (!G) return GK_ERR_INVALID;
    for (gk_handle* h : G->s) {
        if (!h->uploaded) return sfail(G, GK_ERR_STATE, "no state uploaded");
        if (h->path != 1)
            return sfail(G, GK_ERR_UNSUPPORTED,
                         "y-slabs run the fused 2D stage (vz = 0, no point masses or immersed body)");
    }
    GK_SCUDA(G, cudaSetDevice(G->s[0]->device));
    return GK_OK;
}

// Sim::Advance over the whole grid (nsteps = 0) or a fixed step count.
int slabs_run(gk_slabs* G, double dtoutput, int nsteps) {
    int rc = slabs_reduce(G, 1);
    if (rc != GK_OK) return rc;
    const KernelSet& k = *G->s[0]->ks;
    for (gk_handle* h : G->s) k.begin(h->ctx, dtoutput, nsteps, G->stream);
    gk_handle* h0 = G->s[0];
    if (nsteps > 0) {
        for (int i = 0; i < nsteps; ++i)
            if ((rc = slabs_enqueue_step(G)) != GK_OK) return rc;
    } else {
        // every process sees the same clock (one dt for the whole grid), so
        // all of them enqueue the same batches and stop together
        int batch = 1;
        for (;;) {
            for (int i = 0; i < batch; ++i)
                if ((rc = slabs_enqueue_step(G)) != GK_OK) return rc;
            GK_SCUDA(G, cudaMemcpyAsync(&h0->htm->active, &h0->tm->active, sizeof(int),
                                        cudaMemcpyDeviceToHost, G->stream));
            GK_SCUDA(G, cudaStreamSynchronize(G->stream));
            if (!h0->htm->active) break;
            batch = std::min(batch * 2, 64);
        }
    }
    GK_SCUDA(G, cudaGetLastError());
    GK_SCUDA(G, cudaStreamSynchronize(G->stream));
    for (gk_handle* s : G->s)
        if ((rc = pull_time(s)) != GK_OK) return sfail(G, rc, s->err);
    if (h0->htm->status) {
        rc = status_error(h0);
        return sfail(G, rc, h0->err);
    }
    return GK_OK;
}

}  // namespace

extern "C" {

int gk_slab_layout(int ny, int nslab, int k, int periodic, int* j0, int* rows, int* lower,
                   int* upper) {
    if (nslab < 1 || k < 0 || k >= nslab || ny < nslab) return GK_ERR_INVALID;
    int a, b, c, d;
    slab_rows(ny, nslab, k, &a, &b);
    slab_neighbors(nslab, k, periodic != 0, &c, &d);
    if (j0) *j0 = a;
    if (rows) *rows = b;
    if (lower) *lower = c;
    if (upper) *upper = d;
    return GK_OK;
}

int gk_slab_exchange_plan(int nslab, int k, int periodic, int* ops8, int* nops) {
    if (nslab < 1 || k < 0 || k >= nslab || !ops8 || !nops) return GK_ERR_INVALID;
    int ops[4][2];
    *nops = slab_exchange_plan(nslab, k, periodic != 0, ops);
    for (int o = 0; o < *nops; ++o) {
        ops8[2 * o] = ops[o][0];
        ops8[2 * o + 1] = ops[o][1];
    }
    return GK_OK;
}

int gk_slabs_create(const gk_grid_desc* grid, const gk_phys_desc* phys, int nslab, gk_slabs** out) {
    if (!grid || !phys || !out || nslab < 1) return GK_ERR_INVALID;
    *out = nullptr;
    gk_slabs* G = new gk_slabs();
    G->gd = *grid;
    G->pd = *phys;
    G->nslab = nslab;
    G->first = 0;
    int rc = slabs_build(G, 0, nslab);
    if (rc == GK_OK) rc = slabs_device_table(G);
    if (rc != GK_OK) {
        std::fprintf(stderr, "gk_slabs_create: %s\n", G->err.c_str());
        gk_slabs_destroy(G);
        return rc;
    }
    *out = G;
    return GK_OK;
}

int gk_slabs_nccl_id(void* id128) {
    if (!id128) return GK_ERR_INVALID;
    std::string err;
    const NcclApi* api = nccl_api(&err);
    if (!api) {
        std::fprintf(stderr, "gk_slabs_nccl_id: %s\n", err.c_str());
        return GK_ERR_UNSUPPORTED;
    }
    ncclUniqueId id;
    if (api->GetUniqueId(&id) != ncclSuccess) return GK_ERR_CUDA;
    std::memcpy(id128, &id, sizeof(id));
    return GK_OK;
}

int gk_slabs_create_nccl(const gk_grid_desc* grid, const gk_phys_desc* phys, int nranks, int rank,
                         const void* id128, gk_slabs** out) {
    if (!grid || !phys || !out || !id128 || nranks < 1 || rank < 0 || rank >= nranks)
        return GK_ERR_INVALID;
    *out = nullptr;
    gk_slabs* G = new gk_slabs();
    G->gd = *grid;
    G->pd = *phys;
    G->nslab = nranks;
    G->first = rank;
    std::string err;
    G->nccl = nccl_api(&err);
    int rc = G->nccl ? GK_OK : sfail(G, GK_ERR_UNSUPPORTED, err);
    if (rc == GK_OK) rc = slabs_build(G, rank, 1);
    if (rc == GK_OK) {
        gk_handle* h = G->s[0];
        slab_neighbors(nranks, rank, G->pd.bc[2] == 1, &G->lower, &G->upper);
        const size_t cnt = 10 * (size_t)h->ctx.g.nx;
        cudaError_t e = cudaSetDevice(h->device);
        if (e == cudaSuccess) e = cudaMalloc(&G->xbuf, 4 * cnt * sizeof(double));
        if (e == cudaSuccess) e = cudaMemset(G->xbuf, 0, 4 * cnt * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&G->red, 2 * sizeof(unsigned long long));
        if (e != cudaSuccess) rc = sfail(G, GK_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc == GK_OK) {
        ncclUniqueId id;
        std::memcpy(&id, id128, sizeof(id));
        ncclComm_t comm = nullptr;
        const ncclResult_t r = G->nccl->CommInitRank(&comm, nranks, id, rank);
        if (r != ncclSuccess) rc = sfail(G, GK_ERR_CUDA, std::string("ncclCommInitRank: ") +
                                                           G->nccl->GetErrorString(r));
        else G->comm = comm;
    }
    if (rc != GK_OK) {
        std::fprintf(stderr, "gk_slabs_create_nccl: %s\n", G->err.c_str());
        gk_slabs_destroy(G);
        return rc;
    }
    *out = G;
    return GK_OK;
}

void gk_slabs_destroy(gk_slabs* G) {
    if (!G) return;
    if (!G->s.empty()) {
        cudaSetDevice(G->s[0]->device);
        if (G->stream) cudaStreamSynchronize(G->stream);
    }
    if (G->comm && G->nccl) G->nccl->CommDestroy(G->comm);
    cudaFree(G->dsd);
    cudaFree(G->xbuf);
    cudaFree(G->red);
    for (gk_handle* h : G->s) gk_destroy(h);
    delete G;
}

int gk_slabs_upload_cons(gk_slabs* G, const double* cons) {
    Range range("gk_slabs_upload_cons");
    if (!G || !cons) return GK_ERR_INVALID;
    const gk::Geom& g0 = G->s[0]->ctx.g;
    const size_t lenx = g0.lenx, lenz = g0.lenz, leny_all = (size_t)G->gd.ny + 2 * g0.ng;
    for (size_t k = 0; k < G->s.size(); ++k) {
        gk_handle* h = G->s[k];
        const size_t leny = h->ctx.g.leny;
        // the slab's rows j0 .. j0 + leny - 1 of the whole grid, ghosts included
        std::vector<double> part(5 * lenz * leny * lenx);
        for (size_t v = 0; v < 5 * lenz; ++v)
            std::memcpy(part.data() + v * leny * lenx,
                        cons + (v * leny_all + (size_t)G->j0[k]) * lenx,
                        sizeof(double) * leny * lenx);
        int rc = gk_upload_cons(h, part.data());
        if (rc != GK_OK) return sfail(G, rc, h->err);
    }
    return slabs_check_ready(G);
}

int gk_slabs_download_cons(gk_slabs* G, double* cons) {
    Range range("gk_slabs_download_cons");
    int rc = slabs_check_ready(G);
    if (rc != GK_OK) return rc;
    if (!cons) return GK_ERR_INVALID;
    GK_SCUDA(G, cudaStreamSynchronize(G->stream));
    const gk::Geom& g0 = G->s[0]->ctx.g;
    const size_t lenx = g0.lenx, lenz = g0.lenz, ng = g0.ng;
    const size_t leny_all = (size_t)G->gd.ny + 2 * ng;
    for (size_t k = 0; k < G->s.size(); ++k) {
        gk_handle* h = G->s[k];
        const size_t leny = h->ctx.g.leny;
        std::vector<double> part(5 * lenz * leny * lenx);
        rc = gk_download_cons(h, part.data());
        if (rc != GK_OK) return sfail(G, rc, h->err);
        // active rows; the ghost rows too where the slab ends the grid
        const int gk_ = G->first + (int)k;
        const size_t r0 = gk_ == 0 ? 0 : ng;
        const size_t r1 = gk_ == G->nslab - 1 ? leny : leny - ng;
        for (size_t v = 0; v < 5 * lenz; ++v)
            std::memcpy(cons + (v * leny_all + (size_t)G->j0[k] + r0) * lenx,
                        part.data() + (v * leny + r0) * lenx, sizeof(double) * (r1 - r0) * lenx);
    }
    return GK_OK;
}

int gk_slabs_run_steps(gk_slabs* G, int nsteps, int* done) {
    Range range("gk_slabs_run_steps");
    int rc = slabs_check_ready(G);
    if (rc != GK_OK) return rc;
    if (done) *done = 0;
    if (nsteps <= 0) return GK_OK;
    const int before = G->s[0]->htm->step;
    rc = slabs_run(G, 0.0, nsteps);
    if (done) *done = G->s[0]->htm->step - before;
    return rc;
}

int gk_slabs_advance(gk_slabs* G, double dtoutput, double* t, int* step, int* is_continue) {
    Range range("gk_slabs_advance");
    int rc = slabs_check_ready(G);
    if (rc != GK_OK) return rc;
    rc = slabs_run(G, dtoutput, 0);
    const gk::DevTime& c = *G->s[0]->htm;
    if (t) *t = c.t;
    if (step) *step = c.step;
    if (is_continue) *is_continue = c.is_continue;
    return rc;
}

int gk_slabs_dt_log(gk_slabs* G, double* buf, int cap, int* n) {
    if (!G || G->s.empty()) return GK_ERR_INVALID;
    GK_SCUDA(G, cudaStreamSynchronize(G->stream));
    return gk_dt_log(G->s[0], buf, cap, n);
}

int gk_slabs_info(gk_slabs* G, int* nslab_local, int* first, int* j0, int* rows) {
    if (!G || G->s.empty()) return GK_ERR_INVALID;
    if (nslab_local) *nslab_local = (int)G->s.size();
    if (first) *first = G->first;
    if (j0) *j0 = G->j0[0];
    if (rows) *rows = G->ny[0];
    return GK_OK;
}

const char* gk_slabs_last_error(const gk_slabs* G) { return G ? G->err.c_str() : ""; }

}  // extern "C"
