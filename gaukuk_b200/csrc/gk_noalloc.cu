// gk_noalloc.cu -- one RK2 time step on caller-owned device memory, with no
// device allocation by the library.
//
// Who needs it: callers that cannot call cudaMalloc while they run -- code
// that owns all device memory through its own pool or arena, real-time loops
// that must not allocate after start-up, and hosts whose memory budget is
// fixed when they load this library.  gk_create allocates the RK stage
// buffers and the device clock per handle; this entry point instead keeps
// them in one file-scope device array of fixed size, so the caller passes
// only the state.
//
// The scratch array (64 MiB) is part of every GPU context that loads the
// library and lives until the process exits.  In host code its name is a
// host-side stand-in, never a device address: the address used for kernel
// arguments comes from cudaGetSymbolAddress, taken once per device with that
// device current, on the first call made on the device.
//
// The stage state holds all five variable planes: the ghost fill writes the
// ghosts of every plane, MTZ included, so a grid is accepted only when
// 5 * vstride doubles fit (about 1290 x 1290 cells).
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>

#include "gaukuk_cuda.h"
#include "gk_internal.h"

int gk_internal_build_ctx(const gk_grid_desc* gd, const gk_phys_desc* pd, gk::Ctx* ctx,
                          std::string* err);

namespace {

constexpr long long kScratchDoubles = 1LL << 23;  // 64 MiB
constexpr int kMaxDevices = 64;

// Scratch: the intermediate RK stage state (5 variable planes in the device
// layout), then the device clock, the MTZ check flag and the ticket of the
// call whose clock reset ran last.
struct NoallocScratch {
    double stage[kScratchDoubles];
    gk::DevTime clock;
    int flag;
    unsigned long long ticket;
};

static __device__ __align__(256) NoallocScratch gk_noalloc_scratch;

// Device address of the scratch array per device, looked up on the device's
// first call.  Atomic: host threads making their first calls on one device
// at the same time each look it up and store the same value.
std::atomic<NoallocScratch*> g_scratch_addr[kMaxDevices];

// Call tickets: the reset kernel stores its call's ticket, so a call that
// finds its own ticket and step 1 in the clock knows that its launches ran
// (without reading cudaGetLastError, which would also report errors left by
// unrelated work).
std::atomic<unsigned long long> g_ticket{0};

// Resets the clock for one step starting at time 0 with no output limit.
__global__ void k_noalloc_reset(gk::DevTime* tm, int* flag, unsigned long long* ticket_out,
                                unsigned long long ticket) {
    gk::DevTime t{};
    t.t = 0;
    t.dt = 1e10;
    t.tNext = 0;
    t.dtUntilOutput = 1e10;
    t.cmax_last = 1e-16;
    double seed = 1e-16;
    memcpy(&t.cmax_acc, &seed, sizeof(double));
    t.done_ctas = 0;
    t.step = 0;
    t.is_continue = 1;
    t.active = 1;
    t.status = 0;
    t.steps_left = -1;
    t.nlog = 0;
    t.log_cap = 0;
    t.log = nullptr;
    *tm = t;
    *flag = 0;
    *ticket_out = ticket;
}

}  // namespace

extern "C" int gk_rk2_step_noalloc(const gk_grid_desc* grid, const gk_phys_desc* phys,
                                   double* state, double dtmax, double* dt_used, void* stream) {
    if (!grid || !phys || !state) return GK_ERR_INVALID;
    gk::Ctx c{};
    std::string err;
    int rc = gk_internal_build_ctx(grid, phys, &c, &err);
    if (rc != GK_OK) {
        std::fprintf(stderr, "gk_rk2_step_noalloc: %s\n", err.c_str());
        return rc;
    }
    if (c.g.ndim != 2 || c.ph.integrator != 2 || c.ph.grav[2] != 0) {
        std::fprintf(stderr, "gk_rk2_step_noalloc: needs a 2D run with integrator 2 and gz = 0\n");
        return GK_ERR_UNSUPPORTED;
    }
    for (int side = 0; side < 6; ++side) {
        if (c.ph.bc[side] == 4) {
            // fixed sides fill their ghosts from the state at enrollment,
            // which only a handle holds (gk_set_fixed_boundary)
            std::fprintf(stderr, "gk_rk2_step_noalloc: fixed (type 4) sides need a handle\n");
            return GK_ERR_UNSUPPORTED;
        }
    }
    if (5 * c.g.vstride > kScratchDoubles) {
        std::fprintf(stderr,
                     "gk_rk2_step_noalloc: grid too large: the stage state needs %lld doubles, "
                     "the fixed scratch holds %lld (about 1290 x 1290 cells)\n",
                     5 * c.g.vstride, kScratchDoubles);
        return GK_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GK_ERR_CUDA;
    if (!g_scratch_addr[dev].load(std::memory_order_acquire)) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, gk_noalloc_scratch);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "gk_rk2_step_noalloc: cudaGetSymbolAddress: %s\n",
                         cudaGetErrorString(e));
            return GK_ERR_CUDA;
        }
        g_scratch_addr[dev].store(static_cast<NoallocScratch*>(p), std::memory_order_release);
    }
    NoallocScratch* sc = g_scratch_addr[dev].load(std::memory_order_acquire);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    c.tm = &sc->clock;
    double* stage = sc->stage;

    const unsigned long long ticket = ++g_ticket;
    k_noalloc_reset<<<1, 1, 0, s>>>(&sc->clock, &sc->flag, &sc->ticket, ticket);
    const bool fast = phys->mode == GK_MODE_FAST;
    auto mtz = fast ? gk_fast::launch_mtz_check : gk_parity::launch_mtz_check;
    auto cfl = fast ? gk_fast::launch_cfl : gk_parity::launch_cfl;
    auto begin = fast ? gk_fast::launch_begin : gk_parity::launch_begin;
    auto bc = fast ? gk_fast::launch_bc : gk_parity::launch_bc;
    auto stage2d = fast ? gk_fast::launch_stage2d : gk_parity::launch_stage2d;
    auto kick = fast ? gk_fast::launch_kick : gk_parity::launch_kick;
    mtz(c, state, &sc->flag, s);
    int flag = 0;
    if (cudaMemcpyAsync(&flag, &sc->flag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GK_ERR_CUDA;
    if (flag) {
        std::fprintf(stderr, "gk_rk2_step_noalloc: MTZ is not zero; the fused 2D step needs vz = 0\n");
        return GK_ERR_UNSUPPORTED;
    }
    // Sim::Advance for one step with dtUntilOutput = dtmax (sim.cpp:77-81):
    // cmax of the state, dt, the first gravity half kick (sim.cpp:85-86),
    // then the two RK2 stages; the last stage applies the second half kick
    // and its epilogue advances the clock.
    cfl(c, state, 0, s);
    begin(c, dtmax, 0, s);
    if (c.ph.has_grav) kick(c, state, 0, s);
    bc(c, state, s);
    stage2d(c, state, nullptr, stage, 0, 1.0, 1.0, 0.0, s);
    bc(c, stage, s);
    stage2d(c, stage, state, state, 2, 0.5, 0.5, 0.5, s);
    gk::DevTime t{};
    unsigned long long ran = 0;
    if (cudaMemcpyAsync(&t, &sc->clock, sizeof(t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&ran, &sc->ticket, sizeof(ran), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GK_ERR_CUDA;
    if (ran != ticket) {
        std::fprintf(stderr, "gk_rk2_step_noalloc: a kernel of this call did not launch\n");
        return GK_ERR_CUDA;
    }
    if (t.status & gk::STATUS_TMA_TIMEOUT) {
        std::fprintf(stderr, "gk_rk2_step_noalloc: a TMA row load did not complete within the "
                             "stage kernel's wait limit\n");
        return GK_ERR_CUDA;
    }
    if (t.status) return GK_ERR_NONFINITE;
    if (t.step != 1) {
        std::fprintf(stderr, "gk_rk2_step_noalloc: a kernel of this call did not launch\n");
        return GK_ERR_CUDA;
    }
    if (dt_used) *dt_used = t.t;  // one step from t = 0: t is the dt taken
    return GK_OK;
}
