// sim.cpp -- Domain and Sim of the host interface.
//
// Domain geometry is the reference's (src/sim.cpp:16-42).  The device is
// set up at the first Advance from the state then in cons: boundaries
// (self-defined sides captured as fixed ones, fixed data, the immersed
// body's table) and point masses.  Sim::Sim reads
// the same keys (sim.cpp:45-67).  Sim::Advance replaces the reference's host
// loop (sim.cpp:69-117) with one call into libgk_cuda.so: the state is
// uploaded, the device runs every step up to the output time, and the state
// comes back into cons.  The per-step log lines the reference prints
// (sim.cpp:100-103) are printed afterwards from the device's dt log, with
// t accumulated in the same order, so they read the same.
#include <algorithm>
#include <chrono>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "gaukuk_cuda.h"
#include "sim.hpp"
#include "utils/utils.hpp"

namespace Gaukuk {

Domain::Domain(const Grid& grid)
    : xmin(Config::getInstance().get("xmin")),
      xmax(Config::getInstance().get("xmax")),
      ymin(Config::getInstance().get("ymin")),
      ymax(Config::getInstance().get("ymax")),
      zmin(Config::getInstance().get("zmin")),
      zmax(Config::getInstance().get("zmax")) {
    dx = (xmax - xmin) / grid.nx;
    dy = (ymax - ymin) / grid.ny;
    dz = (zmax - zmin) / grid.nz;
    dxRec = 1. / dx;
    dyRec = 1. / dy;
    dzRec = 1. / dz;
    if (grid.ny <= 1) dyRec = 0;
    if (grid.nz <= 1) dzRec = 0;
    drmin = std::min(std::min(dx, dy), dz);
    xc.NewArray(grid.lenx);
    yc.NewArray(grid.leny);
    zc.NewArray(grid.lenz);
    for (int i = 0; i < grid.lenx; i++) xc(i) = xmin - grid.nGhost * dx + 0.5 * dx + i * dx;
    for (int j = 0; j < grid.leny; j++) yc(j) = ymin - grid.nGhost * dy + 0.5 * dy + j * dy;
    for (int k = 0; k < grid.lenz; k++) zc(k) = zmin - grid.nGhost * dz + 0.5 * dz + k * dz;
}

Sim::Sim()
    : isContinue(true), domain(grid), flux(grid.lenx), step(0), t(0), dt(1e10),
      dtUntilOutput(1e10), cmax(1e-16) {
    Config& c = Config::getInstance();
    CFL = c.get("CFL");
    cons.NewArray(NVar, grid.lenz, grid.leny, grid.lenx);
    prim.NewArray(NVar, grid.lenz, grid.leny, grid.lenx);
    integratorType = static_cast<int>(c.get("integrator", 2));
    rcOrder = static_cast<int>(c.get("RcOrder", 1));
    stepMax = static_cast<int>(c.get("stepmax", -1));
    gpuMode_ = static_cast<int>(c.get("gpuMode", 0));
    gpuDevice_ = static_cast<int>(c.get("gpuDevice", 0));
}

Sim::~Sim() { gk_destroy(dev_); }

namespace {

void Check(gk_handle* h, int rc, const char* what) {
    if (rc == GK_OK) return;
    std::string msg = std::string(what) + ": " + gk_strerror(rc);
    if (h && *gk_last_error(h)) msg += std::string(" (") + gk_last_error(h) + ")";
    if (rc == GK_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

}  // namespace

void Sim::EnsureDevice() {
    if (dev_) return;
    std::string why;
    if (!boundary.PrepareDevice(cons, grid, eos, &why)) throw std::runtime_error(why);
    gk_grid_desc gd{};
    gd.nx = grid.nx; gd.ny = grid.ny; gd.nz = grid.nz; gd.nghost = grid.nGhost;
    gd.xmin = domain.xmin; gd.xmax = domain.xmax;
    gd.ymin = domain.ymin; gd.ymax = domain.ymax;
    gd.zmin = domain.zmin; gd.zmax = domain.zmax;
    gk_phys_desc pd{};
    pd.gamma = eos.GetGamma();
    pd.cfl = CFL;
    pd.integrator = integratorType;
    pd.rc_order = rcOrder;
    for (int s = 0; s < 6; ++s) pd.bc[s] = boundary.DeviceType(s);
    pd.grav[0] = srcTerm.Gx();
    pd.grav[1] = srcTerm.Gy();
    pd.grav[2] = srcTerm.Gz();
    pd.dfloor = DENSITY_FLOOR;
    pd.pfloor = PRESSURE_FLOOR;
    pd.stepmax = stepMax;
    pd.mode = gpuMode_ == 1 ? GK_MODE_FAST : GK_MODE_PARITY;
    pd.device = gpuDevice_;
    Check(nullptr, gk_create(&gd, &pd, &dev_), "gk_create");
    if (boundary.HasDeviceFixedData())
        Check(dev_, gk_set_fixed_boundary(dev_, boundary.DeviceFixedData().data(), boundary.FixInner()),
              "gk_set_fixed_boundary");
    if (boundary.ShellCount() > 0)
        Check(dev_, gk_set_immersed(dev_, boundary.ShellCount(), boundary.ShellIds(),
                                    boundary.ShellTargets(), boundary.ShellDirection(),
                                    boundary.ShellWeights()),
              "gk_set_immersed");
    double pm[11];
    const int npoint = srcTerm.PointParams(pm);
    if (npoint > 0) Check(dev_, gk_set_point_gravity(dev_, npoint, pm), "gk_set_point_gravity");
    for (int s = 0; s < 6; ++s) {
        if (boundary.HostDepth(s) <= 0) continue;
        hostSides_[s] = HostSide{this, s};
        Check(dev_, gk_set_host_fill(dev_, s, boundary.HostDepth(s), &Sim::HostFill, &hostSides_[s],
                                     cons.data()),
              "gk_set_host_fill");
    }
}

// A self-defined side run by the library at a ghost fill: the library has
// copied the cells the routine reads into cons and copies its ghost strip
// back afterwards.
// An exception does not cross the C ABI: it is kept and rethrown by Advance.
int Sim::HostFill(void* user, double* /*cons*/) {
    HostSide* h = static_cast<HostSide*>(user);
    try {
        h->sim->boundary.RunSide(h->side, h->sim->cons, h->sim->grid, h->sim->eos);
    } catch (const std::exception& e) {
        h->sim->hostFillError_ = e.what();
        return 1;
    }
    return 0;
}

// The reference's integrators end with cons.Swap(consTemp) (rk2.cpp:21,
// rk3.cpp:27), so its two arrays alternate as the state.  A cell that no
// ghost fill and no update ever writes keeps each array's own value: the
// setup's in cons, zero in consTemp (zero-initialised, sim.cpp:45-67), and
// the written state shows one or the other with the parity of the step
// count.  These cells: in the stored planes (all in 3D, the active one in
// 1D/2D), ghost in two or more directions, or ghost in a direction that is
// not filled (one cell wide, or a 3D z side of type 0, whose fill goes to the
// y ghosts, boundary.cpp:92-121).
void Sim::SwapUnwritten() {
    if (integratorType == 1) return;  // forward Euler updates in place
    if (unwritten_.empty() && spare_.empty()) {
        const int n[3] = {grid.nx, grid.ny, grid.nz};
        bool filled[3][2];
        for (int d = 0; d < 3; ++d)
            for (int s = 0; s < 2; ++s) filled[d][s] = n[d] > 1;
        if (grid.nz > 1)
            for (int s = 0; s < 2; ++s) filled[2][s] = boundary.DeviceType(4 + s) != 0;
        const int k0 = grid.nz > 1 ? 0 : grid.kb, k1 = grid.nz > 1 ? grid.lenz : grid.ke;
        const int lo[3] = {grid.ib, grid.jb, grid.kb}, hi[3] = {grid.ie, grid.je, grid.ke};
        for (int v = 0; v < NVar; ++v)
            for (int k = k0; k < k1; ++k)
                for (int j = 0; j < grid.leny; ++j)
                    for (int i = 0; i < grid.lenx; ++i) {
                        const int c[3] = {i, j, k};
                        int ghosts = 0, gdir = -1, gside = 0;
                        for (int d = 0; d < 3; ++d)
                            if (c[d] < lo[d] || c[d] >= hi[d]) {
                                ++ghosts;
                                gdir = d;
                                gside = c[d] < lo[d] ? 0 : 1;
                            }
                        if (ghosts == 0) continue;
                        if (ghosts == 1 && filled[gdir][gside]) continue;
                        unwritten_.push_back(&cons(v, k, j, i) - cons.data());
                    }
        spare_.assign(unwritten_.size(), 0.0);
    }
    Real* u = cons.data();
    for (size_t q = 0; q < unwritten_.size(); ++q) std::swap(u[unwritten_[q]], spare_[q]);
}

void Sim::Advance(Real dtoutput) {
    EnsureDevice();
    const int step0 = step;
    const Real t0 = t;
    const auto wall0 = std::chrono::steady_clock::now();
    Check(dev_, gk_set_time(dev_, t, step), "gk_set_time");
    Check(dev_, gk_upload_cons(dev_, cons.data()), "gk_upload_cons");
    double tt = t;
    int st = step, cont = 1;
    const int rc = gk_advance(dev_, dtoutput, &tt, &st, &cont);
    int n = 0;
    Check(dev_, gk_dt_log(dev_, nullptr, 0, &n), "gk_dt_log");
    std::vector<double> dts(n);
    if (n > 0) Check(dev_, gk_dt_log(dev_, dts.data(), n, &n), "gk_dt_log");
    Real tp = t0;
    for (int k = 0; k < (int)dts.size(); ++k) {
        tp += dts[k];
        std::cout << "step = " << step0 + k + 1 << ", t = " << tp << ", dt = " << dts[k]
                  << std::endl;
    }
    if (!hostFillError_.empty()) {
        const std::string e = hostFillError_;
        hostFillError_.clear();
        throw std::runtime_error("self-defined boundary: " + e);
    }
    Check(dev_, rc, "gk_advance");
    // The planes the device does not hold (1D/2D: the unused z-planes) and an
    // all-zero z-momentum plane on the fused 2D path are never written during
    // Advance, here or by the reference, so cons keeps its own values there.
    Check(dev_, gk_download_planes(dev_, cons.data()), "gk_download_planes");
    last_ = AdvanceStats{};
    last_.steps = st - step0;
    last_.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    if (!dts.empty()) {
        last_.dt_min = *std::min_element(dts.begin(), dts.end());
        last_.dt_max = *std::max_element(dts.begin(), dts.end());
    }
    Check(dev_, gk_floor_hits(dev_, &last_.floor_density, &last_.floor_pressure), "gk_floor_hits");
    if ((st - step0) % 2 != 0) SwapUnwritten();
    double tdev = 0, dtdev = 0;
    int sdev = 0, cdev = 1;
    Check(dev_, gk_get_time(dev_, &tdev, &dtdev, &sdev, &cdev), "gk_get_time");
    t = tt;
    step = st;
    dt = dtdev;
    isContinue = cont != 0;
    dtUntilOutput = (t0 + dtoutput) - t;
}

}  // namespace Gaukuk
