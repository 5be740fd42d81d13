// setup_rt_baseline.cpp -- Rayleigh-Taylor problem of the benchmark configs.
//
// A problem hook in the reference's API (see setup_kh_baseline.cpp).  The
// shape follows the reference's RT hook (src/setup/setup_rt.cpp:11-70) with
// one added key, p0, the pressure at y = 0 (the reference hard-codes
// 1/gamma, which stays the default):
//   rho = rhoUp for y > 0 else rhoDown,  p = p0 + gravAccY*rho*y
//   vy  = amp*(1 + cos(kx x))*(1 + cos(ky y))/4,  kx = nx_ptb*pi/Lx, ky = ny_ptb*pi/Ly
// and constant gravity (0, gravAccY, 0) is enrolled as a source term.
#include <cmath>

#include "gaukuk.hpp"
#include "sim.hpp"

namespace Gaukuk {

void Sim::Setup() {
    Config& cfg = Config::getInstance();
    const Real gamma = cfg.get("gamma", 1.4);
    const Real rhoUp = cfg.get("rhoUp", 2.0);
    const Real rhoDown = cfg.get("rhoDown", 1.0);
    const Real amp = cfg.get("amp", 0.01);
    const Real gy = cfg.get("gravAccY", -0.1);
    const Real nxPtb = cfg.get("nx_ptb", 2.0);
    const Real nyPtb = cfg.get("ny_ptb", 2.0);
    const Real p0 = cfg.get("p0", 1.0 / gamma);

    const Real Lx = domain.xmax - domain.xmin;
    const Real Ly = domain.ymax - domain.ymin;
    const Real kx = nxPtb * PI / Lx;
    const Real ky = nyPtb * PI / Ly;
    for (int k = grid.kb; k < grid.ke; ++k) {
        for (int j = grid.jb; j < grid.je; ++j) {
            const Real y = domain.yc(j);
            const Real rho = (y > 0.0) ? rhoUp : rhoDown;
            for (int i = grid.ib; i < grid.ie; ++i) {
                const Real x = domain.xc(i);
                const Real shape = (1.0 + std::cos(kx * x)) * (1.0 + std::cos(ky * y)) / 4.0;
                prim(DEN, k, j, i) = rho;
                prim(VLX, k, j, i) = 0.0;
                prim(VLY, k, j, i) = amp * shape;
                prim(VLZ, k, j, i) = 0.0;
                prim(PRE, k, j, i) = p0 + gy * rho * y;
            }
        }
    }
    srcTerm.EnrollConstGravityVector(0, gy, 0);
    eos.PrimToCons(prim, cons, grid);
}

}  // namespace Gaukuk
