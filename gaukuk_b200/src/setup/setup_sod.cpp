// setup_sod.cpp -- Sod shock tube of the benchmark configs.
//
// A problem hook in the reference's API (see setup_kh_baseline.cpp) with the
// parameters of the reference's shock-tube hook (src/setup/setup_shock_tube.cpp:10-48):
// (rhoLeft, 0, pressureLeft) for x < x0, (rhoRight, 0, pressureRight) beyond.
#include "gaukuk.hpp"
#include "sim.hpp"

namespace Gaukuk {

void Sim::Setup() {
    Config& cfg = Config::getInstance();
    const Real x0 = cfg.get("x0", 0.5);
    const Real rhoLeft = cfg.get("rhoLeft", 1.0);
    const Real rhoRight = cfg.get("rhoRight", 0.125);
    const Real preLeft = cfg.get("pressureLeft", 1.0);
    const Real preRight = cfg.get("pressureRight", 0.1);
    for (int k = grid.kb; k < grid.ke; ++k)
        for (int j = grid.jb; j < grid.je; ++j)
            for (int i = grid.ib; i < grid.ie; ++i) {
                const bool left = domain.xc(i) < x0;
                prim(DEN, k, j, i) = left ? rhoLeft : rhoRight;
                prim(VLX, k, j, i) = 0.0;
                prim(VLY, k, j, i) = 0.0;
                prim(VLZ, k, j, i) = 0.0;
                prim(PRE, k, j, i) = left ? preLeft : preRight;
            }
    eos.PrimToCons(prim, cons, grid);
}

}  // namespace Gaukuk
