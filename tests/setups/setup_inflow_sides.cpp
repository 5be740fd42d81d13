// setup_inflow_sides.cpp -- a test hook with a self-defined x-left side.
//
// A uniform flow; the x-left ghosts come from the hook's own routine.  With
// the input key inflowCopies = 1 the routine copies the first active column
// (the copy template of the reference's setup files), so its writes depend
// on the state; with inflowWide = 1 it writes the constant state into the
// corner ghosts as well, outside the side's strip; otherwise it writes a
// constant inflow state into the strip, as the reference's solid-body hook
// does (src/setup/setup_solid_body.cpp:62-96).  With inflowThrowAfter = N > 0
// the routine throws from its (N+1)-th call on (a failing host routine).
#include <stdexcept>

#include "gaukuk.hpp"
#include "sim.hpp"

namespace Gaukuk {

void Sim::Setup() {
    for (int k = grid.kb; k < grid.ke; ++k)
        for (int j = grid.jb; j < grid.je; ++j)
            for (int i = grid.ib; i < grid.ie; ++i) {
                prim(DEN, k, j, i) = 1.0;
                prim(VLX, k, j, i) = 1.0;
                prim(VLY, k, j, i) = 0.0;
                prim(VLZ, k, j, i) = 0.0;
                prim(PRE, k, j, i) = 1.0;
            }
    eos.PrimToCons(prim, cons, grid);
    boundary.EnrollSelfDefineBDXL();
}

void Boundary::SelfDefineBDXL(TArray<Real>& cons, const Grid& grid, const EquationOfState& eos) {
    static int calls = 0;
    const int throw_after = static_cast<int>(Config::getInstance().get("inflowThrowAfter", 0));
    if (throw_after > 0 && ++calls > throw_after) throw std::runtime_error("inflow routine failed");
    const bool copies = Config::getInstance().get("inflowCopies", 0) != 0;
    const bool wide = Config::getInstance().get("inflowWide", 0) != 0;
    const Real q[NVar] = {2.0, 2.0, 0.0, 0.0, 1.0 + eos.EGas(2.0, 1.0)};
    for (int v = DEN; v <= ENG; ++v)
        for (int k = grid.kb; k < grid.ke; ++k)
            for (int j = wide ? grid.jgb : grid.jb; j < (wide ? grid.jge : grid.je); ++j)
                for (int i = grid.igb; i < grid.ib; ++i) {
                    cons(v, k, j, i) = copies ? cons(v, k, j, grid.ib) : q[v];
                }
}

}  // namespace Gaukuk
