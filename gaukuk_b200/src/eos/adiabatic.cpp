// eos/adiabatic.cpp -- host adiabatic EOS.  Same ranges and operation order
// as the reference (src/eos/adiabatic.cpp:12-198), so a setup hook produces
// the same bits here as with the reference.
#include <algorithm>
#include <cmath>

#include "../utils/utils.hpp"
#include "eos.hpp"

namespace Gaukuk {

EquationOfState::EquationOfState() {
    gamma_ = Config::getInstance().get("gamma");
    gm1Rec_ = 1.0 / (gamma_ - 1.0);
}

namespace {

// z range of the primitive/conserved conversions: every plane in 3D, the
// active plane when nz == 1 (adiabatic.cpp:25-28).
void PlaneRange(const Grid& g, int& kl, int& kr) {
    kl = g.kgb;
    kr = g.kge;
    if (g.nz == 1) {
        kl = g.kb;
        kr = g.ke;
    }
}

}  // namespace

void EquationOfState::ConsToPrim(const TArray<Real>& cons, TArray<Real>& prim, const Grid& grid) {
    Real cmax = 0;
    ConsToPrim(cons, prim, grid, cmax);
}

void EquationOfState::ConsToPrim(const TArray<Real>& cons, TArray<Real>& prim, const Grid& grid,
                                 Real& cmax) {
    int kl, kr;
    PlaneRange(grid, kl, kr);
    const Real gm1 = gamma_ - 1.0, dmin = DENSITY_FLOOR, pmin = PRESSURE_FLOOR;
    for (int k = kl; k < kr; k++)
        for (int j = grid.jgb; j < grid.jge; j++)
            for (int i = grid.igb; i < grid.ige; i++) {
                const Real mx = cons(MTX, k, j, i), my = cons(MTY, k, j, i);
                const Real mz = cons(MTZ, k, j, i), e = cons(ENG, k, j, i);
                const Real d = std::max(cons(DEN, k, j, i), dmin);
                const Real denInv = 1.0 / d;
                prim(DEN, k, j, i) = d;
                prim(VLX, k, j, i) = mx * denInv;
                prim(VLY, k, j, i) = my * denInv;
                prim(VLZ, k, j, i) = mz * denInv;
                const Real engKin = 0.5 * denInv * (mx * mx + my * my + mz * mz);
                Real pre = gm1 * (e - engKin);
                pre = (pre > pmin) ? pre : pmin;
                prim(PRE, k, j, i) = pre;
                const Real cs = std::sqrt(gamma_ * pre * denInv);
                Real local = std::abs(prim(VLX, k, j, i)) + cs;
                local = std::max(local, std::abs(prim(VLY, k, j, i)) + cs);
                local = std::max(local, std::abs(prim(VLZ, k, j, i)) + cs);
                cmax = std::max(cmax, local);
            }
}

void EquationOfState::CalCmax(const TArray<Real>& cons, const Grid& grid, Real& cmax) {
    const Real gm1 = gamma_ - 1.0, dmin = DENSITY_FLOOR, pmin = PRESSURE_FLOOR;
    for (int k = grid.kb; k < grid.ke; k++)
        for (int j = grid.jb; j < grid.je; j++)
            for (int i = grid.ib; i < grid.ie; i++) {
                const Real mx = cons(MTX, k, j, i), my = cons(MTY, k, j, i);
                const Real mz = cons(MTZ, k, j, i), e = cons(ENG, k, j, i);
                const Real d = std::max(cons(DEN, k, j, i), dmin);
                const Real denInv = 1.0 / d;
                const Real vx = mx * denInv, vy = my * denInv, vz = mz * denInv;
                const Real engKin = 0.5 * (vx * mx + vy * my + vz * mz);
                Real pres = gm1 * (e - engKin);
                pres = (pres > pmin) ? pres : pmin;
                const Real cs = std::sqrt(gamma_ * pres * denInv);
                Real local = std::abs(vx) + cs;
                local = std::max(local, std::abs(vy) + cs);
                local = std::max(local, std::abs(vz) + cs);
                cmax = std::max(cmax, local);
            }
}

void EquationOfState::PrimToCons(const TArray<Real>& prim, TArray<Real>& cons, const Grid& grid) {
    int kl, kr;
    PlaneRange(grid, kl, kr);
    for (int k = kl; k < kr; k++)
        for (int j = grid.jgb; j < grid.jge; j++)
            for (int i = grid.igb; i < grid.ige; i++) {
                const Real d = prim(DEN, k, j, i), vx = prim(VLX, k, j, i);
                const Real vy = prim(VLY, k, j, i), vz = prim(VLZ, k, j, i);
                const Real p = prim(PRE, k, j, i);
                cons(DEN, k, j, i) = d;
                cons(MTX, k, j, i) = d * vx;
                cons(MTY, k, j, i) = d * vy;
                cons(MTZ, k, j, i) = d * vz;
                cons(ENG, k, j, i) = p * gm1Rec_ + 0.5 * d * (vx * vx + vy * vy + vz * vz);
            }
}

}  // namespace Gaukuk
