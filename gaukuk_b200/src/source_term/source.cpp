// source_term/source.cpp -- host source terms (src/source_term/source.cpp:12-31,
// const_gravity.cpp:10-69).
#include <stdexcept>

#include "source.hpp"

namespace Gaukuk {

void SourceTerm::UpdateSource(TArray<Real>& cons, const Real, const Real dt, const Grid& grid,
                              const Domain&) {
    if (hasConstAcc_) ConstGravity(cons, dt, grid);
    if (nPoint_ > 0) throw std::runtime_error("point gravity is not available");
}

void SourceTerm::ConstGravity(TArray<Real>& cons, const Real dt, const Grid& grid) {
    const Real g[3] = {gx_, gy_, gz_};
    for (int d = 0; d < 3; ++d) {
        if (g[d] == 0) continue;
        const int mom = MTX + d;
        for (int k = grid.kb; k < grid.ke; k++)
            for (int j = grid.jb; j < grid.je; j++)
                for (int i = grid.ib; i < grid.ie; i++) {
                    cons(ENG, k, j, i) += cons(mom, k, j, i) * g[d] * dt;
                    cons(mom, k, j, i) += cons(DEN, k, j, i) * g[d] * dt;
                }
    }
}

void SourceTerm::EnrollConstGravityVector(Real gx, Real gy, Real gz) {
    gx_ = gx;
    gy_ = gy;
    gz_ = gz;
    if (gx_ != 0 || gy_ != 0 || gz_ != 0) {
        sourceEnrolled = true;
        hasConstAcc_ = true;
    }
}

void SourceTerm::EnrollPointGravity(Real gm, Real x, Real y, Real z, Real vx, Real vy, Real vz,
                                    Real rs) {
    if (nPoint_ >= 2) throw std::runtime_error("Setup failed: too many point gravity.");
    GravitySource& o = nPoint_ == 0 ? obj0_ : obj1_;
    o.gm = gm; o.x = x; o.y = y; o.z = z; o.vx = vx; o.vy = vy; o.vz = vz; o.rs = rs;
    ++nPoint_;
    sourceEnrolled = true;
}

}  // namespace Gaukuk
