// source_term/source.cpp -- host source terms (src/source_term/source.cpp:12-68,
// const_gravity.cpp:10-69, point_gravity.cpp:11-92, binary_gravity.cpp).
// Sim::Advance runs the same kicks on the device; these host versions serve
// code that calls UpdateSource itself.
#include <cmath>
#include <stdexcept>

#include "source.hpp"

namespace Gaukuk {

void SourceTerm::UpdateSource(TArray<Real>& cons, const Real t, const Real dt, const Grid& grid,
                              const Domain& domain) {
    if (hasConstAcc_) ConstGravity(cons, dt, grid);
    if (hasPointG_) PointGravity(cons, dt, grid, domain);
    else if (hasBinary_) BinaryGravity(cons, t, dt, grid, domain);
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

namespace {

// The kick of one cell by an acceleration times dt.
inline void Kick(TArray<Real>& cons, int k, int j, int i, Real gxdt, Real gydt, Real gzdt) {
    Real& d = cons(DEN, k, j, i);
    Real& mx = cons(MTX, k, j, i);
    Real& my = cons(MTY, k, j, i);
    Real& mz = cons(MTZ, k, j, i);
    Real& e = cons(ENG, k, j, i);
    e += mx * gxdt + my * gydt + mz * gzdt;
    mx += d * gxdt;
    my += d * gydt;
    mz += d * gzdt;
}

}  // namespace

void SourceTerm::PointGravity(TArray<Real>& cons, const Real dt, const Grid& grid,
                              const Domain& domain) {
    const Real gmdt = obj0_.gm * dt;
    for (int k = grid.kb; k < grid.ke; k++)
        for (int j = grid.jb; j < grid.je; j++)
            for (int i = grid.ib; i < grid.ie; i++) {
                const Real delx = domain.xc(i) - obj0_.x;
                const Real dely = domain.yc(j) - obj0_.y;
                const Real delz = domain.zc(k) - obj0_.z;
                const Real r2 = delx * delx + dely * dely + delz * delz;
                const Real rInv = 1.0 / std::sqrt(r2 + obj0_.rs * obj0_.rs);
                const Real gv = -gmdt * rInv * rInv * rInv;
                Kick(cons, k, j, i, gv * delx, gv * dely, gv * delz);
            }
}

void SourceTerm::BinaryGravity(TArray<Real>& cons, const Real t, const Real dt, const Grid& grid,
                               const Domain& domain) {
    const Real gm0dt = obj0_.gm * dt, gm1dt = obj1_.gm * dt;
    const Real theta = omega_ * t + theta1_;
    obj1_.x = ab_ * std::cos(theta);
    obj1_.y = ab_ * std::sin(theta);
    const Real x1 = obj1_.x, y1 = obj1_.y, z1 = obj1_.z;
    const Real gInd = 0;  // the indirect term, zeroed in binary_gravity.cpp
    for (int k = grid.kb; k < grid.ke; k++)
        for (int j = grid.jb; j < grid.je; j++)
            for (int i = grid.ib; i < grid.ie; i++) {
                const Real xn = domain.xc(i), yn = domain.yc(j), zn = domain.zc(k);
                const Real dx0 = xn - obj0_.x, dy0 = yn - obj0_.y, dz0 = zn - obj0_.z;
                const Real dx1 = xn - x1, dy1 = yn - y1, dz1 = zn - z1;
                const Real r0 = dx0 * dx0 + dy0 * dy0 + dz0 * dz0;
                const Real r0Inv = 1.0 / std::sqrt(r0 + obj0_.rs * obj0_.rs);
                const Real g0 = -gm0dt * r0Inv * r0Inv * r0Inv;
                const Real r1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1;
                const Real r1Inv = 1.0 / std::sqrt(r1 + obj1_.rs * obj1_.rs);
                const Real g1 = -gm1dt * r1Inv * r1Inv * r1Inv;
                Kick(cons, k, j, i, g0 * dx0 + g1 * dx1 + gInd * x1, g0 * dy0 + g1 * dy1 + gInd * y1,
                     g0 * dz0 + g1 * dz1 + gInd * z1);
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

// The first mass is fixed; a second one makes a binary whose separation,
// angular speed and phase are fixed here (source.cpp:33-68).
void SourceTerm::EnrollPointGravity(Real gm, Real x, Real y, Real z, Real vx, Real vy, Real vz,
                                    Real rs) {
    if (hasBinary_) throw std::runtime_error("Setup failed: too many point gravity.");
    if (hasPointG_) {
        obj1_ = GravitySource{gm, x, y, z, vx, vy, vz, rs};
        ab_ = std::sqrt((x - obj0_.x) * (x - obj0_.x) + (y - obj0_.y) * (y - obj0_.y) +
                        (z - obj0_.z) * (z - obj0_.z));
        omega_ = std::sqrt((obj0_.gm + gm) / (ab_ * ab_ * ab_));
        theta1_ = std::atan2(y - obj0_.y, x - obj0_.x);
        hasBinary_ = true;
        hasPointG_ = false;
    } else {
        obj0_ = GravitySource{gm, x, y, z, vx, vy, vz, rs};
        hasPointG_ = true;
    }
    sourceEnrolled = true;
}

int SourceTerm::PointParams(double* p) const {
    const double v[11] = {obj0_.gm, obj0_.x, obj0_.y, obj0_.z, obj0_.rs, obj1_.gm,
                          obj1_.z,  obj1_.rs, omega_, ab_,     theta1_};
    for (int i = 0; i < 11; ++i) p[i] = v[i];
    return hasBinary_ ? 2 : (hasPointG_ ? 1 : 0);
}

}  // namespace Gaukuk
