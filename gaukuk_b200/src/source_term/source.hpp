// source_term/source.hpp -- source terms on the host interface.
//
// Interface of the reference's SourceTerm (src/source_term/source.hpp:23-50).
// A setup hook enrolls a constant gravity vector and up to two point masses
// (one: PointGravity; two: BinaryGravity, the second mass orbiting the
// first); Sim::Advance hands them to the device, which applies the Strang
// half kicks (sim.cpp:85-91).
#pragma once

#include "../gaukuk.hpp"
#include "../grid.hpp"
#include "../template_array.hpp"

namespace Gaukuk {

struct GravitySource {
    Real gm = 0, x = 0, y = 0, z = 0, vx = 0, vy = 0, vz = 0, rs = 0;
};

class SourceTerm {
public:
    SourceTerm() = default;
    bool sourceEnrolled = false;

    void UpdateSource(TArray<Real>& cons, const Real t, const Real dt, const Grid& grid,
                      const Domain& domain);
    void ConstGravity(TArray<Real>& cons, const Real dt, const Grid& grid);
    void PointGravity(TArray<Real>& cons, const Real dt, const Grid& grid, const Domain& domain);
    void BinaryGravity(TArray<Real>& cons, const Real t, const Real dt, const Grid& grid,
                       const Domain& domain);
    void EnrollConstGravityVector(Real gx, Real gy, Real gz);
    void EnrollPointGravity(Real gm, Real x, Real y, Real z, Real vx, Real vy, Real vz, Real rs);

    bool HasConstGravity() const { return hasConstAcc_; }
    bool HasPointGravity() const { return hasPointG_ || hasBinary_; }
    Real Gx() const { return gx_; }
    Real Gy() const { return gy_; }
    Real Gz() const { return gz_; }
    // The point masses as gk_set_point_gravity takes them: returns n (0, 1
    // or 2) and fills p[11] = gm0, x0, y0, z0, rs0, gm1, z1, rs1, omega, ab,
    // theta1.
    int PointParams(double* p) const;

private:
    bool hasConstAcc_ = false, hasPointG_ = false, hasBinary_ = false;
    Real gx_ = 0, gy_ = 0, gz_ = 0;
    GravitySource obj0_, obj1_;
    Real omega_ = 0, ab_ = 0, theta1_ = 0;
};

}  // namespace Gaukuk
