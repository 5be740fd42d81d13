// source_term/source.hpp -- source terms on the host interface.
//
// Interface of the reference's SourceTerm (src/source_term/source.hpp:23-50).
// A setup hook enrolls a constant gravity vector; Sim::Advance hands it to
// the device, which applies the Strang half kicks (sim.cpp:85-91).  Point
// and binary gravity can be enrolled but run on the host only, so
// Sim::Advance rejects them.
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
    void EnrollConstGravityVector(Real gx, Real gy, Real gz);
    void EnrollPointGravity(Real gm, Real x, Real y, Real z, Real vx, Real vy, Real vz, Real rs);

    bool HasConstGravity() const { return hasConstAcc_; }
    bool HasPointGravity() const { return nPoint_ > 0; }
    Real Gx() const { return gx_; }
    Real Gy() const { return gy_; }
    Real Gz() const { return gz_; }

private:
    bool hasConstAcc_ = false;
    Real gx_ = 0, gy_ = 0, gz_ = 0;
    int nPoint_ = 0;
    GravitySource obj0_, obj1_;
};

}  // namespace Gaukuk
