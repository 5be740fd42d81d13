// eos/eos.hpp -- adiabatic equation of state on the host.
//
// Interface of the reference's EquationOfState (src/eos/eos.hpp:13-36).
// Setup hooks call PrimToCons; Sim::WriteData calls ConsToPrim for
// primitive output; the time loop itself runs on the device.
#pragma once

#include <cmath>

#include "../gaukuk.hpp"
#include "../grid.hpp"
#include "../template_array.hpp"

namespace Gaukuk {

class EquationOfState {
public:
    EquationOfState();
    void ConsToPrim(const TArray<Real>& cons, TArray<Real>& prim, const Grid& grid);
    void ConsToPrim(const TArray<Real>& cons, TArray<Real>& prim, const Grid& grid, Real& cmax);
    void CalCmax(const TArray<Real>& cons, const Grid& grid, Real& cmax);
    void PrimToCons(const TArray<Real>& prim, TArray<Real>& cons, const Grid& grid);

    Real GetGamma() const { return gamma_; }
    Real GetGm1Rec() const { return gm1Rec_; }
    Real SoundSpeed(const Real den, const Real pre) const { return std::sqrt(gamma_ * pre / den); }
    Real EGas(const Real /*den*/, const Real pre) const { return pre * gm1Rec_; }

private:
    Real gamma_, gm1Rec_;
};

}  // namespace Gaukuk
