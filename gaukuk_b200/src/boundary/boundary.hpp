// boundary/boundary.hpp -- ghost-zone fill on the host.
//
// Interface of the reference's Boundary (src/boundary/boundary.hpp:15-111):
// one std::function per side chosen from xleft..zright (0 copy, 1 periodic,
// 2 reflective, 3 outflow, 4 fixed), UpdateBD, and the Enroll* hooks with
// which a setup file installs its own static SelfDefineBD* routines or the
// fixed-boundary data.  The host fill is used for the state a setup hook
// produces (main.cpp:30) and for output; during Sim::Advance the device fills
// ghosts with the same rules, fixed sides and the inner reset included.
// Problems that enroll their own routines or an immersed body run on the
// host only and Sim::Advance rejects them.
#pragma once

#include <functional>

#include "../eos/eos.hpp"
#include "../gaukuk.hpp"
#include "../grid.hpp"
#include "../template_array.hpp"

namespace Gaukuk {

class Boundary {
    using BoundaryFunc = std::function<void(TArray<Real>&, const Grid&, const EquationOfState&)>;

public:
    Boundary();
    BoundaryFunc Bdxl, Bdxr, Bdyl, Bdyr, Bdzl, Bdzr;
    void UpdateBD(TArray<Real>& cons, const Grid& grid, const Domain& domain,
                  const EquationOfState& eos);

    void EnrollSelfDefineBDXL() { Bdxl = &SelfDefineBDXL; custom_ |= 1; }
    void EnrollSelfDefineBDXR() { Bdxr = &SelfDefineBDXR; custom_ |= 2; }
    void EnrollSelfDefineBDYL() { Bdyl = &SelfDefineBDYL; custom_ |= 4; }
    void EnrollSelfDefineBDYR() { Bdyr = &SelfDefineBDYR; custom_ |= 8; }
    void EnrollSelfDefineBDZL() { Bdzl = &SelfDefineBDZL; custom_ |= 16; }
    void EnrollSelfDefineBDZR() { Bdzr = &SelfDefineBDZR; custom_ |= 32; }

    void SetupImmersedShell(const Grid& grid, const Domain& domain, Real xShell, Real yShell,
                            Real zShell, Real rShell);
    void EnrollFixedBoundaryData(const TArray<Real>& cons, const Grid& grid, bool fixInner = false);

    // The configured type of side s (xleft, xright, yleft, yright, zleft, zright).
    int Type(int s) const { return types_[s]; }
    // The state at EnrollFixedBoundaryData (empty when not enrolled).
    const TArray<Real>& FixedData() const { return fixedData_; }
    bool HasFixedData() const { return fixedEnrolled_; }
    bool FixInner() const { return fixInner_; }
    // Why the device path cannot take this configuration ("" when it can).
    const char* DeviceBlocker() const;

private:
    static void SelfDefineBDXL(TArray<Real>& cons, const Grid& grid, const EquationOfState& eos);
    static void SelfDefineBDXR(TArray<Real>& cons, const Grid& grid, const EquationOfState& eos);
    static void SelfDefineBDYL(TArray<Real>& cons, const Grid& grid, const EquationOfState& eos);
    static void SelfDefineBDYR(TArray<Real>& cons, const Grid& grid, const EquationOfState& eos);
    static void SelfDefineBDZL(TArray<Real>& cons, const Grid& grid, const EquationOfState& eos);
    static void SelfDefineBDZR(TArray<Real>& cons, const Grid& grid, const EquationOfState& eos);

    int types_[6] = {0, 0, 0, 0, 0, 0};
    int custom_ = 0;
    bool immersed_ = false;
    bool fixedEnrolled_ = false, fixInner_ = false;
    TArray<Real> fixedData_;
    void FixedInner(TArray<Real>& cons, const Grid& grid, const Domain& domain) const;
};

}  // namespace Gaukuk
