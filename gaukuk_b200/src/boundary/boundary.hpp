// boundary/boundary.hpp -- ghost-zone fill on the host.
//
// Interface of the reference's Boundary (src/boundary/boundary.hpp:15-111):
// one std::function per side chosen from xleft..zright (0 copy, 1 periodic,
// 2 reflective, 3 outflow, 4 fixed), UpdateBD, and the Enroll* hooks with
// which a setup file installs its own static SelfDefineBD* routines or the
// fixed-boundary data, and the immersed solid body (immersed.cpp).  The host
// fill is used for the state a setup hook produces (main.cpp:30) and for
// output; during Sim::Advance the device fills ghosts with the same rules:
// fixed sides, the immersed body and the inner reset included.  The device
// cannot call a hook's own routine: PrepareDevice turns one whose writes do
// not depend on the state into a fixed side; one that reads the state runs
// on the host at every ghost fill, on the cells it was found to read.  A
// routine that writes outside its side's ghost strip is rejected.
#pragma once

#include <functional>
#include <string>
#include <vector>

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
    // Readies the device's view of the ghost fill from the state `cons`:
    // every self-defined side must be stationary (see boundary.cpp) and then
    // becomes a fixed side with the values it writes.  False with the reason
    // in *why when a side cannot run on the device.
    bool PrepareDevice(const TArray<Real>& cons, const Grid& grid, const EquationOfState& eos,
                       std::string* why);
    // After PrepareDevice: the ghost-fill type of side s on the device, and
    // the fixed-side data (the enrolled snapshot with captured sides written
    // in; empty when no side is fixed).
    int DeviceType(int s) const { return deviceTypes_[s]; }
    // After PrepareDevice: 0, or for a self-defined side that reads the state
    // the number of cell layers next to its ghost strip that it reads (the
    // library copies strip + layers to the host before each call).
    int HostDepth(int s) const { return hostDepth_[s]; }
    // Runs the routine installed for side s on cons.
    void RunSide(int s, TArray<Real>& cons, const Grid& grid, const EquationOfState& eos) const;
    const TArray<Real>& DeviceFixedData() const { return deviceFixed_; }
    bool HasDeviceFixedData() const { return deviceFixedSet_; }

    // The immersed body's table in the reference's layout (immersed.cpp:146-150):
    // ids (3, nShell, 9), nTars (nShell), direction (4, nShell), disGamma (nShell, 9).
    int ShellCount() const { return nShell_; }
    const int* ShellIds() const { return shellIds_.data(); }
    const int* ShellTargets() const { return nTars_.data(); }
    const Real* ShellDirection() const { return shellDir_.data(); }
    const Real* ShellWeights() const { return disGamma_.data(); }

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

    static constexpr int kTarMax = 8;  // nTarMax (boundary.hpp:109)
    int nShell_ = 0;
    std::vector<int> shellIds_, nTars_;
    std::vector<Real> shellDir_, disGamma_;
    void ImmersedReflective(TArray<Real>& cons, const EquationOfState& eos) const;

    int deviceTypes_[6] = {0, 0, 0, 0, 0, 0};
    int hostDepth_[6] = {0, 0, 0, 0, 0, 0};
    bool deviceFixedSet_ = false;
    TArray<Real> deviceFixed_;
};

}  // namespace Gaukuk
