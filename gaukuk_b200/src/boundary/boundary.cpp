// boundary/boundary.cpp -- host ghost fill.
//
// Side selection follows Boundary::Boundary (src/boundary/boundary.cpp:13-125),
// including its mapping of a z side of type 0 to the y copy routine, and the
// order of Boundary::UpdateBD (boundary.cpp:127-142).  Each side fills the
// ghosts of active rows/columns only, as outflow_copy.cpp, periodic.cpp,
// reflective.cpp and outflow.cpp do; loops run in the reference's order so
// the in-place result is the same even when a direction has fewer cells than
// ghosts.
#include <algorithm>
#include <stdexcept>

#include "../utils/utils.hpp"
#include "boundary.hpp"

namespace Gaukuk {

namespace {

void FillSide(TArray<Real>& u, const Grid& g, int dir, int side, int type) {
    const int len[3] = {g.lenx, g.leny, g.lenz};
    const int n[3] = {g.nx, g.ny, g.nz};
    const int b = g.nGhost, e = g.nGhost + n[dir];
    int lo[3] = {g.ib, g.jb, g.kb}, hi[3] = {g.ie, g.je, g.ke};
    lo[dir] = side == 0 ? 0 : e;
    hi[dir] = side == 0 ? b : len[dir];
    const int mom = MTX + dir;
    auto at = [&](int v, const int c[3]) -> Real& { return u(v, c[2], c[1], c[0]); };
    if (type == 0 || type == 1) {
        for (int v = DEN; v <= ENG; v++)
            for (int k = lo[2]; k < hi[2]; k++)
                for (int j = lo[1]; j < hi[1]; j++)
                    for (int i = lo[0]; i < hi[0]; i++) {
                        int c[3] = {i, j, k}, s[3] = {i, j, k};
                        if (type == 0) s[dir] = side == 0 ? b : e - 1;
                        else s[dir] = side == 0 ? c[dir] + n[dir] : c[dir] - n[dir];
                        at(v, c) = at(v, s);
                    }
        return;
    }
    for (int k = lo[2]; k < hi[2]; k++)
        for (int j = lo[1]; j < hi[1]; j++)
            for (int i = lo[0]; i < hi[0]; i++) {
                int c[3] = {i, j, k}, s[3] = {i, j, k};
                s[dir] = side == 0 ? b + b - c[dir] - 1 : e + e - c[dir] - 1;
                Real q[NVar];
                for (int v = 0; v < NVar; ++v) q[v] = at(v, s);
                if (type == 2) {
                    q[mom] = -q[mom];
                } else {
                    const Real mt = q[mom];
                    const Real mc = side == 0 ? std::min(mt, 0.0) : std::max(mt, 0.0);
                    const Real rho = std::max(q[DEN], DENSITY_FLOOR);
                    const Real rhoInv = 1.0 / rho;
                    const Real keOld = 0.5 * rhoInv * mt * mt;
                    const Real keNew = 0.5 * rhoInv * mc * mc;
                    const Real eint = std::max(q[ENG] - keOld, 1e-16);
                    q[DEN] = rho;
                    q[mom] = mc;
                    q[ENG] = eint + keNew;
                }
                for (int v = 0; v < NVar; ++v) at(v, c) = q[v];
            }
}

}  // namespace

Boundary::Boundary() {
    static const char* keys[6] = {"xleft", "xright", "yleft", "yright", "zleft", "zright"};
    BoundaryFunc* fn[6] = {&Bdxl, &Bdxr, &Bdyl, &Bdyr, &Bdzl, &Bdzr};
    for (int s = 0; s < 6; ++s) {
        int type = static_cast<int>(Config::getInstance().get(keys[s]));
        types_[s] = type;
        if (type == 4) {
            // FixedBD* (fixed.cpp:16-176): ghosts of the side's active
            // rows/columns from the state at enrollment, same index
            int dir = s / 2;
            const int side = s % 2;
            *fn[s] = [this, dir, side](TArray<Real>& u, const Grid& g, const EquationOfState&) {
                if (!fixedEnrolled_)
                    throw std::invalid_argument(
                        "fixed boundary is not initialized. call "
                        "'Boundary::EnrollFixedBoundaryData(const TArray<Real>& cons, const Grid& "
                        "grid)' in your setup");
                const int len[3] = {g.lenx, g.leny, g.lenz};
                const int n[3] = {g.nx, g.ny, g.nz};
                int lo[3] = {g.ib, g.jb, g.kb}, hi[3] = {g.ie, g.je, g.ke};
                lo[dir] = side == 0 ? 0 : g.nGhost + n[dir];
                hi[dir] = side == 0 ? g.nGhost : len[dir];
                for (int v = DEN; v <= ENG; v++)
                    for (int k = lo[2]; k < hi[2]; k++)
                        for (int j = lo[1]; j < hi[1]; j++)
                            for (int i = lo[0]; i < hi[0]; i++) u(v, k, j, i) = fixedData_(v, k, j, i);
            };
            continue;
        }
        if (type < 0 || type > 3) type = 0;
        int dir = s / 2;
        const int side = s % 2;
        if (dir == 2 && type == 0) dir = 1;  // boundary.cpp:92,104,109,121
        *fn[s] = [dir, side, type](TArray<Real>& u, const Grid& g, const EquationOfState&) {
            FillSide(u, g, dir, side, type);
        };
    }
    if (Config::getInstance().get("enableImmersed", 0) != 0) immersed_ = true;
}

void Boundary::UpdateBD(TArray<Real>& cons, const Grid& grid, const Domain& domain,
                        const EquationOfState& eos) {
    Bdxl(cons, grid, eos);
    Bdxr(cons, grid, eos);
    Bdyl(cons, grid, eos);
    Bdyr(cons, grid, eos);
    if (grid.nz > 1) {
        Bdzl(cons, grid, eos);
        Bdzr(cons, grid, eos);
    }
    if (immersed_) throw std::runtime_error("immersed boundaries are not available");
    if (fixInner_) FixedInner(cons, grid, domain);
}

// Boundary::FixedBDInner (fixed.cpp:180-206).
void Boundary::FixedInner(TArray<Real>& cons, const Grid& grid, const Domain& domain) const {
    const int il = static_cast<int>(grid.ib + 0.25 * (grid.ie - grid.ib));
    const int ir = static_cast<int>(grid.ib + 0.75 * (grid.ie - grid.ib));
    const int jl = static_cast<int>(grid.jb + 0.25 * (grid.je - grid.jb));
    const int jr = static_cast<int>(grid.jb + 0.75 * (grid.je - grid.jb));
    for (int v = DEN; v <= ENG; ++v)
        for (int k = grid.kb; k < grid.ke; ++k)
            for (int j = jl; j < jr; ++j)
                for (int i = il; i < ir; ++i) {
                    const Real x = domain.xc(i), y = domain.yc(j), z = domain.zc(k);
                    const Real r2 = x * x + y * y + z * z;
                    if (r2 < 0.5 * 0.5) cons(v, k, j, i) = fixedData_(v, k, j, i);
                }
}

void Boundary::SetupImmersedShell(const Grid&, const Domain&, Real, Real, Real, Real) {
    immersed_ = true;
}

// Boundary::EnrollFixedBoundaryData (fixed.cpp:226-268): the sides read the
// state as it is now; every side reads the same index it fills, so one copy
// of the whole state serves all sides and the inner reset.
void Boundary::EnrollFixedBoundaryData(const TArray<Real>& cons, const Grid&, bool fixInner) {
    fixedEnrolled_ = true;
    fixedData_ = cons;
    if (fixInner) fixInner_ = true;
}

const char* Boundary::DeviceBlocker() const {
    if (custom_) return "self-defined boundary routines run on the host only";
    if (immersed_) return "immersed boundaries are not implemented on the device";
    return "";
}

}  // namespace Gaukuk
