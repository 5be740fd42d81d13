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
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
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
    if (immersed_) ImmersedReflective(cons, eos);
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

namespace {

// FindLeftId / FindRightId (immersed.cpp:19-47): the first active index
// whose centre is at or past centre - 1.2 r (from below), or at or before
// centre + 1.2 r (from above); the body's reach must lie in the domain.
int FirstFrom(const TArray<Real>& xc, int b, int e, Real centre, Real r, Real lo) {
    const Real edge = centre - 1.2 * r;
    if (edge < lo) throw std::invalid_argument("immersed boundary out of domain");
    for (int i = b; i < e; i++)
        if (xc(i) >= edge) return i;
    return e;
}
int LastFrom(const TArray<Real>& xc, int b, int e, Real centre, Real r, Real hi) {
    const Real edge = centre + 1.2 * r;
    if (edge > hi) throw std::invalid_argument("immersed boundary out of domain");
    for (int i = e - 1; i >= b; i--)
        if (xc(i) <= edge) return i;
    return b;
}

Real Norm3(Real a, Real b, Real c) { return std::sqrt(a * a + b * b + c * c); }

// IsShellCell (immersed.cpp:49-68): inside the body, with one of the six
// cells two ghost widths away along an axis outside it.
bool IsShell(Real dx, Real dy, Real dz, Real r, Real sx, Real sy, Real sz) {
    if (!(Norm3(dx, dy, dz) < r)) return false;
    const Real shift[6][3] = {{sx, 0, 0}, {-sx, 0, 0}, {0, sy, 0}, {0, -sy, 0}, {0, 0, sz}, {0, 0, -sz}};
    for (const auto& s : shift)
        if (Norm3(dx + s[0], dy + s[1], dz + s[2]) > r) return true;
    return false;
}

}  // namespace

// Boundary::SetupImmersedShell (immersed.cpp:89-241): the shell cells of a
// sphere (a cylinder through the plane in 2D) and, for each, the active
// cells within one cell of its image point across the surface that lie
// outside the body, with inverse-square-distance weights in which the cell
// itself (distance twice its depth) takes part.  Cells are listed in k, j, i
// order; targets in the reference's search order (i, then j, then k offset).
void Boundary::SetupImmersedShell(const Grid& grid, const Domain& domain, Real xShell, Real yShell,
                                  Real zShell, Real rShell) {
    if (grid.nx <= 1 || grid.ny <= 1)
        throw std::invalid_argument("immersed boundary has to be at least 2D. ");
    immersed_ = true;
    const int il = FirstFrom(domain.xc, grid.ib, grid.ie, xShell, rShell, domain.xmin);
    const int ir = LastFrom(domain.xc, grid.ib, grid.ie, xShell, rShell, domain.xmax);
    const int jl = FirstFrom(domain.yc, grid.jb, grid.je, yShell, rShell, domain.ymin);
    const int jr = LastFrom(domain.yc, grid.jb, grid.je, yShell, rShell, domain.ymax);
    int kl = grid.kb, kr = grid.ke;
    if (grid.nz > 1) {
        kl = FirstFrom(domain.zc, grid.kb, grid.ke, zShell, rShell, domain.zmin);
        kr = LastFrom(domain.zc, grid.kb, grid.ke, zShell, rShell, domain.zmax);
    }
    nShell_ = 0;
    if (il > ir || jl > jr || kl > kr) throw std::invalid_argument("immersed boundary out of domain");
    const Real sx = grid.nGhost * domain.dx, sy = grid.nGhost * domain.dy,
               sz = grid.nGhost * domain.dz;
    std::vector<int> cells;  // (i, j, k) triples
    for (int k = kl; k < kr; k++)
        for (int j = jl; j < jr; j++)
            for (int i = il; i < ir; i++)
                if (IsShell(domain.xc(i) - xShell, domain.yc(j) - yShell, domain.zc(k) - zShell,
                            rShell, sx, sy, sz)) {
                    cells.push_back(i);
                    cells.push_back(j);
                    cells.push_back(k);
                }
    const int n = static_cast<int>(cells.size() / 3);
    const int W = kTarMax + 1;
    shellIds_.assign((size_t)3 * n * W, 0);
    nTars_.assign(n, 0);
    shellDir_.assign((size_t)4 * n, 0.0);
    disGamma_.assign((size_t)n * W, 0.0);
    auto id = [&](int c, int s, int t) -> int& { return shellIds_[((size_t)c * n + s) * W + t]; };
    const int rx = 2 * grid.nGhost, ry = 2 * grid.nGhost, rz = grid.nz > 1 ? 2 * grid.nGhost : 0;
    for (int s = 0; s < n; s++) {
        const int i = cells[3 * s], j = cells[3 * s + 1], k = cells[3 * s + 2];
        id(0, s, 0) = i;
        id(1, s, 0) = j;
        id(2, s, 0) = k;
        const Real delx = domain.xc(i) - xShell, dely = domain.yc(j) - yShell,
                   delz = domain.zc(k) - zShell;
        const Real rnow = Norm3(delx, dely, delz);
        const Real rxy = std::sqrt(delx * delx + dely * dely);
        Real cosp = 1.0, sinp = 0.0, cost = 1.0, sint = 0.0;
        if (!(rxy < 1e-15)) {
            cosp = delx / rxy;
            sinp = dely / rxy;
        }
        if (!(rnow < 1e-15)) {
            cost = delz / rnow;
            sint = rxy / rnow;
        }
        shellDir_[0 * (size_t)n + s] = cosp;
        shellDir_[1 * (size_t)n + s] = sinp;
        shellDir_[2 * (size_t)n + s] = cost;
        shellDir_[3 * (size_t)n + s] = sint;
        // the image point: the cell reflected through the surface
        const Real xImg = sint * cosp * (2 * rShell - rnow) + xShell;
        const Real yImg = sint * sinp * (2 * rShell - rnow) + yShell;
        const Real zImg = cost * (2 * rShell - rnow) + zShell;
        Real dist[kTarMax + 1];
        dist[0] = 2 * (rShell - rnow);
        int nt = 0;
        for (int a = -rx; a < rx + 1; ++a)
            for (int b = -ry; b < ry + 1; ++b)
                for (int c = -rz; c < rz + 1; ++c) {
                    const int it = i + a, jt = j + b, kt = k + c;
                    if (it < grid.ib || it >= grid.ie || jt < grid.jb || jt >= grid.je ||
                        kt < grid.kb || kt >= grid.ke)
                        throw std::invalid_argument(
                            "immersed body is too close to the domain boundary, neighboor search "
                            "out of range.");
                    const Real xt = domain.xc(it), yt = domain.yc(jt), zt = domain.zc(kt);
                    if (!(std::abs(xt - xImg) <= domain.dx && std::abs(yt - yImg) <= domain.dy &&
                          std::abs(zt - zImg) <= domain.dz))
                        continue;
                    if (!(Norm3(xt - xShell, yt - yShell, zt - zShell) > rShell)) continue;
                    if (++nt > kTarMax)
                        throw std::logic_error("n of imagine points is more than nTarMax");
                    id(0, s, nt) = it;
                    id(1, s, nt) = jt;
                    id(2, s, nt) = kt;
                    dist[nt] = Norm3(xt - xImg, yt - yImg, zt - zImg);
                }
        nTars_[s] = nt;
        Real sum = 0.;
        for (int t = 0; t < nt + 1; t++) sum = sum + 1. / (dist[t] * dist[t]);
        for (int t = 0; t < nt + 1; t++) disGamma_[(size_t)s * W + t] = 1. / (dist[t] * dist[t] * sum);
    }
    nShell_ = n;
}

// Boundary::ImmersedReflective (immersed.cpp:243-303): every shell cell gets
// the weighted image-point state of its targets, radial velocity reversed.
// Targets are outside the body and shell cells inside, so the order of the
// cells does not matter.
void Boundary::ImmersedReflective(TArray<Real>& cons, const EquationOfState& eos) const {
    const Real gm1 = eos.GetGamma() - 1;
    const int n = nShell_, W = kTarMax + 1;
    auto id = [&](int c, int s, int t) { return shellIds_[((size_t)c * n + s) * W + t]; };
    for (int s = 0; s < n; s++) {
        const Real cosp = shellDir_[s], sinp = shellDir_[(size_t)n + s],
                   cost = shellDir_[2 * (size_t)n + s], sint = shellDir_[3 * (size_t)n + s];
        const Real w0 = disGamma_[(size_t)s * W];
        Real dens = 0, vr = 0, vp = 0, vt = 0, pres = 0;
        for (int t = 1; t <= nTars_[s]; t++) {
            const int it = id(0, s, t), jt = id(1, s, t), kt = id(2, s, t);
            const Real wt = disGamma_[(size_t)s * W + t];
            const Real denTar = std::max(cons(DEN, kt, jt, it), DENSITY_FLOOR);
            const Real denInv = 1.0 / denTar;
            dens += 1. / (1 - w0) * wt * denTar;
            const Real vx = cons(MTX, kt, jt, it) * denInv;
            const Real vy = cons(MTY, kt, jt, it) * denInv;
            const Real vz = cons(MTZ, kt, jt, it) * denInv;
            // velocity in the local (r, phi, theta) frame (immersed.cpp:72-77)
            const Real vrl = vx * cosp * sint + vy * sinp * sint + vz * cost;
            const Real vpl = -vx * sinp + vy * cosp;
            const Real vtl = vx * cosp * cost + vy * sinp * cost - vz * sint;
            vr += 1. / (-1. - w0) * wt * vrl;
            vp += 1. / (1. - w0) * wt * vpl;
            vt += 1. / (1. - w0) * wt * vtl;
            const Real engKin = 0.5 * denTar * (vx * vx + vy * vy + vz * vz);
            Real pre = gm1 * (cons(ENG, kt, jt, it) - engKin);
            pre = (pre > PRESSURE_FLOOR) ? pre : PRESSURE_FLOOR;
            pres += 1. / (1. - w0) * wt * pre;
        }
        // back to Cartesian (immersed.cpp:80-85)
        const Real vx = vr * sint * cosp + vt * cost * cosp - vp * sinp;
        const Real vy = vr * sint * sinp + vt * cost * sinp + vp * cosp;
        const Real vz = vr * cost - vt * sint;
        const int i = id(0, s, 0), j = id(1, s, 0), k = id(2, s, 0);
        cons(DEN, k, j, i) = dens;
        cons(MTX, k, j, i) = dens * vx;
        cons(MTY, k, j, i) = dens * vy;
        cons(MTZ, k, j, i) = dens * vz;
        const Real engKin = 0.5 * dens * (vx * vx + vy * vy + vz * vz);
        cons(ENG, k, j, i) = engKin + eos.EGas(dens, pres);
    }
}

// Boundary::EnrollFixedBoundaryData (fixed.cpp:226-268): the sides read the
// state as it is now; every side reads the same index it fills, so one copy
// of the whole state serves all sides and the inner reset.
void Boundary::EnrollFixedBoundaryData(const TArray<Real>& cons, const Grid&, bool fixInner) {
    fixedEnrolled_ = true;
    fixedData_ = cons;
    if (fixInner) fixInner_ = true;
}

namespace {

bool SameBits(Real a, Real b) {
    std::uint64_t x, y;
    std::memcpy(&x, &a, sizeof x);
    std::memcpy(&y, &b, sizeof y);
    return x == y;
}

}  // namespace

// A self-defined side (a setup's SelfDefineBD* routine) is run three times
// on copies of the state: the state itself, every value -1e300, every value
// NaN.  It is stationary when it writes exactly the cells a fixed side of
// that side fills (the ghosts of the active rows or columns), each with the
// same bits in all three runs, and nothing else: then its writes depend on
// the state in no way the probes can see, and the device fills the side as
// a fixed side from the values captured.  A cell it skips keeps -1e300 in one
// run and NaN in the other, so partial fills are caught; so are routines
// that copy or scale state values.  A routine that throws, or anything else,
// keeps the run on the host.
void Boundary::RunSide(int s, TArray<Real>& cons, const Grid& grid,
                       const EquationOfState& eos) const {
    const BoundaryFunc* fn[6] = {&Bdxl, &Bdxr, &Bdyl, &Bdyr, &Bdzl, &Bdzr};
    (*fn[s])(cons, grid, eos);
}

// How the device runs each self-defined side, from probes of its routine on
// copies of the state:
// * the routine must write only its side's ghost strip (ghost layers, active
//   transverse cells): on arrays filled with -1e300 and with NaN, every other
//   cell keeps the fill -- otherwise the run is refused;
// * if its writes are the same bits on the state and on both fills, they do
//   not depend on the state: the side becomes a fixed side with those values;
// * else it runs on the host at every ghost fill.  Its read depth is the
//   smallest D in 1, 2, 4, ... such that the routine writes the same bits
//   when every cell farther than D layers from the strip (across the whole
//   transverse extent) is replaced by -1e300 or by NaN; the library copies
//   the strip and those D layers to the host before each call.
bool Boundary::PrepareDevice(const TArray<Real>& cons, const Grid& grid,
                             const EquationOfState& eos, std::string* why) {
    static const char* names[6] = {"x left", "x right", "y left", "y right", "z left", "z right"};
    const BoundaryFunc* fn[6] = {&Bdxl, &Bdxr, &Bdyl, &Bdyr, &Bdzl, &Bdzr};
    for (int s = 0; s < 6; ++s) {
        deviceTypes_[s] = types_[s];
        hostDepth_[s] = 0;
    }
    deviceFixedSet_ = fixedEnrolled_;
    if (fixedEnrolled_) deviceFixed_ = fixedData_;
    const int sides = grid.nz > 1 ? 6 : 4;  // UpdateBD fills z sides in 3D only
    const Real fill[2] = {-1e300, std::numeric_limits<Real>::quiet_NaN()};
    for (int s = 0; s < sides; ++s) {
        if (!((custom_ >> s) & 1)) continue;
        const int dir = s / 2, side = s % 2;
        const int len[3] = {grid.lenx, grid.leny, grid.lenz};
        const int n[3] = {grid.nx, grid.ny, grid.nz};
        int lo[3] = {grid.ib, grid.jb, grid.kb}, hi[3] = {grid.ie, grid.je, grid.ke};
        lo[dir] = side == 0 ? 0 : grid.nGhost + n[dir];
        hi[dir] = side == 0 ? grid.nGhost : len[dir];
        auto inside = [&](int k, int j, int i) {
            return i >= lo[0] && i < hi[0] && j >= lo[1] && j < hi[1] && k >= lo[2] && k < hi[2];
        };
        // distance (in layers) of coordinate c along dir from the strip
        auto layers = [&](int c) {
            return side == 0 ? c - grid.nGhost + 1 : grid.nGhost + n[dir] - c;
        };
        auto coord = [&](int k, int j, int i) { return dir == 0 ? i : (dir == 1 ? j : k); };
        TArray<Real> probe[3] = {cons, cons, cons};
        for (int p = 1; p < 3; ++p) {
            Real* d = probe[p].data();
            for (size_t q = 0; q < probe[p].GetSize(); ++q) d[q] = fill[p - 1];
        }
        try {
            for (auto& a : probe) (*fn[s])(a, grid, eos);
        } catch (const std::exception& e) {
            *why = std::string("the self-defined ") + names[s] +
                   " boundary cannot be probed for the device (" + e.what() + ")";
            return false;
        }
        bool local = true, stationary = true;
        for (int v = 0; v < NVar; ++v)
            for (int k = 0; k < grid.lenz; ++k)
                for (int j = 0; j < grid.leny; ++j)
                    for (int i = 0; i < grid.lenx; ++i) {
                        const Real a = probe[0](v, k, j, i), b = probe[1](v, k, j, i),
                                   c = probe[2](v, k, j, i);
                        if (inside(k, j, i)) {
                            stationary = stationary && SameBits(a, b) && SameBits(a, c);
                        } else {
                            local = local && SameBits(a, cons(v, k, j, i)) && SameBits(b, fill[0]) &&
                                    SameBits(c, fill[1]);
                        }
                    }
        if (!local) {
            *why = std::string("the self-defined ") + names[s] +
                   " boundary writes outside its ghost strip; it runs on the host only";
            return false;
        }
        if (!stationary) {
            // the routine reads the state: find how far from its strip
            int depth = 0;
            for (int d = 1; depth == 0; d *= 2) {
                const int D = std::min(d, n[dir]);
                bool same = true;
                for (int f = 0; f < 2 && same; ++f) {
                    TArray<Real> q = cons;
                    for (int v = 0; v < NVar; ++v)
                        for (int k = 0; k < grid.lenz; ++k)
                            for (int j = 0; j < grid.leny; ++j)
                                for (int i = 0; i < grid.lenx; ++i)
                                    if (layers(coord(k, j, i)) > D) q(v, k, j, i) = fill[f];
                    (*fn[s])(q, grid, eos);
                    for (int v = 0; v < NVar && same; ++v)
                        for (int k = lo[2]; k < hi[2] && same; ++k)
                            for (int j = lo[1]; j < hi[1] && same; ++j)
                                for (int i = lo[0]; i < hi[0] && same; ++i)
                                    same = SameBits(q(v, k, j, i), probe[0](v, k, j, i));
                }
                if (same) depth = D;
                else if (D == n[dir]) depth = n[dir] + grid.nGhost;  // reads the far ghosts: all of it
            }
            hostDepth_[s] = depth;
            continue;
        }
        if (!deviceFixedSet_) {
            deviceFixed_.NewArray(NVar, grid.lenz, grid.leny, grid.lenx);
            deviceFixedSet_ = true;
        }
        for (int v = 0; v < NVar; ++v)
            for (int k = lo[2]; k < hi[2]; ++k)
                for (int j = lo[1]; j < hi[1]; ++j)
                    for (int i = lo[0]; i < hi[0]; ++i) deviceFixed_(v, k, j, i) = probe[0](v, k, j, i);
        deviceTypes_[s] = 4;
    }
    return true;
}

}  // namespace Gaukuk
