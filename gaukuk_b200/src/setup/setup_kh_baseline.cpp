// setup_kh_baseline.cpp -- Kelvin-Helmholtz problem of the benchmark configs.
//
// A problem hook in the reference's API (src/setup/setup_example.cpp:18-114):
// it defines Sim::Setup, fills the primitive variables on the active cells
// and converts them with eos.PrimToCons.  It includes "gaukuk.hpp" and
// "sim.hpp" through the include path, so the same file builds against this
// package's host layer (gaukuk_b200/src) and against the reference's headers.
//
// State on [xmin,xmax]x[ymin,ymax] (default [0,1]^2, periodic):
//   rho = rhoIn, vx = vxIn   where |y - yMid| < halfWidth, else rhoOut, vxOut
//   vy  = amp*sin(4*pi*x) + noise*U(-1,1),  p = pressure,  vz = 0
// U is a counter-based draw keyed on (seed, global cell id): SplitMix64
// (Steele, Lea & Flood 2014) of id ^ (seed * 0xD1B54A32D192ED03), top 53 bits.
#include <cmath>
#include <cstdint>

#include "gaukuk.hpp"
#include "sim.hpp"

namespace {

inline std::uint64_t SplitMix64(std::uint64_t x) {
    std::uint64_t z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

inline double UniformPm1(std::uint64_t seed, std::uint64_t id) {
    std::uint64_t bits = SplitMix64(id ^ (seed * 0xD1B54A32D192ED03ULL));
    double u01 = static_cast<double>(bits >> 11) * (1.0 / 9007199254740992.0);
    return 2.0 * u01 - 1.0;
}

}  // namespace

namespace Gaukuk {

void Sim::Setup() {
    Config& cfg = Config::getInstance();
    const Real rhoIn = cfg.get("rhoIn", 2.0);
    const Real rhoOut = cfg.get("rhoOut", 1.0);
    const Real vxIn = cfg.get("vxIn", -0.5);
    const Real vxOut = cfg.get("vxOut", 0.5);
    const Real pressure = cfg.get("pressure", 2.5);
    const Real amp = cfg.get("amp", 0.01);
    const Real noise = cfg.get("noise", 1e-3);
    const Real yMid = cfg.get("yMid", 0.5);
    const Real halfWidth = cfg.get("halfWidth", 0.25);
    const std::uint64_t seed = static_cast<std::uint64_t>(cfg.get("seed", 0));

    const long long nx = grid.nx, ny = grid.ny;
    for (int k = grid.kb; k < grid.ke; ++k) {
        for (int j = grid.jb; j < grid.je; ++j) {
            const Real y = domain.yc(j);
            const bool inside = std::abs(y - yMid) < halfWidth;
            for (int i = grid.ib; i < grid.ie; ++i) {
                const Real x = domain.xc(i);
                const std::uint64_t id = static_cast<std::uint64_t>(
                    ((k - grid.kb) * ny + (j - grid.jb)) * nx + (i - grid.ib));
                prim(DEN, k, j, i) = inside ? rhoIn : rhoOut;
                prim(VLX, k, j, i) = inside ? vxIn : vxOut;
                prim(VLY, k, j, i) = amp * std::sin(4.0 * PI * x) + noise * UniformPm1(seed, id);
                prim(VLZ, k, j, i) = 0.0;
                prim(PRE, k, j, i) = pressure;
            }
        }
    }
    eos.PrimToCons(prim, cons, grid);
}

}  // namespace Gaukuk
