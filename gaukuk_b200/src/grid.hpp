// grid.hpp -- index ranges (Grid) and geometry (Domain) of the host interface.
//
// Members and friendships as in the reference (src/grid.hpp:11-56): setup
// hooks, being Sim members, read domain.xmin, domain.xc(i), grid.ib, ...
#pragma once

#include <stdexcept>

#include "template_array.hpp"
#include "utils/utils.hpp"

namespace Gaukuk {

class Grid {
public:
    friend class Sim;
    int nx, ny, nz, nGhost, lenx, leny, lenz, lenArr;
    int igb, ige, jgb, jge, kgb, kge;  // ghost-inclusive ranges [b, e)
    int ib, ie, jb, je, kb, ke;        // active ranges [b, e)

    Grid() {
        Config& c = Config::getInstance();
        nx = static_cast<int>(c.get("NX"));
        ny = static_cast<int>(c.get("NY"));
        nz = static_cast<int>(c.get("NZ"));
        nGhost = static_cast<int>(c.get("NGhost"));
        if (nx <= 0 || ny <= 0 || nz <= 0 || nGhost < 0)
            throw std::runtime_error("Invalid grid parameters from config");
        lenx = nx + 2 * nGhost;
        leny = ny + 2 * nGhost;
        lenz = nz + 2 * nGhost;
        lenArr = lenx * leny * lenz;
        igb = jgb = kgb = 0;
        ige = lenx;
        jge = leny;
        kge = lenz;
        ib = nGhost; ie = ib + nx;
        jb = nGhost; je = jb + ny;
        kb = nGhost; ke = kb + nz;
    }
};

class Domain {
public:
    friend class Sim;
    friend class SourceTerm;
    friend class Boundary;
    explicit Domain(const Grid& grid);

private:
    Real xmin, xmax, ymin, ymax, zmin, zmax;
    Real dx, dy, dz, drmin;
    Real dxRec, dyRec, dzRec;
    TArray<Real> xc, yc, zc;  // cell centres, ghosts included
};

}  // namespace Gaukuk
