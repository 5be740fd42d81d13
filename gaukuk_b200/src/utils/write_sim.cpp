// utils/write_sim.cpp -- Sim::WriteData, the reference's cons_/prim_ file
// format (src/utils/write_sim.cpp:14-58): int sizeof(Real), Real t,
// int NVar nx ny nz nGhost, the cell centres with ghosts, int size, then the
// whole array (ghosts and every z plane included).  Sim::ReadData reads a
// cons_ frame back for a restart (the reference has no restart; its reader
// is pypkg/read_gaukuk.py:3-44).
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>
#include <string>

#include "../sim.hpp"

namespace Gaukuk {

void Sim::WriteData(const int outputID, DataType dType) {
    std::ostringstream name;
    name << (dType == DataType::Prim ? "prim_" : "cons_") << std::setw(5) << std::setfill('0')
         << outputID;
    std::ofstream out(name.str(), std::ios::binary);
    if (!out) throw std::runtime_error("Failed to open " + name.str());
    auto put = [&](const void* p, size_t n) { out.write(reinterpret_cast<const char*>(p), n); };
    const int realSize = sizeof(Real);
    put(&realSize, sizeof(int));
    put(&t, sizeof(Real));
    put(&NVar, sizeof(int));
    put(&grid.nx, sizeof(int));
    put(&grid.ny, sizeof(int));
    put(&grid.nz, sizeof(int));
    put(&grid.nGhost, sizeof(int));
    put(domain.xc.data(), domain.xc.GetSizeInBytes());
    put(domain.yc.data(), domain.yc.GetSizeInBytes());
    put(domain.zc.data(), domain.zc.GetSizeInBytes());
    const TArray<Real>* arr = &cons;
    if (dType == DataType::Prim) {
        eos.ConsToPrim(cons, prim, grid);
        arr = &prim;
    }
    const int size = static_cast<int>(arr->GetSize());
    put(&size, sizeof(int));
    put(arr->data(), arr->GetSizeInBytes());
}

void Sim::ReadData(const int outputID) {
    std::ostringstream name;
    name << "cons_" << std::setw(5) << std::setfill('0') << outputID;
    std::ifstream in(name.str(), std::ios::binary);
    if (!in) throw std::runtime_error("Failed to open " + name.str() + " for the restart");
    auto get = [&](void* p, size_t n) {
        in.read(reinterpret_cast<char*>(p), n);
        if (!in) throw std::runtime_error("Truncated frame " + name.str());
    };
    int realSize = 0, nvar = 0, nx = 0, ny = 0, nz = 0, ng = 0;
    Real tFile = 0;
    get(&realSize, sizeof(int));
    if (realSize != static_cast<int>(sizeof(Real)))
        throw std::runtime_error(name.str() + ": written with another floating-point size");
    get(&tFile, sizeof(Real));
    get(&nvar, sizeof(int));
    get(&nx, sizeof(int));
    get(&ny, sizeof(int));
    get(&nz, sizeof(int));
    get(&ng, sizeof(int));
    if (nvar != NVar || nx != grid.nx || ny != grid.ny || nz != grid.nz || ng != grid.nGhost)
        throw std::invalid_argument(name.str() + ": its grid differs from the input file's");
    // cell centres: recomputed from the input file, so only skipped
    in.seekg(static_cast<std::streamoff>(domain.xc.GetSizeInBytes() + domain.yc.GetSizeInBytes() +
                                         domain.zc.GetSizeInBytes()),
             std::ios::cur);
    int size = 0;
    get(&size, sizeof(int));
    if (size != static_cast<int>(cons.GetSize()))
        throw std::runtime_error(name.str() + ": array size differs from the grid's");
    get(cons.data(), cons.GetSizeInBytes());
    t = tFile;
    step = 0;
    isContinue = true;
}

}  // namespace Gaukuk
