// utils/write_sim.cpp -- Sim::WriteData, the reference's cons_/prim_ file
// format (src/utils/write_sim.cpp:14-58): int sizeof(Real), Real t,
// int NVar nx ny nz nGhost, the cell centres with ghosts, int size, then the
// whole array (ghosts and every z plane included).
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

}  // namespace Gaukuk
