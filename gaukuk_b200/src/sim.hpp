// sim.hpp -- Sim, the problem object of the host interface.
//
// Public members and methods as in the reference (src/sim.hpp:23-58): a
// setup hook fills prim/cons using grid and domain and may enroll sources
// or boundaries; main drives Advance / WriteData.  Advance runs the whole
// time loop on the GPU through the C ABI of include/gaukuk_cuda.h: the state
// goes to the device at the start of the call and comes back at the end, so
// cons always holds the current state between calls.
//
// Keys beyond the reference's: gpuMode (0 = bit-identical to the reference
// built with strict IEEE flags, the default; 1 = fast mode, within 1e-12),
// gpuDevice (CUDA ordinal, default 0) and metrics (1: main appends one JSON
// line per output interval to metrics.jsonl, from LastAdvance()).
#pragma once

#include <cstddef>

#include "boundary/boundary.hpp"
#include "eos/eos.hpp"
#include "flux/flux.hpp"
#include "gaukuk.hpp"
#include "grid.hpp"
#include "source_term/source.hpp"
#include "template_array.hpp"

#include <cstddef>
#include <string>
#include <vector>

struct gk_handle;

namespace Gaukuk {

enum class DataType { Prim, Cons };

class Sim {
public:
    Sim();
    ~Sim();
    Sim(const Sim&) = delete;
    Sim& operator=(const Sim&) = delete;

    bool isContinue;
    const Grid grid;
    const Domain domain;
    Flux flux;

    TArray<Real> cons, prim;
    // Face fluxes live on the device; these stay unallocated.
    TArray<Real> flx1, flx2, flx3;

    EquationOfState eos;
    Boundary boundary;
    SourceTerm srcTerm;

    void Setup();
    void Advance(Real dtoutput);
    void WriteData(const int outputID, DataType dType);
    // Restart: loads time and conserved state from the frame cons_<outputID>
    // that WriteData wrote (the grid must match); the step counter restarts
    // at 0, since frames do not carry it.
    void ReadData(const int outputID);

    Real GetTime() { return t; }
    Real Getdt() { return dt; }
    int GetStep() { return step; }

    // What the last Advance did: steps, host wall time around the device
    // call (upload, steps, download), the smallest and largest dt, and the
    // cells the floors repaired (density, pressure).
    struct AdvanceStats {
        int steps = 0;
        double seconds = 0, dt_min = 0, dt_max = 0;
        unsigned long long floor_density = 0, floor_pressure = 0;
    };
    const AdvanceStats& LastAdvance() const { return last_; }

private:
    int step, stepMax;
    Real t, dt, dtUntilOutput, cmax, CFL;
    int rcOrder, integratorType;
    int gpuMode_, gpuDevice_;
    gk_handle* dev_ = nullptr;
    AdvanceStats last_;
    void EnsureDevice();
    // Cells that no ghost fill or update writes (corner and edge ghosts,
    // ghost rows of unused directions) and consTemp's values of them.
    std::vector<size_t> unwritten_;
    std::vector<Real> spare_;
    void SwapUnwritten();
    // Self-defined sides that depend on the state run on the host at every
    // ghost fill (gk_set_host_fill): the library calls HostFill with one of
    // these, on cons.
    struct HostSide {
        Sim* sim;
        int side;
    };
    HostSide hostSides_[6];
    std::string hostFillError_;  // what a host-run side threw, rethrown by Advance
    static int HostFill(void* user, double* cons);
};

}  // namespace Gaukuk
