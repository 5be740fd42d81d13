// main.cpp -- gaukuk.sim, the command-line driver, with the reference's
// interface and output cadence (src/main.cpp:12-65):
//     gaukuk.sim -i input.in
// Setup hook -> ghost fill -> frame 0 -> {Advance(dtoutput); frame n} until
// tmax, then the step count and timings.  An input key `restart = N` (not in
// the reference) resumes from the frame cons_N instead of frame 0: the setup
// hook still runs (it enrolls sources and boundaries), then the frame's time
// and state replace its initial state and frames N+1, ... follow.  With
// `metrics = 1` each output interval also appends one JSON line to
// metrics.jsonl (steps, wall time, zone-updates/s, dt range, floor repairs).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>

#include "gaukuk.hpp"
#include "sim.hpp"

int main(int argc, char* argv[]) {
    using namespace Gaukuk;
    if (argc < 3 || std::string(argv[1]) != "-i") {
        std::cerr << "Usage: " << argv[0] << " -i input.in" << std::endl;
        return 1;
    }
    Config::getInstance().loadFromFile(argv[2]);
    Real tmax = Config::getInstance().get("tmax");
    Real dtoutput = Config::getInstance().get("dtoutput");

    Sim sim;
    sim.Setup();
    int outputStep = 0;
    const int restart = static_cast<int>(Config::getInstance().get("restart", -1));
    if (restart >= 0) {
        sim.ReadData(restart);
        outputStep = restart;
    }
    Real tnow = sim.GetTime();
    sim.boundary.UpdateBD(sim.cons, sim.grid, sim.domain, sim.eos);
    DataType outputType = DataType::Cons;
    if (static_cast<int>(Config::getInstance().get("dataType")) == 1) outputType = DataType::Prim;
    if (restart < 0) sim.WriteData(outputStep, outputType);

    const bool metrics = Config::getInstance().get("metrics", 0) != 0;
    std::ofstream mlog;
    if (metrics) mlog.open("metrics.jsonl", std::ios::app);
    const double cells = double(sim.grid.nx) * sim.grid.ny * sim.grid.nz;

    auto time0 = std::chrono::high_resolution_clock::now();
    clock_t cpu0 = clock();
    while (std::abs(tmax - tnow) > 1e-12 && sim.isContinue) {
        dtoutput = std::min(dtoutput, tmax - tnow);
        sim.Advance(dtoutput);
        tnow = sim.GetTime();
        outputStep++;
        sim.WriteData(outputStep, outputType);
        std::cout << "output " << outputStep << std::endl;
        if (metrics) {
            const Sim::AdvanceStats& a = sim.LastAdvance();
            mlog << std::setprecision(17) << "{\"output\": " << outputStep << ", \"t\": " << tnow
                 << ", \"step\": " << sim.GetStep() << ", \"steps\": " << a.steps
                 << ", \"seconds\": " << a.seconds << ", \"zone_updates_per_s\": "
                 << (a.seconds > 0 ? cells * a.steps / a.seconds : 0.0) << ", \"dt_min\": "
                 << a.dt_min << ", \"dt_max\": " << a.dt_max << ", \"floor_density\": "
                 << a.floor_density << ", \"floor_pressure\": " << a.floor_pressure << "}"
                 << std::endl;
        }
    }
    auto time1 = std::chrono::high_resolution_clock::now();
    clock_t cpu1 = clock();
    Real wall = std::chrono::duration<Real>(time1 - time0).count();
    Real cpu = double(cpu1 - cpu0) / CLOCKS_PER_SEC;
    std::cout << std::right << "Finish! "
              << "\n    total steps = " << std::setw(6) << sim.GetStep()
              << " , \n    walltime = " << std::setw(8) << std::fixed << std::setprecision(3) << wall
              << " s, \n    cputime = " << std::setw(8) << std::fixed << std::setprecision(3) << cpu
              << " s"
              << "\n-----------------------------------------------------------" << std::endl;
    return 0;
}
