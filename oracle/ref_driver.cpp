// ref_driver.cpp -- driver for the reference build (TEST INFRASTRUCTURE ONLY).
//
// Linked against the reference's own objects (everything in src/ except
// main.cpp) by oracle/Makefile.  It reproduces the output-cadence loop of
// main.cpp:44-52 and adds what the checker needs:
//   * the per-step "step = n, t = ..., dt = ..." lines that Sim::Advance
//     prints (sim.cpp:100-103) come out with 17 significant digits, because
//     the driver sets std::cout's precision before the run;
//   * --ic FILE replaces the state written by Sim::Setup with a raw
//     reference-layout array (NVar x lenz x leny x lenx doubles), so any
//     initial condition can be pushed through the reference unchanged;
//   * gravity can be enrolled from the .in keys gx, gy, gz
//     (SourceTerm::EnrollConstGravityVector, source.cpp:23-31);
//   * --out FILE writes the final state as a raw array; --frames writes the
//     reference's own cons_XXXXX files via Sim::WriteData;
//   * wall time spent inside Sim::Advance only (no setup, no I/O) is
//     reported as one JSON line on stderr, with the time at which each
//     per-step line was written (--step-times), so that the first steps,
//     which also page in the reference's arrays, can be left out.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "gaukuk.hpp"
#include "sim.hpp"

namespace {

// Forwards to std::cout's buffer and notes the time of every newline.
class StampBuf : public std::streambuf {
public:
    explicit StampBuf(std::streambuf* out) : out_(out) {}
    std::vector<double> stamps;

protected:
    int overflow(int c) override {
        if (c == traits_type::eof()) return out_->pubsync() == 0 ? 0 : traits_type::eof();
        if (c == '\n')
            stamps.push_back(std::chrono::duration<double>(
                                 std::chrono::steady_clock::now().time_since_epoch()).count());
        return out_->sputc(static_cast<char>(c));
    }
    int sync() override { return out_->pubsync(); }

private:
    std::streambuf* out_;
};

}  // namespace

#ifndef GK_DRIVER_HAS_SETUP
// The problem hook is empty unless a setup file is linked: the state comes
// from --ic.
void Gaukuk::Sim::Setup() {}
#endif

int main(int argc, char** argv) {
    using namespace Gaukuk;
    std::string infile, icfile, outfile;
    bool frames = false, quiet = false, step_times = false;
    double tmax_override = -1.0;
    for (int a = 1; a < argc; ++a) {
        std::string s = argv[a];
        if (s == "-i" && a + 1 < argc) infile = argv[++a];
        else if (s == "--ic" && a + 1 < argc) icfile = argv[++a];
        else if (s == "--out" && a + 1 < argc) outfile = argv[++a];
        else if (s == "--tmax" && a + 1 < argc) tmax_override = std::atof(argv[++a]);
        else if (s == "--frames") frames = true;
        else if (s == "--quiet") quiet = true;
        else if (s == "--step-times") step_times = true;
        else {
            std::cerr << "usage: " << argv[0]
                      << " -i input.in [--ic state.bin] [--out state.bin] [--tmax T] [--frames] [--quiet]\n";
            return 2;
        }
    }
    if (infile.empty()) { std::cerr << "missing -i\n"; return 2; }
    Config::getInstance().loadFromFile(infile);
    Real tmax = Config::getInstance().get("tmax");
    if (tmax_override > 0) tmax = tmax_override;
    Real dtoutput = Config::getInstance().get("dtoutput");
    if (dtoutput <= 0) dtoutput = tmax;

    Sim sim;
    sim.Setup();
    if (!icfile.empty()) {
        FILE* f = std::fopen(icfile.c_str(), "rb");
        if (!f) { std::cerr << "cannot open " << icfile << "\n"; return 3; }
        size_t n = sim.cons.GetSize();
        size_t got = std::fread(sim.cons.data(), sizeof(Real), n, f);
        std::fclose(f);
        if (got != n) { std::cerr << "short ic file\n"; return 3; }
    }
    Real gx = Config::getInstance().get("gx");
    Real gy = Config::getInstance().get("gy");
    Real gz = Config::getInstance().get("gz");
    if (gx != 0 || gy != 0 || gz != 0) sim.srcTerm.EnrollConstGravityVector(gx, gy, gz);

    std::cout.precision(17);
    std::streambuf* const original = std::cout.rdbuf();
    StampBuf stamp(original);
    if (step_times) std::cout.rdbuf(&stamp);
    if (quiet) std::cout.setstate(std::ios_base::failbit);

    int outputStep = 0;
    Real tnow = sim.GetTime();
    sim.boundary.UpdateBD(sim.cons, sim.grid, sim.domain, sim.eos);
    // the frame type of main.cpp:32-38 (dataType 1: primitives)
    const DataType outputType = static_cast<int>(Config::getInstance().get("dataType", 0)) == 1
                                    ? DataType::Prim
                                    : DataType::Cons;
    if (frames) sim.WriteData(outputStep, outputType);

    double seconds = 0.0;
    while (std::abs(tmax - tnow) > 1e-12 && sim.isContinue) {
        dtoutput = std::min(dtoutput, tmax - tnow);
        auto t0 = std::chrono::steady_clock::now();
        sim.Advance(dtoutput);
        auto t1 = std::chrono::steady_clock::now();
        seconds += std::chrono::duration<double>(t1 - t0).count();
        tnow = sim.GetTime();
        outputStep++;
        if (frames) sim.WriteData(outputStep, outputType);
    }
    std::cout.clear();
    std::cout.flush();
    std::cout.rdbuf(original);  // the stamping buffer dies with main()
    if (!outfile.empty()) {
        FILE* f = std::fopen(outfile.c_str(), "wb");
        if (!f) { std::cerr << "cannot open " << outfile << "\n"; return 3; }
        std::fwrite(sim.cons.data(), sizeof(Real), sim.cons.GetSize(), f);
        std::fclose(f);
    }
    long long cells = (long long)sim.grid.nx * sim.grid.ny * sim.grid.nz;
    std::string st = "[";
    for (size_t n = 0; n < stamp.stamps.size(); ++n) {
        char b[40];
        std::snprintf(b, sizeof(b), "%s%.6f", n ? ", " : "", stamp.stamps[n] - stamp.stamps[0]);
        st += b;
    }
    st += "]";
    std::fprintf(stderr,
                 "{\"steps\": %d, \"t\": %.17g, \"advance_seconds\": %.6f, \"cells\": %lld, "
                 "\"step_stamps\": %s}\n",
                 sim.GetStep(), (double)sim.GetTime(), seconds, cells, st.c_str());
    return 0;
}
