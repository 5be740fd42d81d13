// gaukuk.hpp -- core constants and ids of the Gaukuk host interface.
//
// Same names and values as the reference (src/gaukuk.hpp:1-25) so that
// problem hooks written for it compile unchanged: Real is double (the device
// path is FP64 only), the floors come from the same build-time macros, and
// PI keeps the reference's truncated value.
#pragma once

namespace Gaukuk {

using Real = double;

#ifndef GAUKUK_DENSITY_FLOOR
#define GAUKUK_DENSITY_FLOOR 1e-16
#endif
#ifndef GAUKUK_PRESSURE_FLOOR
#define GAUKUK_PRESSURE_FLOOR 1e-16
#endif

constexpr int NVar = 5;
constexpr Real PI = 3.1415926535;
constexpr Real DENSITY_FLOOR = GAUKUK_DENSITY_FLOOR;
constexpr Real PRESSURE_FLOOR = GAUKUK_PRESSURE_FLOOR;

enum ConsIDs { DEN = 0, MTX = 1, MTY = 2, MTZ = 3, ENG = 4 };
enum PrimIDs { VLX = 1, VLY = 2, VLZ = 3, PRE = 4 };

}  // namespace Gaukuk
