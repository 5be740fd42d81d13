// flux/flux.hpp -- placeholder of the reference's Flux member of Sim
// (src/flux/flux.hpp:14-26).  The flux computation itself runs on the
// device; the object keeps Sim's member list source compatible.
#pragma once

namespace Gaukuk {

class Flux {
public:
    explicit Flux(const int lenx) : lenUlUr(lenx + 1) {}
    int FaceBufferLength() const { return lenUlUr; }

private:
    const int lenUlUr;
};

}  // namespace Gaukuk
