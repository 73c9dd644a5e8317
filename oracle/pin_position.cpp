// TEST INFRASTRUCTURE. Compiles the reference's own include/position.hpp (which
#include <cstdint>
// needs nothing outside the C++ standard library) into oracle/_ref/ so the
// oracle's restated Position::setXYZ / updateDelta can be checked against the
// reference's code on the same inputs, and its Position::getReferencePosition
// (the relay point of the EM current's zigzag). Built only where the reference sources
// are present; the GPU box uses the prebuilt library or skips the check.
#include "position.hpp"

extern "C" void ref_position(const double* xyz, int64_t n, int32_t* ijk, double* d) {
    for (int64_t t = 0; t < n; ++t) {
        Position p(xyz[3 * t], xyz[3 * t + 1], xyz[3 * t + 2]);
        ijk[3 * t] = p.i; ijk[3 * t + 1] = p.j; ijk[3 * t + 2] = p.k;
        d[6 * t + 0] = p.dx1; d[6 * t + 1] = p.dy1; d[6 * t + 2] = p.dz1;
        d[6 * t + 3] = p.dx2; d[6 * t + 4] = p.dy2; d[6 * t + 5] = p.dz2;
    }
}

// Position::getReferencePosition (include/position.hpp:88-96) of the new position
// relative to the old one, per pair.
extern "C" void ref_relay(const double* new_xyz, const double* old_xyz, int64_t n, double* out) {
    for (int64_t t = 0; t < n; ++t) {
        const Position nw(new_xyz[3 * t], new_xyz[3 * t + 1], new_xyz[3 * t + 2]);
        const Position od(old_xyz[3 * t], old_xyz[3 * t + 1], old_xyz[3 * t + 2]);
        const Position r = nw.getReferencePosition(od);
        out[3 * t] = r.x; out[3 * t + 1] = r.y; out[3 * t + 2] = r.z;
    }
}
