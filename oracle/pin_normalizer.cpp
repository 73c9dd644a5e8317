// TEST INFRASTRUCTURE. Compiles the reference's own Normalizer
// (include/normalizer.hpp with its static members from src/Misc/Normalizer.cpp,
// and the physical constants of include/global.hpp) into oracle/_ref/, so the
// product's unit conversions can be checked against the reference's code on the
// same dx and dt. Boost is absent here: oracle/pin_stub holds declaration-only
// stand-ins for the two Boost headers that global.hpp includes and the
// Normalizer does not use. Built only where the reference sources are present.
#include <cstdint>
#include <string>

#include "normalizer.hpp"

namespace {

// Initializer::initTDPIC's unit set-up (src/Misc/Initialize.cpp:33-36).
struct Units : Normalizer {
    static void set(double dx, double dt) {
        Normalizer::setLengthUnit(dx);
        Normalizer::setTimeUnit(dt);
        Normalizer::setMassUnit(me);
        Normalizer::setChargeUnit(e);
    }
};

}  // namespace

// The normalised constants and unit factors after the set-up, in this order:
// eps0, mu0, c, unnormalizePotential(1), unnormalizeCurrent(1),
// normalizeVelocity(1), normalizeBfield(1), normalizeCurrentDensity(1),
// normalizeDensity(1), unnormalizeEnergy(1), unnormalizeEnergy(1, "eV"),
// normalizeCapacitance(1). Returns the number written (at most n).
extern "C" int ref_normalizer_units(double dx, double dt, double* out, int n) {
    Units::set(dx, dt);
    const double v[12] = {Normalizer::eps0,
                          Normalizer::mu0,
                          Normalizer::c,
                          Normalizer::unnormalizePotential(1.0),
                          Normalizer::unnormalizeCurrent(1.0),
                          Normalizer::normalizeVelocity(1.0),
                          Normalizer::normalizeBfield(1.0),
                          Normalizer::normalizeCurrentDensity(1.0),
                          Normalizer::normalizeDensity(1.0),
                          Normalizer::unnormalizeEnergy(1.0),
                          Normalizer::unnormalizeEnergy(1.0, std::string("eV")),
                          Normalizer::normalizeCapacitance(1.0)};
    const int m = n < 12 ? n : 12;
    for (int t = 0; t < m; ++t) out[t] = v[t];
    return m;
}

// One conversion applied to n values: 0 normalizeVelocity, 1 unnormalizeVelocity,
// 2 normalizePotential, 3 unnormalizePotential, 4 normalizeCurrentDensity,
// 5 unnormalizeCurrent, 6 unnormalizeCharge, 7 unnormalizeEnergy,
// 8 normalizeCapacitance, 9 normalizeDensity, 10 normalizeBfield.
// Returns 0, or -1 for an unknown kind.
extern "C" int ref_normalizer_apply(double dx, double dt, int kind, const double* in, int64_t n, double* out) {
    Units::set(dx, dt);
    for (int64_t t = 0; t < n; ++t) {
        const double x = in[t];
        switch (kind) {
            case 0: out[t] = Normalizer::normalizeVelocity(x); break;
            case 1: out[t] = Normalizer::unnormalizeVelocity(x); break;
            case 2: out[t] = Normalizer::normalizePotential(x); break;
            case 3: out[t] = Normalizer::unnormalizePotential(x); break;
            case 4: out[t] = Normalizer::normalizeCurrentDensity(x); break;
            case 5: out[t] = Normalizer::unnormalizeCurrent(x); break;
            case 6: out[t] = Normalizer::unnormalizeCharge(x); break;
            case 7: out[t] = Normalizer::unnormalizeEnergy(x); break;
            case 8: out[t] = Normalizer::normalizeCapacitance(x); break;
            case 9: out[t] = Normalizer::normalizeDensity(x); break;
            case 10: out[t] = Normalizer::normalizeBfield(x); break;
            default: return -1;
        }
    }
    return 0;
}
