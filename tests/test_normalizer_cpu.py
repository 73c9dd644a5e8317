"""The product's unit conversions (fopis_b200.config.Normalizer and the factors
make_params derives from it) against the reference's own Normalizer
(include/normalizer.hpp, src/Misc/Normalizer.cpp) compiled into oracle/_ref/,
bit for bit. The C++ host loader gives the Python loader's parameters byte for
byte (tests/test_host_cpp.py), so this pins both."""
import math

import numpy as np
import pytest

from fopis_b200 import config
import oracle as orc

pytestmark = pytest.mark.skipif(not orc.REF_NORM.exists(),
                                reason="oracle/_ref was not built (reference sources absent)")


def _cases():
    rng = np.random.default_rng(7)
    dx0, dt0 = config.plasma_units()
    fixed = [(dx0, dt0), (0.5, 1e-8), (0.1, 2e-9), (1.0, 1e-9), (0.5, 0.999 * 0.5 / config.CLIGHT)]
    return fixed + [(float(10 ** rng.uniform(-3, 1)), float(10 ** rng.uniform(-10, -6))) for _ in range(400)]


def test_unit_factors_match_reference():
    for dx, dt in _cases():
        ref = orc.ref_normalizer_units(dx, dt)
        n = config.Normalizer(dx, dt)
        mine = {"eps0": n.eps0, "mu0": n.mu0, "c": n.c, "V_unit": n.V_unit, "A_unit": n.A_unit,
                "velocity": n.velocity(1.0), "bfield": n.bfield(1.0), "current_density": n.current_density(1.0),
                "density": 1.0 * n.x_pow_3, "energy": n.unenergy(1.0), "energy_ev": n.unenergy_ev(1.0)}
        for k, v in mine.items():
            assert v == ref[k], (k, dx, dt, v, ref[k])


@pytest.mark.parametrize("kind", ["velocity", "unvelocity", "potential", "unpotential", "current_density",
                                  "uncurrent", "uncharge", "unenergy", "bfield"])
def test_conversions_match_reference(kind):
    rng = np.random.default_rng(11)
    vals = np.concatenate([10 ** rng.uniform(-12, 12, 300) * rng.choice([-1.0, 1.0], 300), [0.0, 1.0, -1.0]])
    for dx, dt in _cases()[:40]:
        n = config.Normalizer(dx, dt)
        f = getattr(n, kind)
        want = orc.ref_normalizer_apply(dx, dt, kind, vals)
        got = np.array([f(float(v)) for v in vals])
        assert np.array_equal(got, want), (kind, dx, dt)


def test_make_params_factors_match_reference():
    """eps0, mu0, the static field in nT, the drift in km/s, the eV energy factor and
    the species velocities as Initializer and ParticleType form them
    (Initialize.cpp:314-318, :353-355; ParticleType.cpp:49-55)."""
    dx, dt = config.plasma_units()
    sp = [config.SpeciesInfo("electron", "ambient", 1.0, -1.0, 1e12, 10.0, 8, drift_kms=(400.0, -3.0, 7.5)),
          config.SpeciesInfo("ion", "ambient", 1836.0, 1.0, 1e12, 1.0, 8, drift_kms=(400.0, -3.0, 7.5))]
    bnt = (5.0, -3.0, 1.7)
    p, norm = config.make_params((8, 8, 8), "DDDDDD", dx, dt, sp, bfield_nT=bnt)
    ref = orc.ref_normalizer_units(dx, dt)
    assert p.eps0 == ref["eps0"] and p.mu0 == ref["mu0"] and p.energy_ev == ref["energy_ev"]
    for a in range(3):
        assert p.static_bfield[a] == bnt[a] * (ref["bfield"] * 1e-9)
    by_name = {s.name: s for s in sp}
    for i in range(p.nspecies):
        s = p.species[i]
        info = [q for q in by_name.values() if q.mass == s.mass][0]
        for a in range(3):
            assert s.drift[a] == info.drift_kms[a] * (1e3 * ref["velocity"])
        T = config.E * info.temperature
        vth = orc.ref_normalizer_apply(dx, dt, "velocity", np.array([math.sqrt(2.0 * T / (info.mass * config.ME))]))
        dev = orc.ref_normalizer_apply(dx, dt, "velocity", np.array([math.sqrt(T / (info.mass * config.ME))]))
        assert s.thermal_velocity == vth[0] and s.deviation == dev[0]
