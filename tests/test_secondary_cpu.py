"""CPU tests of the secondary-emission and dielectric-surface path:

* the .obj face textures per surface node (ObjectDataFromFile::textures,
  src/Spacecraft/ObjectUtils.cpp:65-160) and the dielectric capacitance map
  built from them (Spacecraft::construct, src/Spacecraft/Spacecraft.cpp:117-149);
* the oracle's secondary emission (Spacecraft::emitParticles' secondary branch,
  Spacecraft.cpp:901-937, SecondaryParticleType::generateNewParticles and
  Whipple's coefficients, src/Particle/SecondaryParticleType.cpp:16-194) against a
  line-by-line Python restatement on the same Philox draws.
None of these touch a GPU."""
import math

import numpy as np
import pytest

import oracle as orc
from fopis_b200 import _abi, config
from fopis_b200.config import SpeciesInfo, make_params, plasma_units


def obj_file(tmp_path, text):
    p = tmp_path / "body.obj"
    p.write_text(text)
    return str(p)


def test_textures_per_node_follow_the_quads(tmp_path):
    text = config.box_obj_text([((-2, -2, -2), (2, 2, 2))])
    # texture 2 on the +x face (normal index 2), texture 1 elsewhere
    text = "\n".join(l.replace("/1/2", "/2/2") if l.startswith("f ") else l for l in text.splitlines()) + "\n"
    path = obj_file(tmp_path, text)
    nodes, _ = config.parse_obj(path, 25, 25, 25)
    tex = config.parse_obj_textures(path, 25, 25, 25)
    assert len(tex) == len(nodes)
    lo, hi = 10 + 1, 14 + 1            # glue node indices of the cube's faces
    for (i, j, k), t in zip(nodes, tex):
        on = sum(int(v in (lo, hi)) for v in (i, j, k))     # faces the node lies on
        assert len(t) == on, ((i, j, k), t)
        assert t.count(2) == int(i == hi)
    # capacitance: mean over the node's quads of normalizeCapacitance(4 pi eps0 eps_r)
    dx, dt = plasma_units()
    norm = config.Normalizer(dx, dt)
    cap = config.node_capacitance(tex, {1: "Teflon", 2: "Aluminum"}, norm)
    unit = 4.0 * math.pi * config.EPS0 * norm.V_unit / config.E
    for (i, j, k), t, c in zip(nodes, tex, cap):
        want = unit * sum(2.1 if q == 1 else 9.5 for q in t) / len(t)
        assert abs(c - want) <= 1e-15 * want
    with pytest.raises(ValueError, match="Invalid material name"):
        config.node_capacitance(tex, {1: "Teflon"}, norm)


# ---------------------------------------------------------------- secondary emission
FERMI, DMAX, EMAX, Z = 9.1, 3.0, 420.0, 13.0


def py_draw2(seed, c):
    r = orc.philox(c, [seed & 0xFFFFFFFF, seed >> 32])
    x = (r[0] << 32) | r[1]
    y = (r[2] << 32) | r[3]
    return (x >> 11) * 2.0 ** -53, (y >> 11) * 2.0 ** -53


def py_key(rec):
    obj, s, ax = (int(v) for v in rec[:3])
    h = 0xCBF29CE484222325
    M = (1 << 64) - 1

    def mix(h, w):
        h ^= w & M
        h = (h * 0x100000001B3) & M
        return h ^ (h >> 29)

    for v in rec[4:10]:
        h = mix(h, int(np.rint(v * 16777216.0)) & M)
    return mix(h, s | (ax << 8) | (obj << 16))


def py_secondaries(p, rec, sec, step):
    """SecondaryParticleType::generateNewParticles for one incident record."""
    obj, s, ax = (int(v) for v in rec[:3])
    trem, cp, vin = rec[3], rec[4:7], rec[7:10]
    key = py_key(rec)
    draw = lambda i: py_draw2(p.seed, [key & 0xFFFFFFFF, key >> 32, step, (4 << 24) | i])
    m_in, q_in = p.species[s].mass, p.species[s].charge
    v2 = float(np.dot(vin, vin))
    E = 0.5 * m_in * v2 * p.energy_ev
    th = math.acos(abs(vin[ax]) / math.sqrt(v2))
    r = eta = 0.0
    if q_in < 0:
        r = (1 / 13.54) * FERMI ** 4 / (16.0 * ((E + FERMI) ** 3 + FERMI ** 3))
        eta1 = 1 - (2 / E) ** (0.037 * Z)
        eta2 = 0.1 * math.exp(-E / 5000.0)
        eta0 = math.log(E / 50.0) / math.log(20.0) if 50 < E < 1000 else (1.0 if E > 1000 else 0.0)
        eta = eta0 * (eta1 + eta2) * (7.37 * Z ** -0.56875) * (1 - math.cos(th))
    delta = (1.114 * DMAX / math.cos(th)) * (EMAX / E) ** 0.35 * (1 - math.exp(-2.28 * math.cos(th) * (E / EMAX) ** 1.35))
    u = draw(0)
    if u[0] < r:
        kind, count = 1, 1
    elif u[0] < r + eta:
        kind, count = 2, 1
    else:
        d = delta / (1 - r - eta)
        kind, count = 3, int(math.floor(d)) + (1 if u[1] < d - math.floor(d) else 0)
    speed = p.species[sec].thermal_velocity
    if kind == 2:
        speed = math.sqrt(2 * (draw(1)[0] * 0.5 * m_in * v2) / p.species[sec].mass)
    out = []
    for m in range(count):
        v = list(vin)
        if kind == 1:
            v[ax] = -v[ax]
        else:
            a, b = draw(2 + m)
            dep, az = math.asin(2 * a - 1), 2 * math.pi * b
            sgn = -1.0 if vin[ax] > 0 else 1.0
            cn, sa, sb = speed * math.cos(dep) * sgn, speed * math.sin(dep) * math.cos(az), speed * math.sin(dep) * math.sin(az)
            v = [cn, sa, sb] if ax == 0 else ([sb, cn, sa] if ax == 1 else [sa, sb, cn])
        out.append([cp[q] + trem * v[q] for q in range(3)] + v)
    return kind, out


def secondary_cfg(n=25):
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, 2),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, 2),
          SpeciesInfo("Secondary", "secondary", 1.0, -1.0, 1e7, 2.0, 2)]
    p, norm = make_params((n, n, n), "DDDDDD", dx, dt, sp, tol=1e-10, sort_interval=1000000)
    obj = config.objects_from_boxes([((-2, -2, -2), (2, 2, 2))], (n, n, n), obj_parser=orc.parse_obj)
    obj.secondary_species = 2
    return config.SimConfig(params=p, norm=norm, species=sp, objects=[obj])


def incident_records(energy_ev, seed=5, count=400):
    """Hits on the six faces of the cube [10, 14]^3 with energies of 1-45 eV and, for
    the inelastic branch (E > 50 eV, 1 - cos(theta)), grazing electrons of 55-90 eV
    whose remaining time is at least 0.3: every secondary's back-dated position then
    lies within one cell of the face it leaves, as the reference's getCmatNumber
    requires of the nodes it charges."""
    rng = np.random.default_rng(seed)
    recs = []
    for t in range(count):
        s = 0 if t % 4 else 1
        ax = t % 3
        side = (t // 3) % 2                  # 0: the low face, hit moving +; 1: the high face, hit moving -
        cp = rng.uniform(10.05, 13.95, 3)
        cp[ax] = 10.0 if side == 0 else 14.0
        grazing = s == 0 and t % 8 == 1                # inelastic backscatter needs E > 50 eV and 1 - cos(theta)
        e_ev = rng.uniform(55.0, 90.0) if grazing else 10 ** rng.uniform(0, math.log10(45.0))
        m = 1.0 if s == 0 else 100.0
        speed = math.sqrt(2 * e_ev / energy_ev / m)
        dirv = rng.normal(size=3)
        dirv[ax] = 0.0
        dirv /= np.linalg.norm(dirv)
        cn = rng.uniform(0.1, 0.3) if grazing else rng.uniform(0.2, 1.0)
        dirv = cn * np.eye(3)[ax] + math.sqrt(1 - cn * cn) * dirv
        v = speed * dirv
        v[ax] = abs(v[ax]) * (1 if side == 0 else -1)
        recs.append([0, s, ax, rng.uniform(0.3 if grazing else 0.0, 1.0), *cp, *v])
    return np.array(recs)


def test_oracle_secondaries_match_restatement():
    cfg = secondary_cfg()
    p = cfg.params
    o = orc.Oracle(p, cfg.objects)
    o.set_cmatrix(0, np.eye(len(cfg.objects[0].nodes)))
    recs = incident_records(p.energy_ev)
    o.set_incidents(recs)
    assert np.array_equal(o.get_incidents(), recs)
    o.timestep = 7
    assert o.emit() == 0
    assert len(o.get_incidents()) == 0              # clearIncidentEvents
    got = o.particles(2)
    got = np.stack([got[k] for k in ("x", "y", "z", "vx", "vy", "vz")], 1)
    kinds = {1: 0, 2: 0, 3: 0}
    want, inside = [], 0
    cells = {tuple(c) for c in cfg.objects[0].cells}
    for rec in recs:
        kind, parts = py_secondaries(p, rec, 2, 7)
        kinds[kind] += 1
        for q in parts:
            pos = tuple(int(math.floor(c)) + 1 for c in q[:3])
            if pos in cells:
                inside += 1                            # absorbed at once, not appended
            else:
                want.append(q)
    want = np.array(want)
    assert kinds[1] > 0 and kinds[2] > 0 and kinds[3] > 0, kinds
    assert len(got) == len(want) and len(got) > 100
    assert np.allclose(got, want, rtol=0, atol=1e-12)
    # charge: each emitted secondary leaves -q on the surface, each absorbed one +q
    _, _, cur = o.get_object(0)
    q = p.species[2].charge * p.species[2].size
    assert cur[2] == pytest.approx(q * (inside - len(want)), rel=1e-12)
    print(f"\nsecondaries: {kinds} incidents by kind, {len(want)} emitted, {inside} absorbed at once")
