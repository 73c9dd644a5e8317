"""CPU tests of the EM mode (RootGrid::mainLoopEM, src/Grid/RootGrid/RootGrid.cpp:145-191)
in the oracle and the host-side set-up:

* the Courant check of Environment::checkCFLCondition (src/Misc/Environment.cpp:193-203)
  and the normalised mu0 (include/normalizer.hpp:219-221);
* the Yee arrays' index bases and extents with the damping layers of
  RootGrid::initializeField (src/Grid/RootGrid/RootGridField.cpp:7-39);
* the charge-conserving current of Particle::distributeCurrentAtOldPosition /
  AtNewPosition (src/Particle/particle.cpp:258-338): against a line-by-line Python
  restatement on a few particles, and the continuity equation
  rho^{n+1} - rho^n + div J = 0 at every node over a whole particle set (the
  reference's own check, Field::checkChargeConservation, src/Grid/Field.cpp:236-263);
* one FDTD E and B update with damping (RootGridField.cpp:594-820) against an
  independent vectorised numpy restatement, on D and P boxes.
None of these touch a GPU."""
import math

import numpy as np
import pytest

import oracle as orc
from fopis_b200 import _abi, config
from fopis_b200.config import SpeciesInfo, make_params

from helpers import em_config, random_particles


def test_courant_check_and_mu0():
    dx, dt = config.plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, 2)]
    with pytest.raises(ValueError, match="Courant number exceeds 1.0"):
        make_params((9, 9, 9), "DDDDDD", dx, dt, sp, solver="EM")
    make_params((9, 9, 9), "DDDDDD", dx, dt, sp, solver="ES")          # ES runs have no such limit
    with pytest.raises(ValueError, match="neither ES nor EM"):
        make_params((9, 9, 9), "DDDDDD", dx, dt, sp, solver="FDTD")
    cfg = em_config()
    p = cfg.params
    assert p.solver == _abi.SOLVER_EM
    assert p.mu0 == pytest.approx(config.MU0 * config.E ** 2 / (config.ME * cfg.dx), rel=1e-15)
    assert 1.0 / math.sqrt(p.eps0 * p.mu0) == pytest.approx(0.5, rel=1e-8)   # c dt / dx


@pytest.mark.parametrize("boundary", ["DDDDDD", "PPDDPP", "PPPPPP", "NDPPDD"])
def test_yee_extents(boundary):
    cfg = em_config(n=7, boundary=boundary)
    o = orc.Oracle(cfg.params)
    c = (9, 9, 9)
    lo = [0 if boundary[2 * a] == "P" else -7 for a in range(3)]
    up = [c[a] if boundary[2 * a + 1] == "P" else c[a] + 7 for a in range(3)]
    shrink = {32: (1, 0, 0), 33: (0, 1, 0), 34: (0, 0, 1), 35: (0, 1, 1), 36: (1, 0, 1), 37: (1, 1, 0)}
    for which, s in shrink.items():
        got_lo, got_n = o.field_shape(which)
        assert got_lo == tuple(lo)
        assert got_n == tuple(up[a] - s[a] - lo[a] for a in range(3)), (which, got_n)
    for d, which in enumerate((38, 39, 40)):
        assert o.field_shape(which) == ((0, 0, 0), tuple(c[a] - (a == d) for a in range(3)))
    o.close()


# ---------------------------------------------------------------- currents
def py_current(params, recs, shape):
    """Particle::distributeCurrentAtOldPosition / AtNewPosition restated line by
    line for particles that stay inside a D/N box (no boundary crossing)."""
    cx, cy, cz = shape
    jx = np.zeros((cx - 1, cy, cz))
    jy = np.zeros((cx, cy - 1, cz))
    jz = np.zeros((cx, cy, cz - 1))

    def cell(x):
        return int(math.floor(x)) + 1

    def relay(xn, xo):
        i_n, i_o = cell(xn), cell(xo)
        return min(float(min(i_n, i_o)), max(float(max(i_n, i_o)) - 1.0, 0.5 * (xn + xo)))

    def deposit(at, f, w):
        i, j, k = (cell(v) for v in at)
        jx[i, j, k] += f[0] * (1.0 - w[1]) * (1.0 - w[2])
        jx[i, j + 1, k] += f[0] * w[1] * (1.0 - w[2])
        jx[i, j, k + 1] += f[0] * (1.0 - w[1]) * w[2]
        jx[i, j + 1, k + 1] += f[0] * w[1] * w[2]
        jy[i, j, k] += f[1] * (1.0 - w[0]) * (1.0 - w[2])
        jy[i + 1, j, k] += f[1] * w[0] * (1.0 - w[2])
        jy[i, j, k + 1] += f[1] * (1.0 - w[0]) * w[2]
        jy[i + 1, j, k + 1] += f[1] * w[0] * w[2]
        jz[i, j, k] += f[2] * (1.0 - w[0]) * (1.0 - w[1])
        jz[i + 1, j, k] += f[2] * w[0] * (1.0 - w[1])
        jz[i, j + 1, k] += f[2] * (1.0 - w[0]) * w[1]
        jz[i + 1, j + 1, k] += f[2] * w[0] * w[1]

    for r in recs:
        q = params.species[int(r["typeId"])].charge * params.species[int(r["typeId"])].size
        old = [r["x"], r["y"], r["z"]]
        v = [r["vx"], r["vy"], r["vz"]]
        new = [old[a] + v[a] for a in range(3)]
        ref = [relay(new[a], old[a]) for a in range(3)]
        deposit(old, [q * (ref[a] - old[a]) for a in range(3)],
                [0.5 * (ref[a] + old[a]) - (cell(old[a]) - 1.0) for a in range(3)])
        old2 = [new[a] - v[a] for a in range(3)]
        ref2 = [relay(new[a], old2[a]) for a in range(3)]
        deposit(new, [q * (new[a] - ref2[a]) for a in range(3)],
                [0.5 * (ref2[a] + new[a]) - (cell(new[a]) - 1.0) for a in range(3)])
    return jx, jy, jz


def interior_particles(n, count, seed, vmax=0.8, planar=False):
    """Particles away from the box faces with velocities up to vmax per axis;
    planar: one velocity component (a random one per particle) is zero."""
    rng = np.random.default_rng(seed)
    recs = random_particles(count, (3, 3, 3), (n - 4,) * 3, 0.0, seed, 0)
    for key in ("vx", "vy", "vz"):
        recs[key] = rng.uniform(-vmax, vmax, count)
    if planar:
        axis = rng.integers(0, 3, count)
        for a, key in enumerate(("vx", "vy", "vz")):
            recs[key][axis == a] = 0.0
    return recs


def test_oracle_current_matches_restatement():
    cfg = em_config(n=12)
    p = cfg.params
    recs = interior_particles(12, 60, 3)
    o = orc.Oracle(p)
    o.load_particles(0, recs)
    o.update_position()
    want = py_current(p, recs, (14, 14, 14))
    for which, w in zip((38, 39, 40), want):
        got = o.field(which)
        assert np.max(np.abs(got - w)) <= 1e-14 * np.max(np.abs(w)), which
    o.close()


def div_j(o):
    jx, jy, jz = (o.field(w) for w in (38, 39, 40))
    X, Y, Z = jy.shape[0], jx.shape[1], jx.shape[2]
    d = np.zeros((X, Y, Z))
    d[1:-1, 1:-1, 1:-1] = (jx[1:, 1:-1, 1:-1] - jx[:-1, 1:-1, 1:-1] + jy[1:-1, 1:, 1:-1] - jy[1:-1, :-1, 1:-1]
                           + jz[1:-1, 1:-1, 1:] - jz[1:-1, 1:-1, :-1])
    return d


def test_oracle_zigzag_current_conserves_charge():
    """rho^{n+1} - rho^n + div J = 0 (dt = dx = 1) at every node for particles that
    cross cell faces (up to 0.8 cells per step per axis) but no box face, moving
    in a coordinate plane. The reference's weights (the segment midpoints,
    particle.cpp:270-297) leave out the (dy dz / 12)-type terms of the exact
    trilinear identity, so a move along all three axes conserves charge only to
    that order: checked by the second half of the test."""
    cfg = em_config(n=16, ppc=2)
    p = cfg.params
    o = orc.Oracle(p)
    for s in range(2):
        o.load_particles(s, interior_particles(16, 4000, 10 + s, planar=True))
    o.update_rho()
    rho0 = o.field(1)
    o.update_position()
    o.update_rho()
    rho1 = o.field(1)
    res = (rho1 - rho0 + div_j(o))[1:-1, 1:-1, 1:-1]
    scale = np.max(np.abs(rho0))
    assert np.max(np.abs(res)) <= 1e-12 * scale, np.max(np.abs(res)) / scale
    assert np.max(np.abs(rho1 - rho0)) > 1e-3 * scale        # charge did move
    o.close()
    # one particle moving along all three axes: the defect is q/12 (dx dy dz) summed
    # over the corner terms, nonzero and of that order
    o = orc.Oracle(p)
    r = interior_particles(16, 1, 5)
    r["x"], r["y"], r["z"] = 6.55, 6.3, 6.45
    r["vx"], r["vy"], r["vz"] = 0.7, -0.6, 0.5
    o.load_particles(0, r)
    o.update_rho()
    rho0 = o.field(1)
    o.update_position()
    o.update_rho()
    res = rho0 * 0 + (o.field(1) - rho0 + div_j(o))
    q = abs(p.species[0].charge * p.species[0].size)
    assert 1e-3 * q < np.max(np.abs(res)) < 0.7 * 0.6 * 0.5 * q
    o.close()


# ---------------------------------------------------------------- FDTD
class Based:
    """A numpy array indexed with the reference's index bases."""

    def __init__(self, a, lo):
        self.a, self.lo = a, lo

    def __getitem__(self, idx):
        return self.a[tuple(np.asarray(i) - l for i, l in zip(idx, self.lo))]


def np_damp1(r, L, real):
    r = np.asarray(r, dtype=np.float64)
    d = np.where(r <= 0, -r + 1.0, np.where(r >= real - 1, r - real + 2.0, 0.0))
    return 1.0 - (1.0 * d / L) ** 2


def np_glue(arr, per):
    """sendRecvField's self branch along each periodic axis (index base 0 there):
    index 0 <- index m-2, index m-1 <- index 1, x then y then z."""
    for a in per:
        m = arr.shape[a]
        lo = np.take(arr, 1, axis=a).copy()
        sl0 = [slice(None)] * 3
        sl0[a] = 0
        arr[tuple(sl0)] = np.take(arr, m - 2, axis=a)
        sl0[a] = m - 1
        arr[tuple(sl0)] = lo


def np_fdtd(f, j, lo, up, c, L, eps0, mu0, per):
    """updateEfieldFDTDDamping then updateBfieldDamping (RootGridField.cpp:594-820),
    vectorised, each followed by the periodic glue copies: f = [ex, ey, ez, bx,
    by, bz] as arrays starting at index lo; returns the updated arrays."""
    ex, ey, ez, bx, by, bz = (a.copy() for a in f)
    jx, jy, jz = j
    I, J, K = np.meshgrid(*[np.arange(lo[a] + 1, up[a] - 1) for a in range(3)], indexing="ij")

    def m(i, jj, k):
        return np_damp1(i, L[0], c[0]) * np_damp1(jj, L[1], c[1]) * np_damp1(k, L[2], c[2])

    real = (I > 0) & (I < c[0] - 1) & (J > 0) & (J < c[1] - 1) & (K > 0) & (K < c[2] - 1)
    dte = 1.0 / eps0
    C = dte / (mu0 * 1.0)
    BX, BY, BZ = Based(bx, lo), Based(by, lo), Based(bz, lo)

    def upd(arr, cur, jarr, axis, curl, nxt):
        idx = (I, J, K)
        pos = [I, J, K]
        keep = real | (pos[axis] < up[axis] - 2)
        plain = real & (pos[axis] < c[axis] - 2)
        jv = np.zeros(I.shape)
        jv[plain] = jarr[I[plain], J[plain], K[plain]]
        e = Based(arr, lo)[idx]
        new = np.where(plain, e - jv * dte + C * curl, 0.5 * (m(I, J, K) + m(*nxt)) * (e + C * curl))
        sub = tuple(p[keep] - l for p, l in zip(idx, lo))
        arr[sub] = new[keep]

    upd(ex, None, jx, 0, BZ[I, J, K] - BZ[I, J - 1, K] - BY[I, J, K] + BY[I, J, K - 1], (I + 1, J, K))
    upd(ey, None, jy, 1, BX[I, J, K] - BX[I, J, K - 1] - BZ[I, J, K] + BZ[I - 1, J, K], (I, J + 1, K))
    upd(ez, None, jz, 2, BY[I, J, K] - BY[I - 1, J, K] - BX[I, J, K] + BX[I, J - 1, K], (I, J, K + 1))

    for arr in (ex, ey, ez):
        np_glue(arr, per)
    EX, EY, EZ = Based(ex, lo), Based(ey, lo), Based(ez, lo)
    gx = (EY[I, J, K + 1] - EY[I, J, K]) - (EZ[I, J + 1, K] - EZ[I, J, K])
    gy = (EZ[I + 1, J, K] - EZ[I, J, K]) - (EX[I, J, K + 1] - EX[I, J, K])
    gz = (EX[I, J + 1, K] - EX[I, J, K]) - (EY[I + 1, J, K] - EY[I, J, K])
    specs = [(bx, gx, (1, 2), [(I, J, K), (I, J + 1, K), (I, J, K + 1), (I, J + 1, K + 1)]),
             (by, gy, (0, 2), [(I, J, K), (I + 1, J, K), (I, J, K + 1), (I + 1, J, K + 1)]),
             (bz, gz, (0, 1), [(I, J, K), (I + 1, J, K), (I, J + 1, K), (I + 1, J + 1, K)])]
    pos = [I, J, K]
    for arr, g, (a1, a2), corners in specs:
        inner = (pos[a1] != c[a1] - 2) & (pos[a2] != c[a2] - 2)
        keep = real | ((pos[a1] != up[a1] - 2) & (pos[a2] != up[a2] - 2))
        mask = 0.25 * (m(*corners[0]) + m(*corners[1]) + m(*corners[2]) + m(*corners[3]))
        b = Based(arr, lo)[(I, J, K)]
        new = np.where(real & inner, b + 1.0 * g, mask * (b + 1.0 * g))
        sub = tuple(p[keep] - l for p, l in zip((I, J, K), lo))
        arr[sub] = new[keep]
    for arr in (bx, by, bz):
        np_glue(arr, per)
    return ex, ey, ez, bx, by, bz


@pytest.mark.parametrize("boundary", ["DDDDDD", "PPDDPP"])
def test_oracle_fdtd_matches_numpy(boundary):
    n = 6
    cfg = em_config(n=n, boundary=boundary)
    p = cfg.params
    o = orc.Oracle(p)
    rng = np.random.default_rng(1)
    f = []
    for which in range(32, 38):
        _, shp = o.field_shape(which)
        a = rng.standard_normal(shp)
        o.set_field(which, a)
        f.append(a)
    j = []
    for which in (38, 39, 40):
        _, shp = o.field_shape(which)
        a = rng.standard_normal(shp) * 1e-3
        o.set_field(which, a)
        j.append(a)
    lo = o.field_shape(35)[0]
    c = (n + 2,) * 3
    up = tuple(c[a] if boundary[2 * a + 1] == "P" else c[a] + n for a in range(3))
    per = [a for a in range(3) if boundary[2 * a] == "P"]
    want = np_fdtd(f, j, lo, up, c, (n, n, n), p.eps0, p.mu0, per)
    o.update_efield()
    o.update_bfield()
    for q, which in enumerate(range(32, 38)):
        got = o.field(which)
        err = np.max(np.abs(got - want[q])) / np.max(np.abs(want[q]))
        assert err <= 1e-13, (which, err)
        assert np.max(np.abs(got - f[q])) > 1e-3          # the update changed it
    o.close()


def test_relay_point_pinned_to_reference():
    """The oracle's zigzag relay point against the reference's own
    Position::getReferencePosition (include/position.hpp:88-96, compiled into
    oracle/_ref): moves within a cell, across one face, across two and three
    faces, onto and off exact integer coordinates, below zero (periodic glue)."""
    rng = np.random.default_rng(4)
    old = rng.uniform(-1.0, 20.0, (20000, 3))
    step = rng.uniform(-0.99, 0.99, (20000, 3))
    new = old + step
    old[:500] = np.floor(old[:500])                 # start on a node
    new[500:1000] = np.floor(new[500:1000])         # end on a node
    new[1000:1500] = old[1000:1500]                 # no move
    want = orc.ref_relay(new, old)
    if want is None:
        pytest.skip("oracle/_ref was not built (reference sources absent)")
    got = orc.relay(new, old)
    assert np.array_equal(got, want)
    # the relay sits on the shared face when the cells differ
    cross = np.floor(new[:, 0]) != np.floor(old[:, 0])
    assert cross.sum() > 1000
    assert np.all(got[cross, 0] == np.maximum(np.floor(new[cross, 0]), np.floor(old[cross, 0])))


def test_oracle_em_velocity_matches_restatement():
    """Grid::updateParticleVelocityEM (src/Grid/GridParticleTreatmentEM.cpp:13-105)
    restated in numpy on the oracle's own nodal E and B: CIC weights times 0.5 q/m,
    boris = 2 / (1 + |b|^2) with the gathered b."""
    cfg = em_config(n=9)
    p = cfg.params
    o = orc.Oracle(p)
    rng = np.random.default_rng(12)
    for which in range(32, 38):               # random Yee fields, then the nodal references
        o.set_field(which, rng.standard_normal(o.field_shape(which)[1]))
    o.set_field(0, rng.standard_normal((11, 11, 11)))
    o.update_efield()
    o.update_bfield()
    recs = random_particles(500, (0, 0, 0), (8, 8, 8), 0.05, 3, 0)
    o.load_particles(0, recs)
    E = [o.field(w) for w in (2, 3, 4)]
    B = [o.field(w) for w in (5, 6, 7)]
    assert max(np.max(np.abs(b)) for b in B) > 0.1
    o.update_velocity()
    got = o.particles(0)
    qm = 0.5 * p.species[0].charge / p.species[0].mass
    x, y, z = recs["x"], recs["y"], recs["z"]
    i, j, k = (np.floor(c).astype(int) + 1 for c in (x, y, z))
    dx1, dy1, dz1 = x - (i - 1), y - (j - 1), z - (k - 1)
    dx2, dy2, dz2 = 1 - dx1, 1 - dy1, 1 - dz1
    w = [qm * dx2 * dy2 * dz2, qm * dx1 * dy2 * dz2, qm * dx2 * dy1 * dz2, qm * dx1 * dy1 * dz2,
         qm * dx2 * dy2 * dz1, qm * dx1 * dy2 * dz1, qm * dx2 * dy1 * dz1, qm * dx1 * dy1 * dz1]
    corners = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)]

    def gather(a):
        return sum(wc * a[i + c[0], j + c[1], k + c[2]] for wc, c in zip(w, corners))

    ex, ey, ez = (gather(a) for a in E)
    bx, by, bz = (gather(a) for a in B)
    boris = 2.0 / (1.0 + (bx * bx + by * by + bz * bz))
    vx1, vy1, vz1 = recs["vx"] + ex, recs["vy"] + ey, recs["vz"] + ez
    vxt = vx1 + vy1 * bz - vz1 * by
    vyt = vy1 + vz1 * bx - vx1 * bz
    vzt = vz1 + vx1 * by - vy1 * bx
    want = (vx1 + ex + boris * (vyt * bz - vzt * by), vy1 + ey + boris * (vzt * bx - vxt * bz),
            vz1 + ez + boris * (vxt * by - vyt * bx))
    for key, wv in zip(("vx", "vy", "vz"), want):
        assert np.max(np.abs(got[key] - wv)) <= 1e-12 * np.max(np.abs(wv)), key
    o.close()
