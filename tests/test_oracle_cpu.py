"""CPU tests: the oracle against known-answer vectors, the reference's own
Position header and analytic physics; the C ABI library's exports; the
host-side set-up code. None of these touch a GPU."""
import math
import os
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from fopis_b200 import _abi, config
from fopis_b200.config import SpeciesInfo, make_params, plasma_units

from helpers import random_particles

ROOT = Path(__file__).resolve().parent.parent
# the reference checkout, for its sample inputs (tests that need it skip when unset)
REFERENCE = Path(os.environ["FOPIS_REFERENCE"]) if os.environ.get("FOPIS_REFERENCE") else None


def test_philox_known_answers():
    # Random123 kat_vectors for philox4x32-10
    assert orc.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert orc.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert orc.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_position_matches_reference_header():
    rng = np.random.default_rng(1)
    pts = np.concatenate([rng.uniform(-2.0, 40.0, (5000, 3)), np.floor(rng.uniform(-2, 40, (500, 3))),
                          np.array([[0.0, -1.0, 31.999999999]])])
    ijk, d = orc.position(pts)
    ref = orc.ref_position(pts)
    if ref is None:
        pytest.skip("oracle/_ref was not built (reference sources absent)")
    assert np.array_equal(ijk, ref[0])
    assert np.array_equal(d, ref[1])


def test_abi_library_exports_every_declared_symbol():
    lib = _abi.library()
    header = (ROOT / "include" / "fopis_gpu.h").read_text()
    names = set(re.findall(r"\b(fopis_[a-z_0-9]+)\s*\(", header))
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
        assert n in _abi.SIGNATURES, n
    assert lib.fopis_version().startswith(b"fopis-b200")


def test_abi_struct_layout_matches_header(tmp_path):
    """Every field offset and struct size of the ctypes mirror against the C
    compiler's offsetof/sizeof on include/fopis_gpu.h."""
    import ctypes as C
    import subprocess
    structs = {"fopis_species": _abi.Species, "fopis_params": _abi.Params,
               "fopis_object_desc": _abi.ObjectDesc, "fopis_stats": _abi.Stats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT / "include" / "fopis_gpu.h"}"',
             "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} __sizeof__ %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, cls in structs.items():
        assert got[(cname, "__sizeof__")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def _write(tmp_path, text):
    p = tmp_path / "body.obj"
    p.write_text(text)
    return p


@pytest.mark.parametrize("boxes,nxyz,n_cmat", [
    ([((-4, -4, -4), (4, 4, 4))], (65, 65, 65), 386),
    ([((-8, -8, -8), (8, 8, 8))], (129, 129, 129), 1538),
    ([((-3, -2, -1), (3, 2, 5))], (24, 20, 22), None),
    ([((-16, -8, -8), (16, 8, 8)), ((-24, 8, -8), (24, 12, 8))], (97, 97, 97), None),
])
def test_obj_parser_matches_oracle(tmp_path, boxes, nxyz, n_cmat):
    p = _write(tmp_path, config.box_obj_text(boxes))
    a_nodes, a_cells = config.parse_obj(p, *nxyz)
    b_nodes, b_cells = orc.parse_obj(p, *nxyz)
    assert np.array_equal(a_nodes, b_nodes)
    assert np.array_equal(a_cells, b_cells)
    if n_cmat:
        assert len(a_nodes) == n_cmat
    # the inner cells are exactly the union's volume, and every exposed face of
    # that volume has its four nodes among the surface nodes (absorption and
    # emission put charge only there)
    union = np.zeros(tuple(n + 1 for n in nxyz), dtype=bool)
    for lo, hi in boxes:
        union[tuple(slice(l + n // 2 + 1, h + n // 2 + 1) for l, h, n in zip(lo, hi, nxyz))] = True
    cells = np.zeros_like(union)
    cells[tuple(a_cells.reshape(-1, 3).T)] = True
    assert np.array_equal(cells, union)
    surface = {tuple(v) for v in a_nodes.reshape(-1, 3)}
    for ax in range(3):
        u, w = [a for a in range(3) if a != ax]
        for shift, high in ((1, 0), (-1, 1)):
            for c in np.argwhere(cells & ~np.roll(cells, shift, axis=ax)):
                c[ax] += high
                for du in (0, 1):
                    for dw in (0, 1):
                        q = c.copy()
                        q[u] += du
                        q[w] += dw
                        assert tuple(q) in surface


@pytest.mark.skipif(REFERENCE is None or not (REFERENCE / "input_samples/objects").exists(),
                    reason="FOPIS_REFERENCE unset or its sample inputs absent")
@pytest.mark.parametrize("name", ["cube.obj", "4x4x4_Sphere.obj", "8x8x8_Sphere.obj", "20x2x2_Line.obj",
                                  "test_solar_array.obj"])
def test_obj_parser_on_reference_samples(name):
    path = REFERENCE / "input_samples/objects" / name
    a = config.parse_obj(path, 64, 64, 64)
    b = orc.parse_obj(path, 64, 64, 64)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert len(a[0]) > 0


def test_flux_integral_matches_closed_form():
    # isotropic Maxwellian: one-sided flux n vth / (2 sqrt(pi)) per unit area
    f = config.calc_flux(0.2, 1000.0, 10.0, (0, 0, 0), (1,) * 6)
    expect = 0.2 / (2 * math.sqrt(math.pi)) * 1000.0 / 10.0
    assert all(abs(v - expect) / expect < 1e-3 for v in f)
    g = config.calc_flux(0.2, 1000.0, 10.0, (0.1, 0, 0), (0, 1, 1, 1, 1, 1))
    assert g[0] == 0.0 and g[1] < f[1]


def _periodic_params(n=16, ppc=8, cold=False, ion_mass=100.0):
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1e-12 if cold else 1.0, ppc),
          SpeciesInfo("Ion", "ambient", ion_mass, 1.0, 1e7, 1e-12 if cold else 1.0, ppc)]
    p, norm = make_params((n, n, n), "PPPPPP", dx, dt, sp)
    return p


def test_oracle_charge_conservation_and_fixed_point_replay():
    p = _periodic_params()
    o = orc.Oracle(p)
    n = 16 ** 3 * 4
    for s in range(2):
        o.load_particles(s, random_particles(n, (-1, -1, -1), (16, 16, 16), 0.1, 10 + s, s))
    o.update_rho()
    unique = (slice(1, 17),) * 3
    q = [p.species[s].charge * p.species[s].size for s in range(2)]
    for s in range(2):
        rs = o.field(16 + s)
        assert abs(rs[unique].sum() - q[s] * n) < 1e-9 * abs(q[s] * n)
        # the fixed-point replay conserves the charge exactly: 2^51 per particle
        rec = o.particles(s)
        fl = np.floor(np.stack([rec["x"], rec["y"], rec["z"]], 1))
        ijk = fl.astype(np.int64) + 1
        off = (np.stack([rec["x"], rec["y"], rec["z"]], 1) - fl).astype(np.float32)
        packed = (ijk[:, 0] << 20) | (ijk[:, 1] << 10) | ijk[:, 2]
        W = orc.fixed_deposit(p, packed.astype(np.int32), off[:, 0], off[:, 1], off[:, 2])
        assert sum(int(v) for v in W[unique].ravel()) == n * (1 << 51)   # exact, beyond int64
        rfix = W * (q[s] * 2.0 ** -51)
        assert np.max(np.abs(rfix - rs)) < 3e-5 * np.max(np.abs(rs))


def test_oracle_psor_agrees_with_exact_solve():
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, 4)]
    p, _ = make_params((17, 17, 17), "DDDDDD", dx, dt, sp)
    rng = np.random.default_rng(3)
    rho = np.zeros((19, 19, 19))
    rho[2:-2, 2:-2, 2:-2] = rng.standard_normal((15, 15, 15)) * 1e6
    a = orc.Oracle(p)
    a.set_field(1, rho)
    a.set_solver(0, max_post_loop=1000)
    a.solve()
    b = orc.Oracle(p)
    b.set_field(1, rho)
    b.set_solver(1, exact_tol=1e-13)
    b.solve()
    pa, pb = a.field(0), b.field(0)
    assert np.max(np.abs(pa - pb)) < 1e-6 * np.max(np.abs(pb))
    it, res = b.solver_stats()
    assert res < 1e-12


def test_oracle_langmuir_oscillation_at_plasma_frequency():
    """Cold electrons displaced by a sine wave over immobile ions oscillate at
    omega_pe (omega_pe dt = 0.1); the field energy oscillates at 2 omega_pe."""
    n = 16
    p = _periodic_params(n=n, ppc=8, cold=True, ion_mass=1e9)
    o = orc.Oracle(p)
    o.set_solver(1, exact_tol=1e-12)
    rng = np.random.default_rng(7)
    per = n ** 3 * 8
    base = random_particles(per, (0, 0, 0), (n, n, n), 0.0, 5, 0)
    ions = base.copy()
    ions["typeId"] = 1
    elec = base.copy()
    elec["x"] = (elec["x"] + 0.05 * np.sin(2 * np.pi * elec["x"] / n)) % n
    o.load_particles(0, elec)
    o.load_particles(1, ions)
    o.initialize()
    fe = []
    for _ in range(80):
        o.main_loop(1)
        fe.append(o.energy()[1])
    fe = np.array(fe)
    minima = [t for t in range(1, len(fe) - 1) if fe[t] < fe[t - 1] and fe[t] <= fe[t + 1]]
    assert len(minima) >= 2
    period = 2 * np.mean(np.diff(minima))           # field energy period is half the plasma period
    assert abs(period - 2 * np.pi / 0.1) / (2 * np.pi / 0.1) < 0.08, period


def test_oracle_injection_counts_follow_flux_with_carry():
    cfg = config.workload("cube64", ppc=4)
    o = orc.Oracle(cfg.params)
    total = np.zeros((cfg.params.nspecies, 6), np.int64)
    for _ in range(5):
        total += o.inject()
    for s in range(2):
        sp = cfg.params.species[s]
        area = 64.0 * 64.0   # (getYNodeSize()-1)(getZNodeSize()-1), RootGridParticle.cpp:213
        for face in range(6):
            expect = 5 * area * sp.flux[face]
            assert abs(total[s, face] - expect) <= 1.0


def test_exact_capacity_matrix_matches_solved_one():
    """The sine-basis capacity matrix equals the one built by a converged solve
    per surface node (the reference's procedure) on a 25^3 Dirichlet box."""
    from fopis_b200.config import SpeciesInfo, make_params, plasma_units, objects_from_boxes
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, 2)]
    p, _ = make_params((25, 25, 25), "DDDDDD", dx, dt, sp, tol=1e-10)
    obj = objects_from_boxes([((-2, -3, -1), (2, 3, 2))], (25, 25, 25))
    o = orc.Oracle(p, [obj])
    o.set_solver(1, exact_tol=1e-13)
    o.build_cmatrix(0)
    Cs = o.get_cmatrix(0)
    Cx = orc.dirichlet_capacity_matrix(p, obj.nodes)
    assert np.abs(Cx - Cs).max() < 1e-11 * np.abs(Cs).max()
