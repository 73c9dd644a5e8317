"""input.json -> fopis_params, as Initializer::loadEnvironment / loadParticleType /
loadStaticField do it (src/Misc/Initialize.cpp:158-421) with the unit system of
Normalizer (include/normalizer.hpp), plus builders for the synthetic workloads.

Units after normalisation: length dx, time dt, mass m_e, charge e
(Initialize.cpp:33-36).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import tempfile
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _abi

# include/global.hpp:27-31
E = 1.60217733e-19
EPS0 = 8.854187817e-12
MU0 = 4.0 * math.pi * 1.0e-7
ME = 9.1093818872e-31
CLIGHT = 2.99792458e8


class Normalizer:
    """include/normalizer.hpp: x_unit = dx, t_unit = dt, m_unit = m_e, e_unit = e."""

    def __init__(self, dx: float, dt: float):
        # Normalizer::updatePhysicalConstants (include/normalizer.hpp:24-38) in the
        # reference's operation order, so every factor is the reference's to the bit:
        # pow(u, 2) is the product u * u (the compiler's form of it), pow(u, 3) the libm pow
        self.x = dx
        self.t = dt
        self.m = ME
        self.e = E
        self.x_pow_3 = dx ** 3
        self.V_unit = (dx * dx) * ME / (E * (dt * dt))
        self.A_unit = E / dt
        self.eps0 = EPS0 * (self.x_pow_3 * ME) / ((E * E) * (dt * dt))   # normalizeEpsilon
        self.mu0 = MU0 * (E * E) / (ME * dx)                              # normalizeMu
        self.c = self.velocity(CLIGHT)                                    # normalizeVelocity(c): the Courant number

    def velocity(self, v):
        return self.t * v / self.x

    def unvelocity(self, v):
        return v * self.x / self.t

    def bfield(self, b):
        return b * (self.t * self.e) / self.m

    def current_density(self, j):
        return j * (self.x * self.x) / self.A_unit

    def potential(self, phi):
        return phi / self.V_unit

    def unpotential(self, phi):
        return phi * self.V_unit

    def uncharge(self, q):
        return q * self.e

    def uncurrent(self, i):
        return i * self.A_unit

    def unenergy(self, en):
        return en * self.m * (self.x * self.x) / (self.t * self.t)

    def unenergy_ev(self, en):
        """unnormalizeEnergy(en, "eV")."""
        return en * self.m * (self.x * self.x) / (self.e * (self.t * self.t))


def calc_flux(vth: float, density_norm: float, size: float, drift: Sequence[float],
              injection_axis: Sequence[int]) -> List[float]:
    """AmbientParticleType::calcFlux (src/Particle/AmbientParticleType.cpp:8-57):
    numerical integral of v f(v) on [-6, 6] thermal units with step 1e-3, split
    by the sign of v, in super particles per unit area per step."""
    ddv = 1e-3
    nvx = 12.0 / ddv
    flux = [0.0] * 6
    for axis in range(3):
        d = drift[axis] / vth
        lo = hi = 0.0
        i = 0
        while i < nvx - 1:
            arg1 = i * ddv + (d - 6.0)
            argx1 = (arg1 - d) ** 2
            if arg1 > 0.0:
                lo += arg1 * math.exp(-argx1) * ddv
            else:
                hi += arg1 * math.exp(-argx1) * ddv
            i += 1
        flux[2 * axis] = lo * (vth / math.sqrt(math.pi)) * density_norm / size
        flux[2 * axis + 1] = -hi * (vth / math.sqrt(math.pi)) * density_norm / size
    return [f if injection_axis[k] else 0.0 for k, f in enumerate(flux)]


@dataclass
class SpeciesInfo:
    name: str
    kind: str                 # "ambient" | "photoelectron" | "secondary"
    mass: float               # in m_e
    charge: float             # in e
    density: float            # m^-3
    temperature: float        # eV
    ppc: int
    drift_kms: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    injection_axis: Tuple[int, ...] = (1, 1, 1, 1, 1, 1)
    current_density: float = 0.0   # A/m^2, photoelectrons


@dataclass
class ObjectInfo:
    name: str
    nodes: np.ndarray                # [n_cmat, 3] int32 glue-layout
    cells: np.ndarray                # [n_cells, 3] int32 glue-layout
    is_potential_fixed: int = 0
    fixed_potential: float = 0.0     # volts
    initial_potential_offset: float = 0.0
    emit_species: int = -1
    file_name: str = ""              # the .obj file's name without directories (capacity-matrix cache name)
    secondary_species: int = -1      # secondary-electron species this body emits
    dielectric: int = 0              # surface_type "dielectric"
    capacitance: Optional[np.ndarray] = None   # [n_cmat] normalised node capacitance (dielectric)


@dataclass
class SimConfig:
    params: _abi.Params
    norm: Normalizer
    species: List[SpeciesInfo]
    objects: List[ObjectInfo] = field(default_factory=list)
    max_timestep: int = 0
    dx: float = 1.0
    dt: float = 1.0
    use_existing_capacity_matrix: bool = False
    maximum_poisson_post_loop: int = 1000
    plot_energy_width: int = 0       # IO.plot_energy_width: energy log every this many steps, 0 = never


def _species_struct(sp: SpeciesInfo, norm: Normalizer, dx: float) -> _abi.Species:
    s = _abi.Species()
    s.kind = {"ambient": _abi.SPECIES_AMBIENT, "photoelectron": _abi.SPECIES_PHOTOELECTRON,
              "secondary": _abi.SPECIES_SECONDARY}[sp.kind]
    s.particle_per_cell = int(sp.ppc)
    s.charge = float(sp.charge)
    s.mass = float(sp.mass)
    s.size = float(int(dx ** 3 * sp.density / sp.ppc))            # ParticleType::updateSize
    T = E * sp.temperature                                         # setTemperature stores e * T[eV]
    s.thermal_velocity = norm.velocity(math.sqrt(2.0 * T / (sp.mass * ME)))
    s.deviation = norm.velocity(math.sqrt(T / (sp.mass * ME)))
    for a in range(3):
        s.drift[a] = sp.drift_kms[a] * (1e3 * norm.velocity(1.0))      # Initialize.cpp:353-355
    for a in range(6):
        s.injection_axis[a] = int(sp.injection_axis[a])
    if sp.kind == "ambient":
        dens_norm = sp.density * dx ** 3                          # normalizeDensity
        fl = calc_flux(s.thermal_velocity, dens_norm, s.size, list(s.drift), list(s.injection_axis))
        for a in range(6):
            s.flux[a] = fl[a]
    elif sp.kind == "photoelectron":
        j = norm.current_density(sp.current_density)
        s.emission_amount = 1.0 * j / (abs(sp.charge) * s.size)   # area dx^2 = 1 (Spacecraft.cpp:876-877)
    return s


def make_params(nxyz: Tuple[int, int, int], boundary: str, dx: float, dt: float, species: List[SpeciesInfo],
                bfield_nT=(0.0, 0.0, 0.0), shine=(0.0, 0.0, 0.0), seed: int = 12345, tol: float = 1e-8,
                max_vcycles: int = 100, sort_interval: int = 8, guess: int = _abi.GUESS_WARM,
                capacity_factor: float = 1.5, precision: int = _abi.MIXED,
                solver: str = "ES") -> Tuple[_abi.Params, Normalizer]:
    norm = Normalizer(dx, dt)
    if solver not in ("ES", "EM"):
        raise ValueError(f"solver_type {solver} is neither ES nor EM")
    if solver == "EM" and norm.c > 1.0:
        # Environment::checkCFLCondition (src/Misc/Environment.cpp:193-203) aborts the run
        raise ValueError(f"Courant number exceeds 1.0 (c dt / dx = {norm.c:.6g})")
    p = _abi.Params()
    p.nx, p.ny, p.nz = (int(v) for v in nxyz)
    p.boundary = boundary.encode()
    p.eps0 = norm.eps0
    for a in range(3):
        p.static_bfield[a] = bfield_nT[a] * (norm.bfield(1.0) * 1e-9)   # Initialize.cpp:314-318
        p.shine_vector[a] = float(shine[a])
    # Environment::resetParticleTypeOrder (Environment.cpp:360-377): ambient, photoelectron, secondary
    ordered = [s for k in ("ambient", "photoelectron", "secondary") for s in species if s.kind == k]
    species[:] = ordered
    p.nspecies = len(species)
    for i, sp in enumerate(species):
        p.species[i] = _species_struct(sp, norm, dx)
    p.poisson_tol = tol
    p.max_vcycles = max_vcycles
    p.guess_mode = guess
    p.sort_interval = sort_interval
    p.remove_interval = 50
    p.capacity_factor = capacity_factor
    p.precision = precision
    p.seed = seed
    p.energy_ev = norm.unenergy_ev(1.0)                        # Normalizer::unnormalizeEnergy(1, "eV")
    p.solver = _abi.SOLVER_EM if solver == "EM" else _abi.SOLVER_ES
    p.mu0 = norm.mu0
    return p, norm


def parse_obj(path: str, nx: int, ny: int, nz: int) -> Tuple[np.ndarray, np.ndarray]:
    """fopis_parse_obj through the C ABI (ObjectUtils::getObjectNodesFromObjFile)."""
    lib = _abi.library()
    nodes = C.POINTER(C.c_int32)()
    cells = C.POINTER(C.c_int32)()
    nn = C.c_int()
    nc = C.c_int()
    rc = lib.fopis_parse_obj(str(path).encode(), nx, ny, nz, C.byref(nodes), C.byref(nn), C.byref(cells), C.byref(nc))
    if rc != 0:
        raise _abi.FopisError(rc, f"cannot parse {path}")
    a = np.ctypeslib.as_array(nodes, shape=(max(nn.value, 1) * 3,))[: nn.value * 3].reshape(-1, 3).copy()
    b = np.ctypeslib.as_array(cells, shape=(max(nc.value, 1) * 3,))[: nc.value * 3].reshape(-1, 3).copy()
    lib.fopis_free(C.cast(nodes, C.c_void_p))
    lib.fopis_free(C.cast(cells, C.c_void_p))
    return a.astype(np.int32), b.astype(np.int32)


def parse_obj_textures(path: str, nx: int, ny: int, nz: int) -> List[List[int]]:
    """fopis_parse_obj_textures: per surface node (cmat order) the texture index of
    every quad covering it (ObjectDataFromFile::textures, ObjectUtils.cpp:65-160)."""
    lib = _abi.library()
    start = C.POINTER(C.c_int32)()
    tex = C.POINTER(C.c_int32)()
    n = C.c_int()
    rc = lib.fopis_parse_obj_textures(str(path).encode(), nx, ny, nz, C.byref(start), C.byref(tex), C.byref(n))
    if rc != 0:
        raise _abi.FopisError(rc, f"cannot parse {path}")
    st = np.ctypeslib.as_array(start, shape=(n.value + 1,)).copy()
    tx = np.ctypeslib.as_array(tex, shape=(max(int(st[-1]), 1),))[: int(st[-1])].copy()
    lib.fopis_free(C.cast(start, C.c_void_p))
    lib.fopis_free(C.cast(tex, C.c_void_p))
    return [list(map(int, tx[st[m]:st[m + 1]])) for m in range(n.value)]


# Spacecraft::material_property_list (SpacecraftMaterialPropertyList.cpp:3-34).
RELATIVE_PERMITTIVITY = {"Silicon": 12.0, "Aluminum": 9.5, "EpoxyGlass": 5.0, "Bakelite": 4.8,
                         "GlassReinforcedTeflon": 2.32, "Teflon": 2.1}


def node_capacitance(textures: List[List[int]], materials: dict, norm: Normalizer) -> np.ndarray:
    """Spacecraft::construct's dielectric capacitance map (Spacecraft.cpp:117-149): per
    node the mean over its quads of normalizeCapacitance(4 pi eps0 eps_r) of the quad's
    material (texture index -> material name)."""
    per_tex = {}
    out = np.zeros(len(textures))
    for m, tl in enumerate(textures):
        acc = 0.0
        for t in tl:
            if t not in per_tex:
                name = materials.get(t)
                if name not in RELATIVE_PERMITTIVITY:
                    raise ValueError(f"Invalid material name {name} is specified to be assigned the texture index {t}.")
                per_tex[t] = 4.0 * math.pi * EPS0 * RELATIVE_PERMITTIVITY[name] * norm.V_unit / norm.e
            acc += per_tex[t]
        out[m] = acc / len(tl)
    return out


def box_obj_text(boxes: Sequence[Tuple[Tuple[int, int, int], Tuple[int, int, int]]]) -> str:
    """A MagicaVoxel-style .obj of the union of axis-aligned boxes [lo, hi) in
    vertex units (relative to the domain centre). Like a MagicaVoxel export it
    lists only the exposed faces of the voxel union, merged per plane into
    rectangles, in the order axis, side (low then high), plane; a face two boxes
    share is not written (ObjectUtils' pair scan would read it as a closing
    face). A single box gives its six faces."""
    lo = np.min([b[0] for b in boxes], axis=0)
    hi = np.max([b[1] for b in boxes], axis=0)
    occ = np.zeros(tuple(int(h - l) + 2 for l, h in zip(lo, hi)), dtype=bool)   # one empty layer each side
    for (bl, bh) in boxes:
        occ[tuple(slice(int(bl[a] - lo[a]) + 1, int(bh[a] - lo[a]) + 1) for a in range(3))] = True
    verts: List[Tuple[int, int, int]] = []
    faces: List[Tuple[int, int, int, int, int]] = []
    for axis in range(3):
        u, w = [a for a in range(3) if a != axis]
        for side in (0, 1):
            nb = np.roll(occ, 1 if side == 0 else -1, axis=axis)
            exposed = occ & ~nb                           # cells whose low (high) face is on the surface
            for c in range(occ.shape[axis]):
                m = np.take(exposed, c, axis=axis).copy()   # indexed [u, w]
                for a0 in range(m.shape[0]):
                    for b0 in range(m.shape[1]):
                        if not m[a0, b0]:
                            continue
                        b1 = b0
                        while b1 + 1 < m.shape[1] and m[a0, b1 + 1]:
                            b1 += 1
                        a1 = a0
                        while a1 + 1 < m.shape[0] and m[a1 + 1, b0:b1 + 1].all():
                            a1 += 1
                        m[a0:a1 + 1, b0:b1 + 1] = False
                        plane = int(lo[axis]) + c - 1 + side
                        quad = []
                        for (a, b) in ((a0, b0), (a1 + 1, b0), (a1 + 1, b1 + 1), (a0, b1 + 1)):
                            p = [0, 0, 0]
                            p[axis] = plane
                            p[u] = int(lo[u]) + a - 1
                            p[w] = int(lo[w]) + b - 1
                            verts.append(tuple(p))
                            quad.append(len(verts))
                        faces.append((*quad, 2 * axis + side + 1))
    out = ["# voxel bodies", "vt 0.5 0.5"]
    out += [f"v {x} {y} {z}" for (x, y, z) in verts]
    out += [f"f {a}/1/{n} {b}/1/{n} {c}/1/{n} {d}/1/{n}" for (a, b, c, d, n) in faces]
    return "\n".join(out) + "\n"


def objects_from_boxes(boxes, nxyz, name="Spacecraft", emit_species=-1, fixed=None, offset=0.0,
                       obj_parser=None) -> ObjectInfo:
    """The conductor made of `boxes`, written as a MagicaVoxel .obj and parsed by
    `obj_parser(path, nx, ny, nz) -> (nodes, cells)` (default: fopis_parse_obj
    of this library)."""
    fd, path = tempfile.mkstemp(suffix=".obj")
    with os.fdopen(fd, "w") as f:
        f.write(box_obj_text(boxes))
    try:
        nodes, cells = (obj_parser or parse_obj)(path, *nxyz)
    finally:
        os.unlink(path)
    return ObjectInfo(name=name, nodes=nodes, cells=cells, is_potential_fixed=int(fixed is not None),
                      fixed_potential=0.0 if fixed is None else fixed, initial_potential_offset=offset,
                      emit_species=emit_species)


def plasma_units(n0: float = 1e7, te_ev: float = 1.0, dt_omega: float = 0.1):
    """dx = lambda_De (1 - 1e-6) and dt = dt_omega / omega_pe for an electron plasma."""
    lam = math.sqrt(EPS0 * te_ev * E / (E * E * n0))
    wpe = math.sqrt(n0 * E * E / (ME * EPS0))
    return lam * (1.0 - 1e-6), dt_omega / wpe


def workload(name: str, ppc: Optional[int] = None, seed: int = 20251203, obj_parser=None, **kw) -> SimConfig:
    """Synthetic configurations (obj_parser: the .obj loader for the bodies,
    default this library's fopis_parse_obj):
    periodic32   32^3 cells periodic, 16 ppc/species, no object (CPU-runnable case);
    cube64       64^3 cells Dirichlet + injection, 8^3 cube conductor, 32 ppc;
    cube128      128^3 cells Dirichlet + injection, 16^3 cube, photoemission from +x;
    cube128_plain same without photoemission;
    craft256     256^3 cells, 32x16x16 body + 48x4x16 panel, photoemission;
    em128        the EM solver on 128^3 cells Dirichlet + injection, no object,
                 Te = 5 keV, n = 1e12 m^-3, dx = 0.5 m, dt = dx / (2 c) (Courant 0.5).
    Electrons + ions (mass ratio 100), Te = Ti = 1 eV, n = 1e7 m^-3 (em128 as stated)."""
    dx, dt = plasma_units()
    n0, te = 1e7, 1.0
    if name == "em128":
        dx, n0, te = 0.5, 1e12, 5e3
        dt = 0.5 * dx / CLIGHT
        kw.setdefault("solver", "EM")
    if ppc is None:
        ppc = 16 if name == "periodic32" else 32
    e_sp = SpeciesInfo("Electron", "ambient", 1.0, -1.0, n0, te, ppc)
    i_sp = SpeciesInfo("Ion", "ambient", 100.0, 1.0, n0, 1.0 if name == "em128" else te, ppc)
    species = [e_sp, i_sp]
    shine = (0.0, 0.0, 0.0)
    boxes = []
    photo = False
    if name == "periodic32":
        nxyz, boundary = (32, 32, 32), "PPPPPP"
    elif name == "cube64":
        nxyz, boundary = (65, 65, 65), "DDDDDD"
        boxes = [((-4, -4, -4), (4, 4, 4))]
    elif name in ("cube128", "cube128_plain"):
        nxyz, boundary = (129, 129, 129), "DDDDDD"
        boxes = [((-8, -8, -8), (8, 8, 8))]
        photo = name == "cube128"
    elif name == "em128":
        nxyz, boundary = (129, 129, 129), "DDDDDD"
    elif name == "craft256":
        nxyz, boundary = (257, 257, 257), "DDDDDD"
        boxes = [((-16, -8, -8), (16, 8, 8)), ((-24, 8, -8), (24, 12, 8))]
        photo = True
    else:
        raise ValueError(f"unknown workload {name}")
    if photo:
        # photoelectron flux 10x the ambient electron flux e n vbar / 4, T = 0.2 Te
        vbar = math.sqrt(8.0 * te * E / (math.pi * ME))
        j = 10.0 * E * n0 * vbar / 4.0
        species.append(SpeciesInfo("PhotoElectron", "photoelectron", 1.0, -1.0, n0, 0.2 * te, ppc, current_density=j))
        shine = (-1.0, 0.0, 0.0)
    p, norm = make_params(nxyz, boundary, dx, dt, species, shine=shine, seed=seed, **kw)
    objs = []
    if boxes:
        emit = next((k for k, s in enumerate(species) if s.kind == "photoelectron"), -1)
        objs.append(objects_from_boxes(boxes, nxyz, emit_species=emit, obj_parser=obj_parser))
    return SimConfig(params=p, norm=norm, species=species, objects=objs, dx=dx, dt=dt)


def load_input(path: str) -> SimConfig:
    """Initializer::initTDPIC's parsing (Initialize.cpp:158-421) of an input.json."""
    base = Path(path).resolve().parent
    with open(path) as f:
        js = json.load(f)
    env = js["Environment"]
    dx, dt = float(env["dx"]), float(env["dt"])
    nxyz = (int(env["nx"]), int(env["ny"]), int(env["nz"]))
    if int(env.get("proc_x", 1)) * int(env.get("proc_y", 1)) * int(env.get("proc_z", 1)) != 1:
        raise ValueError("the whole domain lives on one GPU: proc_x = proc_y = proc_z = 1")
    species = []
    for name in sorted(js["Plasma"]):                 # picojson objects are std::map (sorted keys)
        pl = js["Plasma"][name]
        kind = pl["type"]
        if kind not in ("ambient", "photoelectron", "secondary"):
            raise ValueError(f"species type {kind} is outside the ES hot path")
        species.append(SpeciesInfo(name, kind, float(pl["mass"]), float(pl["charge"]), float(pl["density"]),
                                   float(pl["temperature"]), int(pl["particle_per_cell"]),
                                   tuple(pl.get("drift_velocity", (0.0, 0.0, 0.0))),
                                   tuple(int(bool(v)) for v in pl.get("injection_axis", [1] * 6)),
                                   float(pl.get("current_density", 0.0))))
    field_in = js.get("Field", {})
    bfield = field_in.get("static_bfield", (0.0, 0.0, 0.0))
    shine = field_in.get("shine_vector", (0.0, 0.0, 0.0))
    opts = js.get("Options", {})
    p, norm = make_params(nxyz, env["boundary"], dx, dt, species, bfield_nT=bfield, shine=shine,
                          solver=str(env.get("solver_type", "ES")))
    objs = []
    names = [s.name for s in species]
    for oname in sorted(js.get("Object", {})):
        o = js["Object"][oname]
        surface = o.get("surface_type", "perfect")
        if surface not in ("perfect", "dielectric"):
            raise ValueError(f"surface_type {surface} is not perfect or dielectric")
        fpath = o["file_name"]
        if not os.path.isabs(fpath):
            fpath = str(base / fpath)
        nodes, cells = parse_obj(fpath, *nxyz)
        emit, second = -1, -1
        for pname in o.get("emit_particles", {}):
            if pname in names and species[names.index(pname)].kind == "photoelectron":
                emit = names.index(pname)
            if pname in names and species[names.index(pname)].kind == "secondary":
                second = names.index(pname)
        cap = None
        if surface == "dielectric":
            mats = {int(k): v for k, v in o.get("materials", {}).items()}
            cap = node_capacitance(parse_obj_textures(fpath, *nxyz), mats, norm)
        objs.append(ObjectInfo(oname, nodes, cells, int(o.get("is_potential_fixed", False)),
                               norm.potential(float(o.get("fixed_potential", 0.0))),
                               norm.potential(float(o.get("initial_potential_offset", 0.0))), emit,
                               file_name=os.path.basename(o["file_name"]), secondary_species=second,
                               dielectric=int(surface == "dielectric"), capacitance=cap))
    return SimConfig(params=p, norm=norm, species=species, objects=objs, max_timestep=int(env.get("max_timestep", 0)),
                     dx=dx, dt=dt, use_existing_capacity_matrix=bool(opts.get("use_existing_capacity_matrix", False)),
                     maximum_poisson_post_loop=int(opts.get("maximum_poisson_post_loop", 1000)),
                     plot_energy_width=int(float(js.get("IO", {}).get("plot_energy_width", 0))))
