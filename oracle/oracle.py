"""TEST INFRASTRUCTURE — ctypes wrapper of oracle/liboracle.so, the CPU FP64
restatement of the reference's ES timestep (see fopis_oracle.cpp's header).

Only the tests, the smoke check and the benchmark's CPU leg import this
module; the product never does. ``pin_position`` wraps the reference's own
include/position.hpp compiled into oracle/_ref/ (present only where the
reference sources were available at build time).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_PIN = HERE / "_ref" / "libpin_position.so"
REF_NORM = HERE / "_ref" / "libpin_normalizer.so"

PARTICLE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8"),
                           ("typeId", "<i4"), ("isValid", "<i4")])

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise ImportError(f"{LIB} missing: run `make -C oracle`")
        L = C.CDLL(str(LIB))
        vp, dp, i64p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)
        sig = {
            "orc_create": (vp, [vp]), "orc_destroy": (None, [vp]), "orc_threads": (C.c_int, []),
            "orc_set_threads": (None, [C.c_int]),
            "orc_philox": (None, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
            "orc_set_solver": (None, [vp, C.c_int, C.c_int, C.c_double]),
            "orc_solver_stats": (None, [vp, C.POINTER(C.c_int), dp]),
            "orc_pointwise_residual": (C.c_double, [vp]),
            "orc_add_object": (C.c_int, [vp, vp]), "orc_build_cmatrix": (C.c_int, [vp, C.c_int]),
            "orc_set_cmatrix": (C.c_int, [vp, C.c_int, dp, C.c_int]),
            "orc_get_cmatrix": (C.c_int, [vp, C.c_int, dp, C.c_int]),
            "orc_get_object": (None, [vp, C.c_int, dp, dp, dp]),
            "orc_get_charge_map": (None, [vp, C.c_int, dp]),
            "orc_load_particles": (C.c_int64, [vp, C.c_int, vp, C.c_int64]),
            "orc_num_particles": (C.c_int64, [vp, C.c_int]),
            "orc_get_particles": (C.c_int64, [vp, C.c_int, vp, C.c_int64]),
            "orc_generate_ambient": (None, [vp]), "orc_reset_objects": (None, [vp]),
            "orc_update_velocity": (None, [vp]), "orc_emit": (C.c_int, [vp]),
            "orc_update_position": (None, [vp]), "orc_inject": (None, [vp, i64p]),
            "orc_update_rho": (C.c_int, [vp]), "orc_solve_poisson": (None, [vp]),
            "orc_update_efield": (None, [vp]), "orc_remove_invalid": (None, [vp]),
            "orc_main_loop": (C.c_int, [vp, C.c_int]), "orc_initialize": (C.c_int, [vp]),
            "orc_set_timestep": (None, [vp, C.c_int64]), "orc_get_timestep": (C.c_int64, [vp]),
            "orc_step_counts": (None, [vp, i64p, i64p, i64p]),
            "orc_get_field": (C.c_int, [vp, C.c_int, dp]), "orc_set_field": (C.c_int, [vp, C.c_int, dp]),
            "orc_energy": (None, [vp, dp, dp]),
            "orc_parse_obj": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.POINTER(C.c_int), vp,
                                        C.c_int, C.POINTER(C.c_int)]),
            "orc_fixed_deposit": (None, [vp, vp, vp, vp, vp, C.c_int64, vp]),
            "orc_fixed_fold": (None, [vp, vp]),
            "orc_position": (None, [vp, C.c_int64, vp, vp]),
            "orc_get_incidents": (C.c_int64, [vp, dp, C.c_int64]),
            "orc_update_bfield": (None, [vp]), "orc_bfield_energy": (C.c_double, [vp]),
            "orc_relay": (None, [vp, vp, C.c_int64, vp]),
            "orc_field_shape": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "orc_set_incidents": (None, [vp, dp, C.c_int64]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def philox(ctr, key):
    out = (C.c_uint32 * 4)()
    lib().orc_philox((C.c_uint32 * 4)(*ctr), (C.c_uint32 * 2)(*key), out)
    return list(out)


def parse_obj(path: str, nx: int, ny: int, nz: int):
    cap = nx * ny * nz
    nodes = np.zeros(3 * cap, np.int32)
    cells = np.zeros(3 * cap, np.int32)
    nn, nc = C.c_int(), C.c_int()
    rc = lib().orc_parse_obj(str(path).encode(), nx, ny, nz, nodes.ctypes.data, cap, C.byref(nn), cells.ctypes.data,
                             cap, C.byref(nc))
    if rc:
        raise ValueError(f"oracle could not parse {path}: {rc}")
    return nodes[: 3 * nn.value].reshape(-1, 3), cells[: 3 * nc.value].reshape(-1, 3)


def fixed_deposit(params, cell, ox, oy, oz) -> np.ndarray:
    """Integer CIC replay of one species (sum 2^51 per particle), then the periodic fold."""
    shape = (params.nx + 2, params.ny + 2, params.nz + 2)
    out = np.zeros(int(np.prod(shape)), np.int64)
    cell = np.ascontiguousarray(cell, np.int32)
    f = [np.ascontiguousarray(a, np.float32) for a in (ox, oy, oz)]
    lib().orc_fixed_deposit(C.addressof(params), cell.ctypes.data, f[0].ctypes.data, f[1].ctypes.data,
                            f[2].ctypes.data, len(cell), out.ctypes.data)
    lib().orc_fixed_fold(C.addressof(params), out.ctypes.data)
    return out.reshape(shape)


def position(xyz: np.ndarray):
    """The oracle's restatement of Position::setXYZ on the given points."""
    xyz = np.ascontiguousarray(xyz, np.float64)
    n = len(xyz)
    ijk = np.zeros((n, 3), np.int32)
    d = np.zeros((n, 6), np.float64)
    lib().orc_position(xyz.ctypes.data, n, ijk.ctypes.data, d.ctypes.data)
    return ijk, d


def relay(new_xyz: np.ndarray, old_xyz: np.ndarray) -> np.ndarray:
    """The oracle's zigzag relay points for pairs of positions."""
    a = np.ascontiguousarray(new_xyz, np.float64)
    b = np.ascontiguousarray(old_xyz, np.float64)
    out = np.zeros_like(a)
    lib().orc_relay(a.ctypes.data, b.ctypes.data, len(a), out.ctypes.data)
    return out


def ref_relay(new_xyz: np.ndarray, old_xyz: np.ndarray):
    """The reference's own Position::getReferencePosition (oracle/_ref), or None
    where the reference sources were absent at build time."""
    if not REF_PIN.exists():
        return None
    L = C.CDLL(str(REF_PIN))
    L.ref_relay.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    a = np.ascontiguousarray(new_xyz, np.float64)
    b = np.ascontiguousarray(old_xyz, np.float64)
    out = np.zeros_like(a)
    L.ref_relay(a.ctypes.data, b.ctypes.data, len(a), out.ctypes.data)
    return out


NORMALIZER_UNITS = ("eps0", "mu0", "c", "V_unit", "A_unit", "velocity", "bfield", "current_density", "density",
                    "energy", "energy_ev", "capacitance")
NORMALIZER_APPLY = {"velocity": 0, "unvelocity": 1, "potential": 2, "unpotential": 3, "current_density": 4,
                    "uncurrent": 5, "uncharge": 6, "unenergy": 7, "capacitance": 8, "density": 9, "bfield": 10}


def ref_normalizer_units(dx: float, dt: float):
    """The reference's own Normalizer (include/normalizer.hpp, src/Misc/Normalizer.cpp)
    after Initializer's unit set-up with dx and dt: a dict over NORMALIZER_UNITS, or None."""
    if not REF_NORM.exists():
        return None
    L = C.CDLL(str(REF_NORM))
    L.ref_normalizer_units.argtypes = [C.c_double, C.c_double, C.c_void_p, C.c_int]
    L.ref_normalizer_units.restype = C.c_int
    out = np.zeros(len(NORMALIZER_UNITS), np.float64)
    m = L.ref_normalizer_units(dx, dt, out.ctypes.data, len(out))
    return dict(zip(NORMALIZER_UNITS[:m], out[:m].tolist()))


def ref_normalizer_apply(dx: float, dt: float, kind: str, values: np.ndarray):
    """One of the reference Normalizer's conversions (NORMALIZER_APPLY) on values, or None."""
    if not REF_NORM.exists():
        return None
    L = C.CDLL(str(REF_NORM))
    L.ref_normalizer_apply.argtypes = [C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_int64, C.c_void_p]
    L.ref_normalizer_apply.restype = C.c_int
    x = np.ascontiguousarray(values, np.float64)
    out = np.zeros_like(x)
    if L.ref_normalizer_apply(dx, dt, NORMALIZER_APPLY[kind], x.ctypes.data, len(x), out.ctypes.data) != 0:
        raise ValueError(kind)
    return out


def ref_position(xyz: np.ndarray):
    """The reference's own Position (include/position.hpp) on the given points, or None."""
    if not REF_PIN.exists():
        return None
    L = C.CDLL(str(REF_PIN))
    L.ref_position.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    xyz = np.ascontiguousarray(xyz, np.float64)
    n = len(xyz)
    ijk = np.zeros((n, 3), np.int32)
    d = np.zeros((n, 6), np.float64)
    L.ref_position(xyz.ctypes.data, n, ijk.ctypes.data, d.ctypes.data)
    return ijk, d


def dirichlet_capacity_matrix(params, nodes, max_table: float = 6e7) -> np.ndarray:
    """Capacity matrix of one conductor in a box whose six faces are Dirichlet
    (phi = 0), built exactly instead of by one Poisson solve per surface node.

    RootGrid::initializeObjectsCmatrix (src/Grid/RootGrid/RootGridObject.cpp:77-148)
    fills M[c][r] = phi at surface node r for rho = 1 at surface node c (the
    Poisson solve ignores the body) and inverts M. With Dirichlet faces the
    unknowns of axis d are glue indices 2..n_d-1 (u = 1..m_d, m_d = n_d - 2) and
    the 7-point operator diagonalises in the sine basis
        s_k(u) = sqrt(2/(m+1)) sin(pi k u/(m+1)),  lambda_k = 2 - 2 cos(pi k/(m+1)),
    so M[c][r] = (1/eps0) sum_k prod_d s_{k_d}(r_d) s_{k_d}(c_d) / sum_d lambda_{k_d}.
    The sum is taken over pairs of the distinct surface coordinates per axis
    (three BLAS contractions), which is the converged solve the reference's
    PSOR approximates. Returns C = M^-1 (numpy's LU inverse in place of Eigen's).
    """
    b = bytes(params.boundary).split(b"\0")[0].decode()
    if b != "DDDDDD":
        raise NotImplementedError("exact capacity matrix needs six Dirichlet faces, got " + b)
    nodes = np.asarray(nodes, np.int64)
    dims = (params.nx, params.ny, params.nz)
    S, W, idx = [], None, []
    lam = []
    for d in range(3):
        m = dims[d] - 2
        u = nodes[:, d] - 1
        if u.min() < 1 or u.max() > m:
            raise ValueError("a surface node sits on a Dirichlet face")
        U, inv = np.unique(u, return_inverse=True)
        k = np.arange(1, m + 1)
        S.append(np.sqrt(2.0 / (m + 1)) * np.sin(np.pi * np.outer(k, U) / (m + 1)))   # (m, |U|)
        lam.append(2.0 - 2.0 * np.cos(np.pi * k / (m + 1)))
        idx.append(inv)
    mx, my, mz = (s.shape[1] for s in S)
    if float(mx * my * mz) ** 2 > max_table:
        raise NotImplementedError("surface spans too many distinct coordinates for the pair table")
    W = 1.0 / (lam[0][:, None, None] + lam[1][None, :, None] + lam[2][None, None, :])
    P = [np.einsum("ka,kb->kab", s, s).reshape(s.shape[0], -1) for s in S]     # (m, |U|^2)
    nx_, ny_, nz_ = W.shape
    Q1 = W.reshape(nx_ * ny_, nz_) @ P[2]                                        # (kx*ky, C)
    Q1 = Q1.reshape(nx_, ny_, -1)
    Q2 = np.einsum("yb,xyc->xbc", P[1], Q1, optimize=True)                       # (kx, B, C)
    T = (P[0].T @ Q2.reshape(nx_, -1)).reshape(mx, mx, my, my, mz, mz)
    ix, iy, iz = idx
    M = T[ix[:, None], ix[None, :], iy[:, None], iy[None, :], iz[:, None], iz[None, :]] / params.eps0
    return np.linalg.inv(M)


class Oracle:
    """One CPU simulation with the reference's semantics (FP64)."""

    def __init__(self, params, objects=(), cmatrices=None):
        self.L = lib()
        self.params = params
        self.h = self.L.orc_create(C.addressof(params))
        self.shape = (params.nx + 2, params.ny + 2, params.nz + 2)
        self.nsp = params.nspecies
        self.objects = list(objects)
        self._keep = []
        for k, o in enumerate(self.objects):
            self.add_object(o)

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_object(self, o):
        from fopis_b200 import _abi
        nodes = np.ascontiguousarray(o.nodes, np.int32)
        cells = np.ascontiguousarray(o.cells, np.int32)
        self._keep += [nodes, cells]
        d = _abi.ObjectDesc()
        d.n_cmat = len(nodes)
        d.cmat_nodes = nodes.ctypes.data_as(C.POINTER(C.c_int32))
        d.n_cells = len(cells)
        d.cells = cells.ctypes.data_as(C.POINTER(C.c_int32))
        d.is_potential_fixed = o.is_potential_fixed
        d.fixed_potential = o.fixed_potential
        d.initial_potential_offset = o.initial_potential_offset
        d.emit_species = o.emit_species
        d.secondary_species = getattr(o, "secondary_species", -1)
        d.dielectric = getattr(o, "dielectric", 0)
        if d.dielectric:
            cap = np.ascontiguousarray(o.capacitance, np.float64)
            self._keep.append(cap)
            d.capacitance = cap.ctypes.data_as(C.POINTER(C.c_double))
        return self.L.orc_add_object(self.h, C.addressof(d))

    def get_incidents(self):
        """Spacecraft::incident_events as an [n, 10] array (object, species, axis,
        remaining time, x, y, z, vx, vy, vz)."""
        n = self.L.orc_get_incidents(self.h, None, 0)
        out = np.zeros((max(n, 1), 10))
        self.L.orc_get_incidents(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), n)
        return out[:n]

    def set_incidents(self, recs):
        recs = np.ascontiguousarray(recs, np.float64).reshape(-1, 10)
        self.L.orc_set_incidents(self.h, recs.ctypes.data_as(C.POINTER(C.c_double)), len(recs))

    def set_solver(self, mode: int, max_post_loop: int = 1000, exact_tol: float = 1e-13):
        self.L.orc_set_solver(self.h, mode, max_post_loop, exact_tol)

    def solver_stats(self):
        it, res = C.c_int(), C.c_double()
        self.L.orc_solver_stats(self.h, C.byref(it), C.byref(res))
        return it.value, res.value

    def pointwise_residual(self):
        """RootGrid::checkPhiResidual's measure on the current phi and rho."""
        return self.L.orc_pointwise_residual(self.h)

    def build_cmatrix(self, obj=0):
        rc = self.L.orc_build_cmatrix(self.h, obj)
        if rc:
            raise RuntimeError("oracle capacity matrix inversion failed")

    def set_cmatrix(self, obj, Cm):
        Cm = np.ascontiguousarray(Cm, np.float64)
        assert self.L.orc_set_cmatrix(self.h, obj, Cm.ctypes.data_as(C.POINTER(C.c_double)), Cm.shape[0]) == 0

    def get_cmatrix(self, obj=0):
        n = len(self.objects[obj].nodes)
        out = np.zeros((n, n))
        assert self.L.orc_get_cmatrix(self.h, obj, out.ctypes.data_as(C.POINTER(C.c_double)), n) == 0
        return out

    def get_object(self, obj=0):
        V, Q = C.c_double(), C.c_double()
        cur = np.zeros(self.nsp)
        self.L.orc_get_object(self.h, obj, C.byref(V), C.byref(Q), cur.ctypes.data_as(C.POINTER(C.c_double)))
        return V.value, Q.value, cur

    def charge_map(self, obj=0):
        n = len(self.objects[obj].nodes)
        out = np.zeros((self.nsp, n))
        self.L.orc_get_charge_map(self.h, obj, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def load_particles(self, s, recs):
        recs = np.ascontiguousarray(recs, PARTICLE_DTYPE)
        return self.L.orc_load_particles(self.h, s, recs.ctypes.data, len(recs))

    def particles(self, s):
        n = self.L.orc_num_particles(self.h, s)
        out = np.zeros(max(n, 1), PARTICLE_DTYPE)
        k = self.L.orc_get_particles(self.h, s, out.ctypes.data, n)
        return out[:k]

    def generate_ambient(self):
        self.L.orc_generate_ambient(self.h)

    def reset_objects(self):
        self.L.orc_reset_objects(self.h)

    def update_velocity(self):
        self.L.orc_update_velocity(self.h)

    def emit(self):
        return self.L.orc_emit(self.h)

    def update_position(self):
        self.L.orc_update_position(self.h)

    def inject(self):
        counts = np.zeros(6 * self.nsp, np.int64)
        self.L.orc_inject(self.h, counts.ctypes.data_as(C.POINTER(C.c_int64)))
        return counts.reshape(self.nsp, 6)

    def update_rho(self):
        return self.L.orc_update_rho(self.h)

    def solve(self):
        self.L.orc_solve_poisson(self.h)

    def update_efield(self):
        self.L.orc_update_efield(self.h)

    def remove_invalid(self):
        self.L.orc_remove_invalid(self.h)

    def main_loop(self, n=1):
        return self.L.orc_main_loop(self.h, n)

    def initialize(self):
        return self.L.orc_initialize(self.h)

    @property
    def timestep(self):
        return self.L.orc_get_timestep(self.h)

    @timestep.setter
    def timestep(self, t):
        self.L.orc_set_timestep(self.h, t)

    def step_counts(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        self.L.orc_step_counts(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def field_shape(self, which):
        """(first index, extent) per axis; the EM Yee arrays start below 0 on
        axes with damping layers."""
        lo, n = (C.c_int * 3)(), (C.c_int * 3)()
        assert self.L.orc_field_shape(self.h, which, lo, n) == 0
        return tuple(lo), tuple(n)

    def field(self, which):
        _, n = self.field_shape(which)
        out = np.zeros(n)
        assert self.L.orc_get_field(self.h, which, out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        return out

    def set_field(self, which, a):
        _, n = self.field_shape(which)
        a = np.ascontiguousarray(a, np.float64).reshape(n)
        assert self.L.orc_set_field(self.h, which, a.ctypes.data_as(C.POINTER(C.c_double))) == 0

    def update_bfield(self):
        self.L.orc_update_bfield(self.h)

    def bfield_energy(self):
        return self.L.orc_bfield_energy(self.h)

    def energy(self):
        pe, fe = C.c_double(), C.c_double()
        self.L.orc_energy(self.h, C.byref(pe), C.byref(fe))
        return pe.value, fe.value
