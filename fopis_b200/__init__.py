"""fopis_b200 — the electrostatic PIC timestep of FOPIS on B200 (sm_100a).

``RootGrid`` mirrors the reference's RootGrid ES surface (include/grid.hpp:233-300:
updateParticleVelocity, emitParticlesFromObjects, updateParticlePosition,
injectParticlesFromBoundary, updateRho, solvePoisson, updateEfield,
mainLoopES) over the C ABI of libfopis_gpu.so (include/fopis_gpu.h). Every
method calls a hand-written CUDA path; when the library or a CUDA device is
missing the constructor raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import FopisError, library
from .config import ObjectInfo, SimConfig, load_input, workload

__all__ = ["RootGrid", "FopisError", "library", "load_input", "workload", "PARTICLE_DTYPE"]

# The reference's 56-byte Particle record (include/particle.hpp:14-20).
PARTICLE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8"),
                           ("typeId", "<i4"), ("isValid", "<i4")])
assert PARTICLE_DTYPE.itemsize == 56


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class RootGrid:
    """One simulation context on one GPU."""

    def __init__(self, cfg: SimConfig, device: int = 0):
        self.lib = library()
        self.cfg = cfg
        self.p = cfg.params
        self.nspecies = self.p.nspecies
        self.shape = (self.p.nx + 2, self.p.ny + 2, self.p.nz + 2)
        self.N = int(np.prod(self.shape))
        h = C.c_void_p()
        rc = self.lib.fopis_create(C.byref(self.p), int(device), C.byref(h))
        if rc != 0:
            raise FopisError(rc, self.lib.fopis_last_error(None).decode())
        self.h = h
        self._keep = []
        self.object_ids = []
        for o in cfg.objects:
            self.add_object(o)

    # ------------------------------------------------------------ plumbing
    def _check(self, rc: int, allow=(0,)):
        if rc not in allow:
            raise FopisError(rc, self.lib.fopis_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.fopis_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------ objects
    def add_object(self, o: ObjectInfo) -> int:
        nodes = np.ascontiguousarray(o.nodes, dtype=np.int32)
        cells = np.ascontiguousarray(o.cells, dtype=np.int32)
        d = _abi.ObjectDesc()
        d.n_cmat = len(nodes)
        d.cmat_nodes = nodes.ctypes.data_as(C.POINTER(C.c_int32))
        d.n_cells = len(cells)
        d.cells = cells.ctypes.data_as(C.POINTER(C.c_int32))
        d.is_potential_fixed = o.is_potential_fixed
        d.fixed_potential = o.fixed_potential
        d.initial_potential_offset = o.initial_potential_offset
        d.emit_species = o.emit_species
        d.secondary_species = o.secondary_species
        d.dielectric = o.dielectric
        if o.dielectric:
            cap = np.ascontiguousarray(o.capacitance, dtype=np.float64)
            self._keep.append(cap)
            d.capacitance = cap.ctypes.data_as(C.POINTER(C.c_double))
        oid = C.c_int()
        self._check(self.lib.fopis_add_object(self.h, C.byref(d), C.byref(oid)))
        self.object_ids.append(oid.value)
        return oid.value

    def initializeObjectsCmatrix(self, obj: int = 0):
        self._check(self.lib.fopis_build_capacity_matrix(self.h, obj))

    def set_cmatrix(self, obj: int, Cm: np.ndarray):
        Cm = np.ascontiguousarray(Cm, dtype=np.float64)
        self._check(self.lib.fopis_set_capacity_matrix(self.h, obj, _dp(Cm), Cm.shape[0]))

    def get_cmatrix(self, obj: int = 0) -> np.ndarray:
        n = len(self.cfg.objects[obj].nodes)
        out = np.empty((n, n))
        self._check(self.lib.fopis_get_capacity_matrix(self.h, obj, _dp(out), n))
        return out

    def getObject(self, obj: int = 0):
        """(potential, total charge, current per species), normalised (Spacecraft::getLogEntry)."""
        V, Q = C.c_double(), C.c_double()
        cur = np.zeros(self.nspecies)
        self._check(self.lib.fopis_get_object(self.h, obj, C.byref(V), C.byref(Q), _dp(cur)))
        return V.value, Q.value, cur

    def get_incidents(self) -> np.ndarray:
        """The pending incident events as an [n, 10] array: object, species, axis,
        remaining time, crossing point x, y, z, velocity vx, vy, vz."""
        n = C.c_int64()
        self._check(self.lib.fopis_get_incidents(self.h, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), _abi.INCIDENT_DOUBLES))
        self._check(self.lib.fopis_get_incidents(self.h, _dp(out), n.value, C.byref(n)))
        return out[: n.value]

    def set_incidents(self, recs: np.ndarray):
        recs = np.ascontiguousarray(recs, dtype=np.float64).reshape(-1, _abi.INCIDENT_DOUBLES)
        self._check(self.lib.fopis_set_incidents(self.h, _dp(recs), len(recs)))

    def getChargeMap(self, obj: int = 0) -> np.ndarray:
        n = len(self.cfg.objects[obj].nodes)
        out = np.zeros((self.nspecies, n))
        self._check(self.lib.fopis_get_charge_map(self.h, obj, _dp(out), out.size))
        return out

    # ------------------------------------------------------------ particles
    def load_particles(self, species: int, recs: np.ndarray):
        recs = np.ascontiguousarray(recs, dtype=PARTICLE_DTYPE)
        self._check(self.lib.fopis_load_particles(self.h, species, recs.ctypes.data, len(recs)))

    def generate_ambient(self):
        self._check(self.lib.fopis_generate_ambient(self.h))

    def getParticles(self, species: int) -> np.ndarray:
        st = self.stats()
        cap = int(st.num_particles[species])
        out = np.zeros(max(cap, 1), dtype=PARTICLE_DTYPE)
        n = C.c_int64()
        self._check(self.lib.fopis_get_particles(self.h, species, out.ctypes.data, cap, C.byref(n)))
        return out[: n.value]

    def getParticlesRaw(self, species: int):
        st = self.stats()
        cap = int(st.num_particles[species])
        cell = np.zeros(max(cap, 1), np.int32)
        f = [np.zeros(max(cap, 1), np.float32) for _ in range(6)]
        n = C.c_int64()
        self._check(self.lib.fopis_get_particles_raw(self.h, species, cell.ctypes.data, *[a.ctypes.data for a in f],
                                                     cap, C.byref(n)))
        k = n.value
        return cell[:k], [a[:k] for a in f]

    def sort(self):
        self._check(self.lib.fopis_sort_particles(self.h))

    # ------------------------------------------------------------ ES step
    def initialize(self):
        """Grid::initialize (src/Grid/Grid.cpp:23-36)."""
        return self._check(self.lib.fopis_initialize(self.h), allow=(0, _abi.ERR_NOT_CONVERGED))

    def mainLoopES(self, n: int = 1):
        return self._check(self.lib.fopis_step(self.h, int(n)), allow=(0, _abi.ERR_NOT_CONVERGED))

    step = mainLoopES

    def updateParticleVelocity(self):
        self._check(self.lib.fopis_update_velocity(self.h))

    def emitParticlesFromObjects(self):
        self._check(self.lib.fopis_emit_particles(self.h))

    def updateParticlePosition(self):
        self._check(self.lib.fopis_update_position(self.h))

    def injectParticlesFromBoundary(self):
        self._check(self.lib.fopis_inject_particles(self.h))

    def updateRho(self):
        return self._check(self.lib.fopis_update_rho(self.h), allow=(0, _abi.ERR_NOT_CONVERGED))

    def solvePoisson(self):
        return self._check(self.lib.fopis_solve_poisson(self.h), allow=(0, _abi.ERR_NOT_CONVERGED))

    def updateEfield(self):
        self._check(self.lib.fopis_update_efield(self.h))

    def removeInvalidParticles(self):
        self._check(self.lib.fopis_remove_invalid_particles(self.h))

    def advance_timestep(self):
        self._check(self.lib.fopis_advance_timestep(self.h))

    # ------------------------------------------------------------ fields
    def field_shape(self, which: int):
        """(first index, extent) per axis of a field; the EM Yee arrays start
        below 0 on axes with damping layers (boost::multi_array index bases)."""
        lo, n = (C.c_int * 3)(), (C.c_int * 3)()
        self._check(self.lib.fopis_field_shape(self.h, which, lo, n))
        return tuple(lo), tuple(n)

    def get_field(self, which: int) -> np.ndarray:
        _, n = self.field_shape(which)
        out = np.empty(n)
        self._check(self.lib.fopis_get_field(self.h, which, _dp(out), out.size))
        return out

    def set_field(self, which: int, a: np.ndarray):
        _, n = self.field_shape(which)
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(n)
        self._check(self.lib.fopis_set_field(self.h, which, _dp(a), a.size))

    def updateReferenceFields(self):
        """Nodal E (and in the EM mode B) from the current fields, as Grid::initializeForLoad."""
        self._check(self.lib.fopis_update_reference_fields(self.h))

    def updateBfield(self):
        """RootGrid::updateBfield (EM mode)."""
        self._check(self.lib.fopis_update_bfield(self.h))

    def mainLoopEM(self, n: int = 1):
        """n calls of RootGrid::mainLoopEM (fopis_step of a context created with solver EM)."""
        if self.p.solver != _abi.SOLVER_EM:
            raise _abi.FopisError(_abi.ERR_STATE, "the context runs the ES solver")
        return self.mainLoopES(n)

    def getBref(self):
        return tuple(self.get_field(w) for w in (_abi.FIELD_BXREF, _abi.FIELD_BYREF, _abi.FIELD_BZREF))

    def getBfieldEnergy(self) -> float:
        e = C.c_double()
        self._check(self.lib.fopis_get_bfield_energy(self.h, C.byref(e)))
        return e.value

    def getPhi(self):
        return self.get_field(_abi.FIELD_PHI)

    def getRho(self, species: Optional[int] = None):
        return self.get_field(_abi.FIELD_RHO0 if species is None else _abi.FIELD_RHO_SPECIES + species)

    def getEref(self):
        return tuple(self.get_field(w) for w in (_abi.FIELD_EXREF, _abi.FIELD_EYREF, _abi.FIELD_EZREF))

    def getEnergy(self):
        pe, fe = C.c_double(), C.c_double()
        self._check(self.lib.fopis_get_energy(self.h, C.byref(pe), C.byref(fe)))
        return pe.value, fe.value

    def stats(self) -> _abi.Stats:
        st = _abi.Stats()
        self._check(self.lib.fopis_get_stats(self.h, C.byref(st)))
        return st

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        self._check(self.lib.fopis_get_stream(self.h, C.byref(s)))
        return int(s.value or 0)

    def set_guess_mode(self, mode: int):
        self._check(self.lib.fopis_set_guess_mode(self.h, mode))

    def unet_training(self, enable: bool, lr: float = 1e-3):
        self._check(self.lib.fopis_unet_set_training(self.h, int(enable), float(lr)))

    def unet_state(self):
        loss, steps = C.c_double(), C.c_int64()
        self._check(self.lib.fopis_unet_get_state(self.h, C.byref(loss), C.byref(steps)))
        return loss.value, steps.value

    def unet_policy(self):
        """(history-start V-cycles average, learned V-cycles average, learned guess enabled)."""
        a, b, on = C.c_double(), C.c_double(), C.c_int()
        self._check(self.lib.fopis_unet_get_policy(self.h, C.byref(a), C.byref(b), C.byref(on)))
        return a.value, b.value, bool(on.value)

    def unet_last(self):
        """(history-start residual, guess residual, forward ms, training ms) of the last first solve."""
        v = [C.c_double() for _ in range(4)]
        self._check(self.lib.fopis_unet_get_last(self.h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def unet_params(self, new=None):
        """The FP32 parameter vector; replaced by `new` when given."""
        n = C.c_int64()
        self._check(self.lib.fopis_unet_params(self.h, None, None, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        src = None
        if new is not None:
            src = np.ascontiguousarray(new, np.float32)
            assert src.size == n.value
        self._check(self.lib.fopis_unet_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)),
                                               None if src is None else src.ctypes.data_as(C.POINTER(C.c_float)),
                                               C.byref(n)))
        return out

    def unet_eval(self, rho0, phi1, phi2, phi_target=None, grads=True):
        """Prediction (glue layout), loss and parameter gradients on caller fields."""
        f = [np.ascontiguousarray(a, np.float64).ravel() for a in (rho0, phi1, phi2)]
        tgt = None if phi_target is None else np.ascontiguousarray(phi_target, np.float64).ravel()
        pred = np.zeros(f[0].size)
        n = C.c_int64()
        self._check(self.lib.fopis_unet_params(self.h, None, None, C.byref(n)))
        g = np.zeros(n.value, np.float32) if (grads and tgt is not None) else None
        loss = C.c_double()
        dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.fopis_unet_eval(self.h, dp(f[0]), dp(f[1]), dp(f[2]), dp(tgt), dp(pred),
                                             None if g is None else g.ctypes.data_as(C.POINTER(C.c_float)),
                                             C.byref(loss)))
        return pred.reshape(self.shape), loss.value, g

    def unet_tensor(self, which: int):
        """An activation / gradient buffer of the last evaluation (unknowns x channels)."""
        n = C.c_int64()
        self._check(self.lib.fopis_unet_tensor(self.h, which, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        self._check(self.lib.fopis_unet_tensor(self.h, which, out.ctypes.data_as(C.POINTER(C.c_float)), n.value,
                                               C.byref(n)))
        return out
