"""ctypes mirror of include/fopis_gpu.h and the loader of libfopis_gpu.so.

The library is built in-tree (``fopis_b200/libfopis_gpu.so``). Loading fails
with an ImportError that names the build step when it is missing: there is no
fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

MAX_SPECIES = 8
MAX_OBJECTS = 8

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_NOMEM = -3
ERR_STATE = -4
ERR_NOT_CONVERGED = -5
ERR_DEVICE = -6
ERR_CAPACITY = -7
ERR_NO_CUDA = -8

DEV_PARTICLE_OVERFLOW = 0x1
DEV_ABSORB_OVERFLOW = 0x2
DEV_BAD_CMAT_NODE = 0x4
DEV_SURFACE_NOT_FOUND = 0x8
DEV_INJECT_REJECTS = 0x10
DEV_NONFINITE = 0x20
DEV_RHO_OVERFLOW = 0x40

SPECIES_AMBIENT = 0
SPECIES_PHOTOELECTRON = 1
SPECIES_SECONDARY = 2
INCIDENT_DOUBLES = 10
MIXED = 0
FP64 = 1
GUESS_ZERO = 0
GUESS_WARM = 1
GUESS_LEARNED = 2
GUESS_HISTORY = 3
SOLVER_ES = 0
SOLVER_EM = 1

FIELD_PHI = 0
FIELD_RHO0 = 1
FIELD_EXREF = 2
FIELD_EYREF = 3
FIELD_EZREF = 4
FIELD_BXREF = 5
FIELD_BYREF = 6
FIELD_BZREF = 7
FIELD_JXREF = 8
FIELD_JYREF = 9
FIELD_JZREF = 10
FIELD_RHO_SPECIES = 16
FIELD_EX = 32
FIELD_EY = 33
FIELD_EZ = 34
FIELD_BX = 35
FIELD_BY = 36
FIELD_BZ = 37
FIELD_JX = 38
FIELD_JY = 39
FIELD_JZ = 40


class Species(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("particle_per_cell", C.c_int),
        ("charge", C.c_double),
        ("mass", C.c_double),
        ("size", C.c_double),
        ("thermal_velocity", C.c_double),
        ("deviation", C.c_double),
        ("drift", C.c_double * 3),
        ("injection_axis", C.c_int * 6),
        ("flux", C.c_double * 6),
        ("emission_amount", C.c_double),
    ]


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("nz", C.c_int),
        ("boundary", C.c_char * 8),
        ("eps0", C.c_double),
        ("static_bfield", C.c_double * 3),
        ("shine_vector", C.c_double * 3),
        ("nspecies", C.c_int),
        ("species", Species * MAX_SPECIES),
        ("poisson_tol", C.c_double),
        ("max_vcycles", C.c_int),
        ("guess_mode", C.c_int),
        ("sort_interval", C.c_int),
        ("remove_interval", C.c_int),
        ("capacity_factor", C.c_double),
        ("precision", C.c_int),
        ("solver", C.c_int),
        ("seed", C.c_uint64),
        ("energy_ev", C.c_double),
        ("mu0", C.c_double),
    ]


class ObjectDesc(C.Structure):
    _fields_ = [
        ("n_cmat", C.c_int),
        ("cmat_nodes", C.POINTER(C.c_int32)),
        ("n_cells", C.c_int),
        ("cells", C.POINTER(C.c_int32)),
        ("is_potential_fixed", C.c_int),
        ("fixed_potential", C.c_double),
        ("initial_potential_offset", C.c_double),
        ("emit_species", C.c_int),
        ("secondary_species", C.c_int),
        ("dielectric", C.c_int),
        ("capacitance", C.POINTER(C.c_double)),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("timestep", C.c_int64),
        ("vcycles_last", C.c_int),
        ("vcycles_step", C.c_int),
        ("solves_step", C.c_int),
        ("converged", C.c_int),
        ("residual_last", C.c_double),
        ("residual_initial", C.c_double),
        ("num_particles", C.c_int64 * MAX_SPECIES),
        ("capacity", C.c_int64 * MAX_SPECIES),
        ("absorbed_step", C.c_int64),
        ("injected_step", C.c_int64),
        ("emitted_step", C.c_int64),
        ("device_status", C.c_uint32),
        ("learned_used", C.c_int),
        ("ms_phase", C.c_double * 8),
        ("kernel_launches", C.c_int64),
        ("solve_mode", C.c_int),
        ("pad", C.c_int),
        ("residual_pointwise", C.c_double),
        ("valid_particles", C.c_int64 * MAX_SPECIES),
        ("pushed_step", C.c_int64 * MAX_SPECIES),
    ]


# Every exported entry point: name -> (restype, argtypes).
_VP = C.c_void_p
_DP = C.POINTER(C.c_double)
SIGNATURES = {
    "fopis_create": (C.c_int, [C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)]),
    "fopis_destroy": (None, [_VP]),
    "fopis_last_error": (C.c_char_p, [_VP]),
    "fopis_version": (C.c_char_p, []),
    "fopis_add_object": (C.c_int, [_VP, C.POINTER(ObjectDesc), C.POINTER(C.c_int)]),
    "fopis_build_capacity_matrix": (C.c_int, [_VP, C.c_int]),
    "fopis_set_capacity_matrix": (C.c_int, [_VP, C.c_int, _DP, C.c_int]),
    "fopis_get_capacity_matrix": (C.c_int, [_VP, C.c_int, _DP, C.c_int]),
    "fopis_get_object": (C.c_int, [_VP, C.c_int, _DP, _DP, _DP]),
    "fopis_get_charge_map": (C.c_int, [_VP, C.c_int, _DP, C.c_int]),
    "fopis_load_particles": (C.c_int, [_VP, C.c_int, _VP, C.c_int64]),
    "fopis_get_particles": (C.c_int, [_VP, C.c_int, _VP, C.c_int64, C.POINTER(C.c_int64)]),
    "fopis_get_particles_raw": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP, _VP, _VP, _VP, _VP, C.c_int64,
                                          C.POINTER(C.c_int64)]),
    "fopis_generate_ambient": (C.c_int, [_VP]),
    "fopis_sort_particles": (C.c_int, [_VP]),
    "fopis_initialize": (C.c_int, [_VP]),
    "fopis_step": (C.c_int, [_VP, C.c_int]),
    "fopis_update_velocity": (C.c_int, [_VP]),
    "fopis_emit_particles": (C.c_int, [_VP]),
    "fopis_update_position": (C.c_int, [_VP]),
    "fopis_inject_particles": (C.c_int, [_VP]),
    "fopis_update_rho": (C.c_int, [_VP]),
    "fopis_solve_poisson": (C.c_int, [_VP]),
    "fopis_update_efield": (C.c_int, [_VP]),
    "fopis_update_bfield": (C.c_int, [_VP]),
    "fopis_update_reference_fields": (C.c_int, [_VP]),
    "fopis_field_shape": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fopis_get_bfield_energy": (C.c_int, [_VP, _DP]),
    "fopis_remove_invalid_particles": (C.c_int, [_VP]),
    "fopis_advance_timestep": (C.c_int, [_VP]),
    "fopis_get_field": (C.c_int, [_VP, C.c_int, _DP, C.c_size_t]),
    "fopis_set_field": (C.c_int, [_VP, C.c_int, _DP, C.c_size_t]),
    "fopis_get_energy": (C.c_int, [_VP, _DP, _DP]),
    "fopis_get_stats": (C.c_int, [_VP, C.POINTER(Stats)]),
    "fopis_set_guess_mode": (C.c_int, [_VP, C.c_int]),
    "fopis_get_stream": (C.c_int, [_VP, C.POINTER(C.c_void_p)]),
    "fopis_unet_set_training": (C.c_int, [_VP, C.c_int, C.c_double]),
    "fopis_unet_get_state": (C.c_int, [_VP, _DP, C.POINTER(C.c_int64)]),
    "fopis_unet_get_policy": (C.c_int, [_VP, _DP, _DP, C.POINTER(C.c_int)]),
    "fopis_unet_get_last": (C.c_int, [_VP, _DP, _DP, _DP, _DP]),
    "fopis_unet_eval": (C.c_int, [_VP, _DP, _DP, _DP, _DP, _DP, C.POINTER(C.c_float), _DP]),
    "fopis_unet_params": (C.c_int, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int64)]),
    "fopis_unet_tensor": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_float), C.c_int64, C.POINTER(C.c_int64)]),
    "fopis_parse_obj": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_int32)),
                                  C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.c_int)]),
    "fopis_set_charge_map": (C.c_int, [_VP, C.c_int, _DP, C.c_int]),
    "fopis_set_timestep": (C.c_int, [_VP, C.c_int64]),
    "fopis_get_injection_carry": (C.c_int, [_VP, _DP, C.c_int]),
    "fopis_set_injection_carry": (C.c_int, [_VP, _DP, C.c_int]),
    "fopis_free": (None, [_VP]),
    "fopis_check_bounded_wait": (C.c_int, [C.c_int, C.c_uint32, C.c_int, C.POINTER(C.c_uint32)]),
    "fopis_efield_energy_noalloc": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, C.c_double, _VP, _VP]),
    "fopis_get_incidents": (C.c_int, [_VP, _DP, C.c_int64, C.POINTER(C.c_int64)]),
    "fopis_set_incidents": (C.c_int, [_VP, _DP, C.c_int64]),
    "fopis_parse_obj_textures": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_int32)),
                                           C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.c_int)]),
}

LIB_PATH = Path(__file__).resolve().parent / "libfopis_gpu.so"
_lib = None


def library() -> C.CDLL:
    """Loads libfopis_gpu.so (built by ``make -C fopis_b200``); raises ImportError if absent."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("FOPIS_GPU_LIB", LIB_PATH))
    if not path.exists():
        raise ImportError(f"{path} is missing: build it with `make -C fopis_b200` (nvcc, sm_100a)")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class FopisError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"fopis status {code}: {message}")
        self.code = code
