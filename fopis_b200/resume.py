"""Resume data and the capacity-matrix cache in the named-dataset files the C++
host writes (fopis_b200/host/datafile.hpp), for the Python host:

* ``resume/environment.bin``: dx, dt, timestep (Environment::saveInfo /
  loadInfo, src/Misc/Environment.cpp:379-438; a dx or dt that differs from
  the run's is rejected with ValueError, as the reference throws
  std::invalid_argument);
* ``resume/grid_id_0.bin``: per species ``<name>/size``, ``x`` .. ``vz``,
  ``generated_counts``, ``injection_carry``; ``Potential/phi``;
  ``Efield/exref`` ..; ``<object>/charge_map`` (RootGrid::saveResumeData /
  loadResumeData, src/Grid/RootGrid/RootGridIO.cpp:25-290);
* ``resume/objects/<file>.bin``: capacity_matrix, grid_spacing, time_spacing
  (IO::writeCmatrixData / loadCmatrixData, src/Misc/IO.cpp:28-120; valid only
  when the size, dx and dt match, IO.cpp:88-90).

File layout: magic ``FOPISDS1``, uint32 dataset count, then per dataset a
uint16 name length and name, uint8 element type (1 float64, 2 int64), uint8
rank, rank uint64 extents, uint64 payload bytes and the payload; a trailing
uint64 checksum of everything before it (the bytes as zero-padded 8-byte words
w_i: sum_i w_i (2i + 1) + byte count, modulo 2^64). All little-endian.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
from pathlib import Path
from typing import Dict

import numpy as np

from . import _abi

MAGIC = b"FOPISDS1"
F64, I64 = 1, 2


class CorruptFile(ValueError):
    pass


def checksum(data: bytes) -> int:
    """The file checksum: the bytes as zero-padded little-endian 8-byte words
    w_i, sum_i w_i (2i + 1) + byte count, modulo 2^64."""
    n = len(data)
    pad = (-n) % 8
    w = np.frombuffer(data + b"\0" * pad, dtype="<u8")
    k = np.arange(len(w), dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    with np.errstate(over="ignore"):
        return int((np.sum(w * k, dtype=np.uint64) + np.uint64(n)) & np.uint64(0xFFFFFFFFFFFFFFFF))


def write(path, sets: Dict[str, np.ndarray]) -> None:
    out = bytearray(MAGIC)
    out += struct.pack("<I", len(sets))
    for name in sorted(sets):
        a = np.asarray(sets[name])
        kind = I64 if a.dtype.kind in "iu" else F64
        a = np.asarray(a, dtype="<i8" if kind == I64 else "<f8")     # keeps 0-d scalars at rank 0
        nb = name.encode()
        out += struct.pack("<H", len(nb)) + nb + struct.pack("<BB", kind, a.ndim)
        out += b"".join(struct.pack("<Q", d) for d in a.shape)
        payload = a.tobytes()
        out += struct.pack("<Q", len(payload)) + payload
    out += struct.pack("<Q", checksum(bytes(out)))
    Path(path).write_bytes(bytes(out))


def read(path) -> Dict[str, np.ndarray]:
    b = Path(path).read_bytes()
    if len(b) < 20 or b[:8] != MAGIC:
        raise CorruptFile(f"corrupt data file {path}: bad magic")
    (stored,) = struct.unpack("<Q", b[-8:])
    if checksum(b[:-8]) != stored:
        raise CorruptFile(f"corrupt data file {path}: checksum mismatch")
    pos, end = 8, len(b) - 8

    def take(fmt):
        nonlocal pos
        n = struct.calcsize(fmt)
        if end - pos < n:
            raise CorruptFile(f"corrupt data file {path}: truncated")
        v = struct.unpack_from(fmt, b, pos)
        pos += n
        return v

    (count,) = take("<I")
    out = {}
    for _ in range(count):
        (ln,) = take("<H")
        if end - pos < ln:
            raise CorruptFile(f"corrupt data file {path}: truncated")
        name = b[pos:pos + ln].decode()
        pos += ln
        kind, rank = take("<BB")
        if kind not in (F64, I64):
            raise CorruptFile(f"corrupt data file {path}: element type")
        dims = take("<" + "Q" * rank) if rank else ()
        (nbytes,) = take("<Q")
        if nbytes > end - pos or nbytes != 8 * int(np.prod(dims, dtype=np.int64)):
            raise CorruptFile(f"corrupt data file {path}: extents")
        a = np.frombuffer(b, dtype="<i8" if kind == I64 else "<f8", count=nbytes // 8, offset=pos).reshape(dims)
        pos += nbytes
        out[name] = a.copy()
    if pos != end:
        raise CorruptFile(f"corrupt data file {path}: trailing bytes")
    return out


# ---------------------------------------------------------------- RootGrid helpers
def cmatrix_file(resume_dir, obj) -> Path:
    return Path(resume_dir) / "objects" / f"{getattr(obj, 'file_name', None) or obj.name}.bin"


def write_cmatrix(grid, k: int, resume_dir) -> None:
    """IO::writeCmatrixData for object k of a fopis_b200.RootGrid."""
    cfg = grid.cfg
    Cm = grid.get_cmatrix(k)
    os.makedirs(Path(resume_dir) / "objects", exist_ok=True)
    write(cmatrix_file(resume_dir, cfg.objects[k]),
          {"capacity_matrix": Cm, "grid_spacing": np.float64(cfg.dx), "time_spacing": np.float64(cfg.dt)})


def load_cmatrix(grid, k: int, resume_dir) -> bool:
    """IO::loadCmatrixData: sets object k's matrix from the cache when its size,
    dx and dt match; False (nothing set) otherwise."""
    cfg = grid.cfg
    f = cmatrix_file(resume_dir, cfg.objects[k])
    if not f.exists():
        return False
    try:
        d = read(f)
    except CorruptFile:
        return False
    n = len(cfg.objects[k].nodes)
    Cm = d.get("capacity_matrix")
    if Cm is None or Cm.shape != (n, n):
        return False
    if float(d["grid_spacing"]) != cfg.dx or float(d["time_spacing"]) != cfg.dt:
        return False
    grid.set_cmatrix(k, Cm)
    return True


def save_info(cfg, timestep: int, resume_dir) -> None:
    os.makedirs(resume_dir, exist_ok=True)
    write(Path(resume_dir) / "environment.bin",
          {"dx": np.float64(cfg.dx), "dt": np.float64(cfg.dt), "timestep": np.int64(timestep)})


def load_info(cfg, resume_dir) -> int:
    f = Path(resume_dir) / "environment.bin"
    if not f.exists():
        raise ValueError(f"[ERROR] resume file_name {f} does not exist.")
    d = read(f)
    if float(d["dx"]) != cfg.dx:
        raise ValueError(f"[ERROR] dx {float(d['dx'])} in the resume data does not match the dx {cfg.dx} from input.json.")
    if float(d["dt"]) != cfg.dt:
        raise ValueError(f"[ERROR] dt {float(d['dt'])} in the resume data does not match the dt {cfg.dt} from input.json.")
    return int(d["timestep"])


EM_SETS = ("Efield/ex", "Efield/ey", "Efield/ez", "Bfield/bx", "Bfield/by", "Bfield/bz")


def save_resume(grid, resume_dir) -> None:
    """Environment::saveInfo + RootGrid::saveResumeData for a fopis_b200.RootGrid."""
    cfg = grid.cfg
    nsp = cfg.params.nspecies
    lib = grid.lib
    carry = np.zeros(6 * nsp)
    grid._check(lib.fopis_get_injection_carry(grid.h, carry.ctypes.data_as(C.POINTER(C.c_double)), 6 * nsp))
    ts = int(grid.stats().timestep)
    sets = {}
    for s, sp in enumerate(cfg.species):
        r = grid.getParticles(s)
        g = sp.name + "/"
        sets[g + "size"] = np.float64(len(r))
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            sets[g + k] = np.ascontiguousarray(r[k])
        sets[g + "generated_counts"] = np.array([cfg.params.seed, ts], np.int64)
        sets[g + "injection_carry"] = carry[6 * s:6 * s + 6]
    sets["Potential/phi"] = grid.getPhi()
    ex, ey, ez = grid.getEref()
    sets["Efield/exref"], sets["Efield/eyref"], sets["Efield/ezref"] = ex, ey, ez
    if cfg.params.solver == _abi.SOLVER_EM:
        # RootGrid::saveResumeFieldData (RootGridIO.cpp:236-271): the Yee E and B
        for name, which in zip(EM_SETS, range(_abi.FIELD_EX, _abi.FIELD_BZ + 1)):
            sets[name] = grid.get_field(which)
    for k, o in enumerate(cfg.objects):
        sets[o.name + "/charge_map"] = grid.getChargeMap(k)
    os.makedirs(resume_dir, exist_ok=True)
    write(Path(resume_dir) / "grid_id_0.bin", sets)
    save_info(cfg, ts, resume_dir)


def load_resume(grid, resume_dir) -> int:
    """Environment::loadInfo + RootGrid::loadResumeData + Grid::initializeForLoad
    into a fresh fopis_b200.RootGrid whose objects already hold their capacity
    matrices; returns the timestep the run continues from."""
    from . import PARTICLE_DTYPE
    cfg = grid.cfg
    ts = load_info(cfg, resume_dir)
    d = read(Path(resume_dir) / "grid_id_0.bin")
    nsp = cfg.params.nspecies
    lib = grid.lib
    grid._check(lib.fopis_set_timestep(grid.h, ts))
    carry = np.zeros(6 * nsp)
    for s, sp in enumerate(cfg.species):
        g = sp.name + "/"
        n = int(d[g + "size"])
        if n:
            r = np.zeros(n, PARTICLE_DTYPE)
            for k in ("x", "y", "z", "vx", "vy", "vz"):
                r[k] = d[g + k]
            r["typeId"] = s
            r["isValid"] = 1
            grid.load_particles(s, r)
        if g + "injection_carry" in d:
            carry[6 * s:6 * s + 6] = d[g + "injection_carry"]
    grid._check(lib.fopis_set_injection_carry(grid.h, carry.ctypes.data_as(C.POINTER(C.c_double)), 6 * nsp))
    grid.set_field(_abi.FIELD_PHI, d["Potential/phi"])
    em = cfg.params.solver == _abi.SOLVER_EM
    if em:   # RootGrid::loadResumeFieldData (RootGridIO.cpp:181-234)
        for name, which in zip(EM_SETS, range(_abi.FIELD_EX, _abi.FIELD_BZ + 1)):
            grid.set_field(which, d[name])
    for k, o in enumerate(cfg.objects):
        cm = np.ascontiguousarray(d[o.name + "/charge_map"], np.float64)
        grid._check(lib.fopis_set_charge_map(grid.h, grid.object_ids[k], cm.ctypes.data_as(C.POINTER(C.c_double)),
                                             cm.size))
    # Grid::initializeForLoad (Grid.cpp:38-50)
    if em:
        grid.sort()
        grid.updateRho()
        grid.updateReferenceFields()
        return ts
    grid.updateEfield()
    grid.sort()
    grid.updateRho()
    return ts
