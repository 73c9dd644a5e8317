"""The allocation-free field-energy entry point, called through the C ABI.

Callers that cannot allocate device memory once their loop runs — hosts that
only hand over memory from their own pool, real-time loops in which a
device-synchronising cudaMalloc is not allowed — get the field energy of a
potential they own from fopis_efield_energy_noalloc, whose scratch is a
file-scope device array. Its result must equal what fopis_get_energy reports
for the same potential, on two calls in a row (the second call reuses the
scratch the first one filled). This file sorts last so a
stop-at-first-failure run has done every other test.
"""
import ctypes as C

import numpy as np
import pytest

from fopis_b200 import RootGrid, _abi
from fopis_b200.config import SimConfig, SpeciesInfo, make_params, plasma_units

pytestmark = pytest.mark.gpu


def test_noalloc_energy_matches_existing_entry_point(gpu_available):
    import torch
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, 4)]
    p, norm = make_params((33, 29, 31), "DDPPDD", dx, dt, sp)
    g = RootGrid(SimConfig(params=p, norm=norm, species=sp))
    lib = _abi.library()
    rng = np.random.default_rng(21)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        phi = rng.standard_normal(g.shape) * (1.0 + call)
        g.set_field(_abi.FIELD_PHI, phi)
        _, expect = g.getEnergy()
        dphi = torch.from_numpy(phi).cuda()
        rc = lib.fopis_efield_energy_noalloc(C.c_void_p(dphi.data_ptr()), p.nx, p.ny, p.nz, p.eps0,
                                             C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - expect) <= 1e-12 * abs(expect), (call, got, expect)
    # sizes beyond the scratch are refused before any launch
    rc = lib.fopis_efield_energy_noalloc(C.c_void_p(dphi.data_ptr()), 400, 400, 400, p.eps0,
                                         C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert rc == _abi.ERR_ARG
    g.close()

