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


def test_noalloc_energy_replays_in_a_cuda_graph(gpu_available):
    """The stated purpose: the call recorded once under stream capture and replayed
    with the caller's potential changed in place, allocating nothing; each replay
    equals fopis_get_energy for the potential it saw."""
    import torch
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, 4)]
    p, norm = make_params((25, 27, 23), "DDDDPP", dx, dt, sp)
    g = RootGrid(SimConfig(params=p, norm=norm, species=sp))
    lib = _abi.library()
    rng = np.random.default_rng(5)
    dphi = torch.zeros(g.shape, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    # the first call of the context looks the scratch address up outside any capture
    assert lib.fopis_efield_energy_noalloc(C.c_void_p(dphi.data_ptr()), p.nx, p.ny, p.nz, p.eps0,
                                           C.c_void_p(out.data_ptr()), C.c_void_p(side.cuda_stream)) == 0
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        rc = lib.fopis_efield_energy_noalloc(C.c_void_p(dphi.data_ptr()), p.nx, p.ny, p.nz, p.eps0,
                                             C.c_void_p(out.data_ptr()), C.c_void_p(side.cuda_stream))
    assert rc == 0
    for call in range(2):
        phi = rng.standard_normal(g.shape) * (2.0 + call)
        dphi.copy_(torch.from_numpy(phi))
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        g.set_field(_abi.FIELD_PHI, phi)
        _, expect = g.getEnergy()
        got = float(out.item())
        assert abs(got - expect) <= 1e-12 * abs(expect), (call, got, expect)
    del graph
    g.close()
