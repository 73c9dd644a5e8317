"""Error paths of the C ABI on the GPU, each made on the host side or by
inputs that only overflow counters: none of them faults the device.

* a node's int64 fixed-point charge sum passing 2^64 (more than 2^13 full
  particle weights of one species on one node), in the deposit of
  RootGrid::updateRho (src/Grid/RootGrid/RootGridField.cpp:1153-1214) and in
  the fused step's brick push: FOPIS_DEV_RHO_OVERFLOW -> FOPIS_ERR_DEVICE;
* a solve that cannot reach its tolerance within the V-cycle cap (the
  reference's maximum_poisson_post_loop cap, RootGridField.cpp:65-103):
  FOPIS_ERR_NOT_CONVERGED after the warm start and the zero-start retry;
* NaN in rho written from the host: FOPIS_ERR_DEVICE with
  FOPIS_DEV_NONFINITE latched, and the next finite solve succeeds;
* more absorbed particles in one step than the absorbed list holds
  (Spacecraft::distributeInnerParticleCharge, Spacecraft.cpp:512-592):
  FOPIS_ERR_CAPACITY;
* the bounded mbarrier wait of the tensor-core kernels run out on purpose:
  status 1 instead of a hang."""
import ctypes as C

import numpy as np
import pytest

from fopis_b200 import PARTICLE_DTYPE, FopisError, RootGrid, _abi, config
from fopis_b200.config import SpeciesInfo, make_params, objects_from_boxes, plasma_units

from helpers import random_particles

pytestmark = pytest.mark.gpu


def plasma(n, boundary="PPPPPP", ppc=4, **kw):
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, ppc),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, ppc)]
    p, norm = make_params((n, n, n), boundary, dx, dt, sp, **kw)
    return config.SimConfig(params=p, norm=norm, species=sp)


def point_set(n, x, v):
    r = np.zeros(n, PARTICLE_DTYPE)
    r["x"], r["y"], r["z"] = x
    r["vx"], r["vy"], r["vz"] = v
    r["isValid"] = 1
    return r


def status(g):
    return int(g.stats().device_status)


def test_rho_overflow_in_update_rho(gpu_available):
    # 9000 particles at a node: 9000 * 2^51 > 2^64 on that node
    g = RootGrid(plasma(8, sort_interval=1000000))
    for s in range(2):
        g.load_particles(s, point_set(9000, (2.0, 2.0, 2.0), (0.0, 0.0, 0.0)))
    with pytest.raises(FopisError) as e:
        g.updateRho()
    assert e.value.code == _abi.ERR_DEVICE and "2^64" in str(e.value)
    assert status(g) & _abi.DEV_RHO_OVERFLOW
    g.close()


def test_rho_overflow_in_fused_step(gpu_available):
    # 8000 + 1000 particles: below 2^64 at initialize, 9000 full weights on one
    # node after the 1000 move onto it; electrons and ions coincide, so rho = 0,
    # E = 0 and nothing but the move changes the deposit
    g = RootGrid(plasma(8, sort_interval=1000000))
    for s in range(2):
        g.load_particles(s, np.concatenate([point_set(8000, (2.0, 2.0, 2.0), (0.0, 0.0, 0.0)),
                                            point_set(1000, (2.5, 2.5, 2.5), (-0.5, -0.5, -0.5))]))
    g.initialize()
    assert status(g) & _abi.DEV_RHO_OVERFLOW == 0
    with pytest.raises(FopisError) as e:
        g.mainLoopES(1)
    assert e.value.code == _abi.ERR_DEVICE
    assert status(g) & _abi.DEV_RHO_OVERFLOW
    g.close()


def test_solver_cap_reports_not_converged(gpu_available):
    cfg = plasma(16, tol=1e-12, max_vcycles=1, sort_interval=1000000)
    g = RootGrid(cfg)
    for s in range(2):
        g.load_particles(s, random_particles(16 ** 3 * 4, (0, 0, 0), (16, 16, 16), 0.1, 7 + s, species=s))
    rc = g.initialize()
    st = g.stats()
    assert rc == _abi.ERR_NOT_CONVERGED
    assert st.converged == 0 and st.residual_last > 1e-12
    assert st.vcycles_step >= 2        # the warm start, then the retry from zero (one V-cycle each at most)
    assert status(g) == 0              # not a device error: the run may go on
    assert g.mainLoopES(1) == _abi.ERR_NOT_CONVERGED
    g.close()


def test_nan_rho_reports_device_error(gpu_available):
    cfg = plasma(16, boundary="DDDDDD", sort_interval=1000000)
    g = RootGrid(cfg)
    rho = np.zeros(g.shape)
    rho[8, 8, 8] = 1.0
    rho[5, 9, 7] = np.nan
    g.set_field(_abi.FIELD_RHO0, rho)
    g.set_field(_abi.FIELD_PHI, np.zeros(g.shape))
    with pytest.raises(FopisError) as e:
        g.solvePoisson()
    assert e.value.code == _abi.ERR_DEVICE and "non-finite" in str(e.value)
    assert status(g) & _abi.DEV_NONFINITE
    rho[5, 9, 7] = 0.0
    g.set_field(_abi.FIELD_RHO0, rho)
    g.set_field(_abi.FIELD_PHI, np.zeros(g.shape))
    assert g.solvePoisson() == 0
    phi = g.getPhi()
    assert np.isfinite(phi).all() and phi[8, 8, 8] != 0.0
    g.close()


def test_absorbed_list_capacity(gpu_available):
    # more particles inside the body than the absorbed list's 2^20 entries
    cfg = plasma(17, boundary="DDDDDD", sort_interval=1000000)
    obj = objects_from_boxes([((-2, -2, -2), (2, 2, 2))], (17, 17, 17))
    cfg.objects = [obj]
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    n = (1 << 20) + 50000
    cells = obj.cells[np.arange(n) % len(obj.cells)]
    r = point_set(n, (cells[:, 0] - 0.5, cells[:, 1] - 0.5, cells[:, 2] - 0.5), (0.0, 0.0, 0.0))
    g.load_particles(0, r)
    with pytest.raises(FopisError) as e:
        g.initialize()
    assert e.value.code == _abi.ERR_CAPACITY
    assert status(g) & _abi.DEV_ABSORB_OVERFLOW
    g.close()


def test_bounded_wait_runs_out(gpu_available):
    lib = _abi.library()
    st = C.c_uint32(99)
    assert lib.fopis_check_bounded_wait(0, 1000, 0, C.byref(st)) == 0
    assert st.value == 1               # nothing arrived: the wait gave up and reported
    assert lib.fopis_check_bounded_wait(0, 1000, 1, C.byref(st)) == 0
    assert st.value == 0               # the phase completed
    # the device is still usable afterwards
    g = RootGrid(plasma(8))
    g.close()
