"""Error paths of the C ABI on cuda:0: invalid sizes, cellsizes and settings are refused with the
documented codes (the reference returns a BError instead of running), nothing runs for them, and the
context stays usable afterwards: the same small RK4 run still matches the oracle (FP64, 1e-9 of Ms)."""
import ctypes

import numpy as np
import pytest

from oracle_libs import OracleSolver, sphere_random

pytestmark = pytest.mark.gpu

EINVAL, ESTATE, EUNSUPPORTED = 1, 4, 5


def _raw(bm, c):
    return bm.lib(), c._h


def test_invalid_meshes_and_settings_are_refused(bm):
    c = bm.Context(precision=bm.FP64)
    L, h = _raw(bm, c)
    mid = ctypes.c_int(-1)
    d = ctypes.c_double
    # empty and ragged dimensions, non-positive cellsizes, sizes beyond the supported FFT lengths
    assert L.bm_add_mesh(h, 0, 4, 1, d(1e-9), d(1e-9), d(1e-9), d(0), d(0), d(0), ctypes.byref(mid)) == EINVAL
    assert L.bm_add_mesh(h, 4, -1, 1, d(1e-9), d(1e-9), d(1e-9), d(0), d(0), d(0), ctypes.byref(mid)) == EINVAL
    assert L.bm_add_mesh(h, 4, 4, 1, d(0.0), d(1e-9), d(1e-9), d(0), d(0), d(0), ctypes.byref(mid)) == EINVAL
    assert L.bm_add_mesh(h, 4, 4, 1, d(1e-9), d(-1e-9), d(1e-9), d(0), d(0), d(0), ctypes.byref(mid)) == EINVAL
    assert L.bm_add_mesh(h, 5000, 4, 1, d(1e-9), d(1e-9), d(1e-9), d(0), d(0), d(0), ctypes.byref(mid)) == EUNSUPPORTED
    assert mid.value == -1
    # nothing to run yet
    st = bm.Stats()
    assert L.bm_run(h, 1, ctypes.byref(st)) == ESTATE
    # a valid mesh, then settings and indices that are refused
    c.add_mesh((12, 8, 1), (3e-9, 3e-9, 2e-9))
    assert L.bm_set_ode(h, 7, d(1e-13)) == EUNSUPPORTED
    assert L.bm_set_ode(h, bm.RK4, d(0.0)) == EINVAL
    assert L.bm_set_m(h, 3, None) == EINVAL            # bad mesh index
    assert L.bm_set_m(h, 0, None) == EINVAL            # null buffer
    assert L.bm_get_m(h, -1, None) == EINVAL
    assert L.bm_run(h, -2, ctypes.byref(st)) == EINVAL
    assert L.bm_last_error()                           # the reason is recorded
    c.close()


def test_context_usable_after_refused_calls(bm):
    mesh = dict(n=(12, 8, 1), h=(3e-9, 3e-9, 2e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16,
                Ha=(2e3, 0, 0))
    N = 12 * 8
    M = sphere_random(N, seed=11, Ms=8e5)
    s = OracleSolver([mesh], evaluation=0, dt=2e-14)
    s.set_m(M)
    s.run(10)
    c = bm.Context(precision=bm.FP64)
    L, h = _raw(bm, c)
    d = ctypes.c_double
    mid = ctypes.c_int(-1)
    assert L.bm_add_mesh(h, 0, 8, 1, d(3e-9), d(3e-9), d(2e-9), d(0), d(0), d(0), ctypes.byref(mid)) == EINVAL
    c.add_mesh(mesh["n"], mesh["h"])
    c.set_material(0, Ms=8e5, A=1.3e-11, alpha=0.3)
    c.set_modules(0, mesh["modules"])
    c.set_field(0, mesh["Ha"])
    assert L.bm_set_ode(h, bm.RK4, d(-1.0)) == EINVAL
    c.setode("RK4", 2e-14)
    c.set_m(M)
    st = bm.Stats()
    assert L.bm_run(h, -1, ctypes.byref(st)) == EINVAL
    assert c.run(0)["accepted"] == 0                   # zero steps: a no-op
    c.run(10)
    m = c.get_m()
    c.close()
    assert np.abs(m - s.get_m()).max() / 8e5 < 1e-9
