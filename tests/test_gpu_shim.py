"""The Boris-side shim (boris2_b200/shim: DemagB200, a ModulesCUDA in place of DemagCUDA, and ODEB200,
the setode / setdt / astepctrl / Iterate forwarder), built against the reference's own headers, driven
on a mesh whose M and Heff are the reference's cu_obj<cuVEC_VC<cuReal3>> / cu_obj<cuVEC<cuReal3>>
(FP32 cuBReal, the reference's default):

  * DemagB200::UpdateField adds the demag field into Heff (DemagCUDA::UpdateField,
    Boris/DemagCUDA.cpp:106-121): Heff after - Heff before equals bm_compute_hdemag of the same M in
    mixed precision to 1e-6 of max |H|, and its energy density to 1e-6
  * ODEB200 advances M in place: 12 RK4 steps give this library's own run of the same mesh (same
    precision, same kernel variants) to 1e-6 of Ms at the same time; 8 adaptive RKDP54 steps to 1e-4 of
    Ms and 1e-5 of the simulated time
"""
import ctypes
import os

import numpy as np
import pytest

from oracle_libs import sphere_random, tilted_z

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM_SO = os.path.join(ROOT, "boris2_b200", "shim", "_build", "libboris_shim.so")
P, D, I, DP = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)


def _dp(a):
    return a.ctypes.data_as(DP)


def shim():
    if not os.path.exists(SHIM_SO):
        pytest.skip("shim not built (boris2_b200/shim/Makefile needs the reference headers)")
    L = ctypes.CDLL(SHIM_SO)
    L.shim_demag_create.restype = P
    L.shim_demag_create.argtypes = [I, I, I, D, D, D, I]
    L.shim_demag_update.argtypes = [P, DP, DP, DP, DP]
    L.shim_demag_destroy.argtypes = [P]
    L.shim_demag_set_pbc.argtypes = [P, I, I, I, ctypes.POINTER(ctypes.c_int)]
    L.shim_ode_create.restype = P
    L.shim_ode_create.argtypes = [I, I, I, D, D, D, I]
    L.shim_ode_context.restype = P
    L.shim_ode_context.argtypes = [P]
    L.shim_ode_setode.argtypes = [P, I, D]
    L.shim_ode_astepctrl.argtypes = [P, D, D, D, D]
    L.shim_ode_set_m.argtypes = [P, DP]
    L.shim_ode_get_m.argtypes = [P, DP]
    L.shim_ode_iterate.argtypes = [P, I, DP]
    L.shim_ode_destroy.argtypes = [P]
    return L


@pytest.mark.parametrize("n", [(64, 32, 1), (32, 32, 8)])
def test_demag_module_adds_field(bm, n):
    L = shim()
    assert L.shim_real_bytes() == 4
    h = (3e-9, 3e-9, 2e-9)
    N = int(np.prod(n))
    M = np.ascontiguousarray(sphere_random(N, seed=5, Ms=8e5).reshape(-1))
    Hpre = np.ascontiguousarray(np.random.default_rng(1).normal(0, 1e3, 3 * N))
    H = np.zeros(3 * N)
    e = np.zeros(1)
    s = L.shim_demag_create(n[0], n[1], n[2], h[0], h[1], h[2], 0)
    assert s
    assert L.shim_demag_update(s, _dp(M), _dp(Hpre), _dp(H), _dp(e)) == 0
    L.shim_demag_destroy(s)
    c = bm.Context(precision=bm.MIXED)
    c.add_mesh(n, h)
    c.set_modules(0, bm.DEMAG)
    c.set_m(M.reshape(-1, 3))
    Href, eref = c.demag_field(with_energy=True)
    c.close()
    Hd = (H - Hpre).reshape(-1, 3)
    assert np.abs(Hd - Href).max() / np.abs(Href).max() < 1e-6
    assert abs(e[0] - eref) <= 1e-6 * abs(eref)


def test_demag_module_set_pbc(bm):
    """DemagB200::Set_PBC (DemagBase::Set_PBC) rebuilds the kernels with the images; the field equals the
    library's own periodic demag of the same M (mixed precision, 1e-6 of max |H|)."""
    L = shim()
    n, h, pbc = (32, 32, 2), (3e-9, 3e-9, 2e-9), (4, 4, 0)
    N = int(np.prod(n))
    M = np.ascontiguousarray(sphere_random(N, seed=6, Ms=8e5).reshape(-1))
    Hpre = np.zeros(3 * N)
    H = np.zeros(3 * N)
    e = np.zeros(1)
    s = L.shim_demag_create(n[0], n[1], n[2], h[0], h[1], h[2], 0)
    assert s
    got = (ctypes.c_int * 3)()
    assert L.shim_demag_set_pbc(s, pbc[0], pbc[1], pbc[2], got) == 0
    assert tuple(got) == pbc
    assert L.shim_demag_update(s, _dp(M), _dp(Hpre), _dp(H), _dp(e)) == 0
    L.shim_demag_destroy(s)
    c = bm.Context(precision=bm.MIXED)
    c.add_mesh(n, h)
    c.set_modules(0, bm.DEMAG)
    c.set_pbc(0, pbc)
    c.set_m(M.reshape(-1, 3))
    Href = c.demag_field()
    c.close()
    assert np.abs(H.reshape(-1, 3) - Href).max() / np.abs(Href).max() < 1e-6


@pytest.mark.parametrize("evaluation,steps", [("RK4", 12), ("RKDP54", 8)])
def test_ode_forwarder_advances_mesh(bm, evaluation, steps, monkeypatch):
    # both contexts on the same kernel variants (independent tuning may pick transforms that round
    # differently in FP32, and RKDP54's step control follows such differences)
    monkeypatch.setenv("BM_TILES", "1,8,8,1")
    L = shim()
    n, h = (32, 24, 4), (2e-9, 2e-9, 2e-9)
    N = int(np.prod(n))
    M = np.ascontiguousarray(tilted_z(N, seed=9, Ms=1.1e6).reshape(-1))
    s = L.shim_ode_create(n[0], n[1], n[2], h[0], h[1], h[2], 0)
    assert s
    ctx = L.shim_ode_context(s)
    lib = bm.lib()
    ea = (ctypes.c_double * 3)(0, 0, 1)
    assert lib.bm_set_material(ctx, 0, 1.1e6, 1.5e-11, 0.1, 1.0, 5e5, 0.0, ea, 1.5e-3) == 0
    assert lib.bm_set_modules(ctx, 0, bm.DEMAG | bm.IDMI | bm.ANIUNI) == 0
    ev = 1 if evaluation == "RKDP54" else 0
    assert L.shim_ode_setode(s, ev, 1e-14) == 0
    if ev:
        L.shim_ode_astepctrl(s, 1e-5, 2.0, 1e-15, 3e-12)
    L.shim_ode_set_m(s, _dp(M))
    t = np.zeros(1)
    rc = L.shim_ode_iterate(s, steps, _dp(t))
    assert rc == 0, bm.lib().bm_last_error().decode()
    Mout = np.zeros(3 * N)
    L.shim_ode_get_m(s, _dp(Mout))
    L.shim_ode_destroy(s)
    c = bm.Context(precision=bm.MIXED)
    c.add_mesh(n, h)
    c.set_material(0, Ms=1.1e6, A=1.5e-11, alpha=0.1, K1=5e5, ea=(0, 0, 1), D=1.5e-3)
    c.set_modules(0, bm.DEMAG | bm.IDMI | bm.ANIUNI)
    c.setode(evaluation, 1e-14)
    if ev:
        c.astepctrl(1e-5, 2.0, 1e-15, 3e-12)
    c.set_m(M.reshape(-1, 3))
    st = c.run(steps)
    ref = c.get_m()
    c.close()
    if ev:
        # RKDP54: the cuVEC's FP32 copy of M and this library's own rounding may differ by an ulp in a
        # cell, which moves the adaptive steps slightly
        assert abs(t[0] - st["time"]) <= 1e-5 * st["time"]
        assert np.abs(Mout.reshape(-1, 3) - ref).max() / 1.1e6 < 1e-4
    else:
        assert abs(t[0] - st["time"]) <= 1e-12 * st["time"]
        assert np.abs(Mout.reshape(-1, 3) - ref).max() / 1.1e6 < 1e-6
