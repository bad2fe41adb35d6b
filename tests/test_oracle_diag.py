"""The oracle's torque and dm/dt diagnostics (orc_solver_get_mxh / get_dmdt, restating the reference's
Get_mxh / Get_dmdt, Boris/DiffEq_CommonBase_Get.cpp:7,19) on CPU: 0 before any request, the value of
a requested step equal to the formula of the reference's reductions evaluated directly from the
solver's own state (max |M x Heff| / |M|^2 at the step start, Boris/DiffEqFM_Evals_RK4.cpp:78-80;
max |M - M_start| / (dT GAMMA |M|^2) after the step, :191-199), one request serving one step, and
meshes with grel = 0 left out."""
import numpy as np
import pytest

from oracle_libs import OracleSolver, tilted_z

GAMMA = 2.212761569e5
MESH = dict(n=(12, 10, 3), h=(3e-9, 3e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, K1=2e5, modules=1 | 2 | 8 | 16,
            Ha=(1e3, 2e3, 0))


def _mxh(M, H):
    return (np.linalg.norm(np.cross(M, H), axis=1) / (M * M).sum(axis=1)).max()


def _dmdt(M, M1, dT):
    return (np.linalg.norm(M - M1, axis=1) / (dT * GAMMA * (M * M).sum(axis=1))).max()


@pytest.mark.parametrize("evaluation", [0, 1])
def test_oracle_diag_formula(evaluation):
    N = int(np.prod(MESH["n"]))
    M0 = tilted_z(N, seed=3, Ms=8e5)
    dt = 2e-14
    kw = dict(tol=1e-5, dT_incr=2.0, dT_min=dt, dT_max=dt) if evaluation == 1 else {}
    s = OracleSolver([MESH], evaluation=evaluation, dt=dt, **kw)
    s.set_m(M0)
    assert s.get_mxh() == 0.0 and s.get_dmdt() == 0.0   # nothing computed yet; both now requested
    H0 = s.heff()
    s.run(1)
    M1 = s.get_m()
    assert abs(s.get_mxh() / _mxh(M0, H0) - 1) < 1e-12
    assert abs(s.get_dmdt() / _dmdt(M1, M0, dt) - 1) < 1e-12
    # requested again by the calls above: the next step serves them; the one after computes nothing
    H1 = s.heff()
    s.run(2)
    assert abs(s.get_mxh() / _mxh(M1, H1) - 1) < 1e-12
    s.close()


def test_oracle_diag_grel_zero_left_out():
    N = int(np.prod(MESH["n"]))
    frozen = dict(MESH, grel=0.0, Ha=(1e6, 0, 0))   # a large torque that must not count
    s = OracleSolver([MESH, frozen], evaluation=0, dt=2e-14)
    M0 = tilted_z(N, seed=5, Ms=8e5)
    s.set_m(M0, 0)
    s.set_m(tilted_z(N, seed=6, Ms=8e5), 1)
    s.get_mxh()
    H0 = s.heff(0)
    s.run(1)
    assert abs(s.get_mxh() / _mxh(M0, H0) - 1) < 1e-12
    s.close()
