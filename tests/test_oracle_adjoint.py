"""CPU tests of the oracle's FP64 discrete adjoint of RK4 (orc_adjoint_rk4) against central finite
differences of the same forward computation: gradients of the final-state loss with respect to the
per-cell Ms map, the per-cell K1 map and the applied-field samples (demag + exchange + uniaxial
anisotropy + Zeeman, 20 steps). Tolerance 1e-5 relative (the finite differences are accurate to
~1e-7 at these step sizes)."""
import numpy as np
import pytest

from oracle_libs import orc_adjoint


def _case(seed=1, n=(10, 8, 1), nHa=4, steps=20, dt=1e-13):
    rng = np.random.default_rng(seed)
    N = int(np.prod(n))
    mesh = dict(n=n, h=(4e-9, 4e-9, 3e-9), Ms_map=8e5 * (1 + 0.1 * rng.normal(size=N)),
                K1_map=rng.uniform(0, 2e5, N), A=1.3e-11, alpha=0.02, Ha=rng.normal(0, 5e3, (nHa, 3)),
                Ha_tspan=steps * dt)
    m0 = rng.normal(size=(N, 3))
    m0 /= np.linalg.norm(m0, axis=1)[:, None]
    tgt = rng.normal(size=(N, 3))
    tgt /= np.linalg.norm(tgt, axis=1)[:, None]
    return mesh, m0, tgt, steps, dt


def _loss(mesh, m0, tgt, steps, dt, **over):
    return orc_adjoint(dict(mesh, **over), m0, tgt, steps, dt)[0]


def test_adjoint_gradients_match_central_differences():
    mesh, m0, tgt, steps, dt = _case()
    loss, gMs, gK, gHa = orc_adjoint(mesh, m0, tgt, steps, dt)
    assert np.isfinite(loss) and loss > 0
    for i in (0, 41, 79):
        e = 1e-4 * mesh["Ms_map"][i]
        a, b = mesh["Ms_map"].copy(), mesh["Ms_map"].copy()
        a[i] += e
        b[i] -= e
        fd = (_loss(mesh, m0, tgt, steps, dt, Ms_map=a) - _loss(mesh, m0, tgt, steps, dt, Ms_map=b)) / (2 * e)
        assert abs(gMs[i] - fd) <= 1e-5 * abs(fd)
    for i in (0, 13, 79):
        e = 200.0
        a, b = mesh["K1_map"].copy(), mesh["K1_map"].copy()
        a[i] += e
        b[i] -= e
        fd = (_loss(mesh, m0, tgt, steps, dt, K1_map=a) - _loss(mesh, m0, tgt, steps, dt, K1_map=b)) / (2 * e)
        assert abs(gK[i] - fd) <= 1e-5 * abs(fd)
    for j, c in ((0, 0), (2, 1), (3, 2)):
        e = 10.0
        a, b = mesh["Ha"].copy(), mesh["Ha"].copy()
        a[j, c] += e
        b[j, c] -= e
        fd = (_loss(mesh, m0, tgt, steps, dt, Ha=a) - _loss(mesh, m0, tgt, steps, dt, Ha=b)) / (2 * e)
        assert abs(gHa[j, c] - fd) <= 1e-5 * abs(fd)


def test_adjoint_without_demag_and_exchange():
    """Each field term on its own: gradients still agree (anisotropy + Zeeman only)."""
    mesh, m0, tgt, steps, dt = _case(seed=3, n=(6, 5, 1))
    mesh = dict(mesh, modules=8 | 16)
    loss, gMs, gK, gHa = orc_adjoint(mesh, m0, tgt, steps, dt)
    i = 7
    e = 1e-4 * mesh["Ms_map"][i]
    a, b = mesh["Ms_map"].copy(), mesh["Ms_map"].copy()
    a[i] += e
    b[i] -= e
    fd = (_loss(mesh, m0, tgt, steps, dt, Ms_map=a) - _loss(mesh, m0, tgt, steps, dt, Ms_map=b)) / (2 * e)
    assert abs(gMs[i] - fd) <= 1e-5 * abs(fd)
