"""The persistent 3D y passes fed by bulk tensor copies (ytma.cu: a two-stage shared-memory ring of
TMA loads completed on mbarriers) on cuda:0, selected explicitly (BM_TILES / BM_Y_XV=2) and checked
against the oracle: H_demag FP64 1e-9 and mixed 1e-5 of max |H_ref| over the transform lengths the
kernel has (Ny 8 .. 1024), odd cell counts (rows past the last box), several tile widths and column
counts that are not a multiple of the tile width; RK4 steps FP64 1e-9 of Ms."""
import numpy as np
import pytest

from oracle_libs import orc_hdemag, sphere_random, OracleSolver

pytestmark = pytest.mark.gpu

CASES = [
    ((8, 4, 2), 2),        # Ny = 8
    ((12, 7, 3), 4),       # Ny = 16, LX = 12 (a partial column tile)
    ((16, 16, 4), 8),      # Ny = 32
    ((30, 60, 3), 8),      # Ny = 128, LX = 32
    ((64, 100, 2), 4),     # ny = 100: one box of 100 rows forward; Ny = 256
    ((12, 200, 2), 8),     # Ny = 512, LX = 12: the second column tile half past the row end
    ((24, 400, 2), 8),     # ny = 400: a box of 256 rows and one reaching past the plane; Ny = 1024
    ((40, 512, 2), 8),     # Ny = 1024, inverse ring of two 64 KB tiles
    ((6, 8, 16), 2),       # Ny = 16, 16 planes
]


def _force(monkeypatch, W):
    monkeypatch.setenv("BM_TILES", "2,%d,8,1" % W)
    monkeypatch.setenv("BM_Y_XV", "2")


@pytest.mark.parametrize("n,W", CASES)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_ytma_hdemag(bm, monkeypatch, n, W, prec):
    if prec == "fp64" and n[1] > 256:
        W //= 2   # Ny = 1024 in FP64: the two-stage ring and the transpose tile fit 200 KB at W = 4
    _force(monkeypatch, W)
    h = (3e-9, 2e-9, 2.5e-9)
    N = int(np.prod(n))
    M = sphere_random(N, seed=500 + N, Ms=8e5)
    Href, _ = orc_hdemag(M, n, h)
    with bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_m(M)
        H = c.demag_field()
        t = c.tiles()
    assert t["ypass_yv"] == 2 and t["ypass_W"] == W, t
    tol = 1e-9 if prec == "fp64" else 1e-5
    assert np.abs(H - Href).max() / np.abs(Href).max() < tol


def test_ytma_rk4_steps(bm, monkeypatch):
    _force(monkeypatch, 8)
    mesh = dict(n=(32, 32, 4), h=(3e-9, 3e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(1e3, 0, 0))
    N = int(np.prod(mesh["n"]))
    M = sphere_random(N, seed=7, Ms=8e5)
    s = OracleSolver([mesh], evaluation=0, dt=1e-13)
    s.set_m(M)
    s.run(15)
    mref = s.get_m()
    s.close()
    from test_gpu_step import _make
    c = _make(bm, "fp64", mesh, M, "RK4", 1e-13)
    c.run(15)
    assert c.tiles()["ypass_yv"] == 2
    m = c.get_m()
    c.close()
    assert np.abs(m - mref).max() / 8e5 < 1e-9
