"""The parity-split 3D z pass (demag.cu k_zmid_par: each pencil's even and odd kz in two threads of
two warp groups, the inverse halves added through shared memory) on cuda:0, selected explicitly
(BM_TILES / BM_Z_XV=1) and checked against the oracle: H_demag FP64 1e-9 and mixed 1e-5 of
max |H_ref| for every Nz it has (12, 16, 24, 32, 48, 64; nz from 5 to 32, so the rows past nz in
the padded input are exercised), tile widths 8 and 16 (at 8, threads past the six (component,
pencil) rows idle in each group), column counts that are not a multiple of the width,
self-mirrored pencils (ky = 0 and Ny / 2) and the packed kx = 0 column; RK4 steps FP64 1e-9 of Ms."""
import numpy as np
import pytest

from oracle_libs import orc_hdemag, sphere_random, OracleSolver

pytestmark = pytest.mark.gpu

CASES = [
    ((12, 10, 5), 8),      # Nz = 12, nz = 5; 12 packed x columns: a partial last tile
    ((20, 12, 7), 8),      # Nz = 16, nz = 7
    ((20, 8, 9), 16),      # Nz = 24; 24 packed x columns: a partial last tile
    ((16, 16, 16), 16),    # Nz = 32, nz = 16 (every input row present)
    ((10, 6, 17), 8),      # Nz = 48, nz = 17
    ((8, 4, 32), 8),       # Nz = 64, nz = 32
]


def _force(monkeypatch, W):
    monkeypatch.setenv("BM_TILES", "2,4,%d,1" % W)
    monkeypatch.setenv("BM_Z_XV", "1")


@pytest.mark.parametrize("n,W", CASES)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_zpar_hdemag(bm, monkeypatch, n, W, prec):
    _force(monkeypatch, W)
    h = (3e-9, 2e-9, 2.5e-9)
    N = int(np.prod(n))
    M = sphere_random(N, seed=900 + N, Ms=8e5)
    Href, _ = orc_hdemag(M, n, h)
    with bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_m(M)
        H = c.demag_field()
        t = c.tiles()
    assert t["zmid_zv"] == 1 and t["zmid_W"] == W, t
    tol = 1e-9 if prec == "fp64" else 1e-5
    assert np.abs(H - Href).max() / np.abs(Href).max() < tol


def test_zpar_rk4_steps(bm, monkeypatch):
    _force(monkeypatch, 16)
    mesh = dict(n=(24, 20, 12), h=(3e-9, 3e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(1e3, 0, 0))
    N = int(np.prod(mesh["n"]))
    M = sphere_random(N, seed=11, Ms=8e5)
    s = OracleSolver([mesh], evaluation=0, dt=1e-13)
    s.set_m(M)
    s.run(12)
    mref = s.get_m()
    s.close()
    from test_gpu_step import _make
    c = _make(bm, "fp64", mesh, M, "RK4", 1e-13)
    c.run(12)
    assert c.tiles()["zmid_zv"] == 1
    m = c.get_m()
    c.close()
    assert np.abs(m - mref).max() / 8e5 < 1e-9
