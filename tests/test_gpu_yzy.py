"""GPU parity of the fused y -> z -> y cluster pass (one thread-block-cluster kernel per field
evaluation of a 3D mesh, boris2_b200/csrc/yzy.cu) against the oracle's FP64 restatement of the
convolution and the RK4 trajectory.

Cases cover Ny 512 and 1024 (the two-level y splits 32 x 16 and 32 x 32), Nz 4 .. 32, a ny that fills
Ny / 2 and one that leaves zero rows, nz below Nz / 2, x lengths LX of 2^k and 3 * 2^k (the packed
kx = 0 column sits in the first tile), in mixed precision and in FP64. Tolerances: H_demag
max |H - H_ref| / max |H_ref| <= 1e-5 mixed, <= 1e-9 FP64; m after the run <= 1e-4 mixed, <= 1e-9 FP64.
"""
import numpy as np
import pytest

from oracle_libs import OracleSolver, orc_hdemag, sphere_random

pytestmark = pytest.mark.gpu

# (nx, ny, nz): Nz = 2 * (smallest 2^p or 3 * 2^p >= nz); LX = the same rounding of nx
CASES = [
    ((8, 256, 2), "mixed"), ((12, 250, 6), "mixed"), ((16, 512, 4), "mixed"), ((8, 509, 7), "mixed"),
    ((24, 256, 16), "mixed"), ((4, 512, 16), "mixed"), ((12, 400, 11), "mixed"), ((8, 256, 5), "fp64"),
    ((12, 512, 8), "fp64"),
]


def _ctx(bm, prec, n, M):
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    c.add_mesh(n, (3e-9, 3e-9, 2e-9))
    c.set_material(0, Ms=8e5, A=1.3e-11, alpha=0.3)
    c.set_modules(0, bm.DEMAG | bm.EXCH | bm.ZEEMAN)
    c.set_field(0, (2e3, 1e3, 0))
    c.setode("RK4", 2e-14)
    c.set_m(M)
    return c


@pytest.mark.parametrize("n,prec", CASES, ids=["%dx%dx%d-%s" % (c[0] + (c[1],)) for c in CASES])
def test_yzy_matches_oracle(bm, n, prec, monkeypatch):
    monkeypatch.setenv("BM_TILES", "1,4,8,1")
    monkeypatch.setenv("BM_YZY", "1")
    N = n[0] * n[1] * n[2]
    M = sphere_random(N, seed=n[1] + n[2], Ms=8e5)
    Href, _ = orc_hdemag(M, n, (3e-9, 3e-9, 2e-9))
    htol, mtol = (1e-9, 1e-9) if prec == "fp64" else (1e-5, 1e-4)
    c = _ctx(bm, prec, n, M)
    H = c.demag_field()
    assert c.tiles()["yzy"] == 1, "the fused cluster pass did not run"
    assert np.abs(H - Href).max() / np.abs(Href).max() < htol
    c.set_m(M)
    c.run(6)
    m = c.get_m()
    c.close()
    s = OracleSolver([dict(n=n, h=(3e-9, 3e-9, 2e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16,
                           Ha=(2e3, 1e3, 0))], evaluation=0, dt=2e-14)
    s.set_m(M)
    s.run(6)
    assert np.abs(m - s.get_m()).max() / 8e5 < mtol
    s.close()


def test_yzy_chosen_on_the_headline_film(bm):
    """The autotuner times the fused pass against the three tuned launches on the 512 x 512 x 16 film;
    whichever it keeps, the field matches the FP64 form."""
    n = (512, 512, 16)
    M = sphere_random(n[0] * n[1] * n[2], seed=99, Ms=1.1e6)
    H = {}
    for prec in ("mixed", "fp64"):
        c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
        c.add_mesh(n, (2e-9, 2e-9, 2e-9))
        c.set_material(0, Ms=1.1e6, A=1.5e-11, alpha=0.1)
        c.set_modules(0, bm.DEMAG)
        c.set_m(M)
        H[prec] = c.demag_field()
        c.close()
    assert np.abs(H["mixed"] - H["fp64"]).max() / np.abs(H["fp64"]).max() < 1e-5
