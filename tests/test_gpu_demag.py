"""GPU parity of the demag path against the oracle (C ABI calls on cuda:0).

Tolerances:
  FFT            FP64 <= 1e-13, FP32 <= 2e-6 relative to max |X|
  tensor         FP64 <= 5e-11 absolute (values are O(1); the 27-point differences cancel
                 to ~1e-11 near the 40-cell far-field switch, so GPU and CPU libm roundings differ there)
  kernels        FP64 <= 1e-9 absolute
  H_demag        FP64 <= 1e-9, mixed <= 1e-5 relative to max |H_ref| (the stated tolerance)
  H_eff terms    FP64 <= 1e-10, mixed <= 1e-5 relative to max |H_ref|
"""
import numpy as np
import pytest

from oracle_libs import (oracle, orc_hdemag, dp, OracleSolver, sphere_random, tilted_z, reference, ref_hdemag)

pytestmark = pytest.mark.gpu


def _relmax(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("L", [1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 2048, 3072, 4096])
def test_fft_lengths(bm, L):
    rng = np.random.default_rng(L)
    x = rng.normal(size=(5, L)) + 1j * rng.normal(size=(5, L))
    ref = np.fft.fft(x, axis=-1)
    g64 = bm.debug_fft(x, precision=bm.FP64)
    assert _relmax(g64, ref) < 1e-13
    g32 = bm.debug_fft(x, precision=bm.MIXED)
    assert _relmax(g32, ref) < 2e-6
    gi = bm.debug_fft(x, precision=bm.FP64, inverse=True)
    assert _relmax(gi, np.fft.ifft(x, axis=-1) * L) < 1e-13


@pytest.mark.parametrize("n,h", [((8, 6, 1), (5e-9, 5e-9, 3e-9)), ((6, 5, 4), (2e-9, 2e-9, 2e-9)),
                                 ((50, 45, 1), (4e-9, 4e-9, 3e-9)), ((45, 7, 3), (1e-9, 2e-9, 3.5e-9)),
                                 ((64, 48, 2), (2e-9, 2e-9, 1e-9))])
def test_tensor_octant(bm, n, h):
    nx, ny, nz = n
    Nx, Ny, Nz = 2 * nx, 2 * ny, (2 * nz if nz > 1 else 1)
    npt = Nx * Ny * Nz
    dg = np.zeros(3 * npt)
    od = np.zeros(3 * npt)
    oracle().orc_tensor(nx, ny, nz, Nx, Ny, Nz, h[0], h[1], h[2], dp(dg), dp(od))
    dg = dg.reshape(Nz, Ny, Nx, 3)[:nz, :ny, :nx]
    od = od.reshape(Nz, Ny, Nx, 3)[:nz, :ny, :nx]
    g = bm.debug_tensor(n, h)
    assert np.abs(g[..., :3] - dg).max() < 5e-11
    assert np.abs(g[..., 3:] - od).max() < 5e-11


@pytest.mark.parametrize("n,h", [((8, 6, 1), (5e-9, 5e-9, 3e-9)), ((6, 5, 4), (2e-9, 2e-9, 2e-9)),
                                 ((50, 45, 1), (4e-9, 4e-9, 3e-9)), ((12, 7, 3), (1e-9, 2e-9, 3.5e-9))])
def test_kernel_spectra(bm, n, h):
    """GPU FP64 spectra vs the oracle on the same (product) FFT sizes."""
    with bm.Context(precision=bm.FP64) as c:
        c.add_mesh(n, h)
        N = c.fft_sizes()
        K = c.debug_kernels()
    nk = (N[0] // 2 + 1) * (N[1] // 2 + 1) * (N[2] // 2 + 1)
    kd = np.zeros(3 * nk)
    ko = np.zeros(3 * nk)
    oracle().orc_kernels(n[0], n[1], n[2], N[0], N[1], N[2], h[0], h[1], h[2], dp(kd), dp(ko))
    kd = kd.reshape(N[2] // 2 + 1, N[1] // 2 + 1, N[0] // 2 + 1, 3)
    ko = ko.reshape(N[2] // 2 + 1, N[1] // 2 + 1, N[0] // 2 + 1, 3)
    for c_ in range(3):
        assert np.abs(K[c_] - kd[..., c_]).max() < 1e-9
        assert np.abs(K[3 + c_] - ko[..., c_]).max() < 1e-9


DEMAG_CASES = [
    ((16, 8, 1), (5e-9, 5e-9, 3e-9)),
    ((5, 3, 1), (2e-9, 3e-9, 1e-9)),        # odd sizes, 3 * 2^k FFT lengths
    ((1, 7, 1), (2e-9, 2e-9, 2e-9)),        # single column
    ((9, 1, 1), (2e-9, 2e-9, 2e-9)),        # single row
    ((10, 6, 4), (2e-9, 2e-9, 2e-9)),
    ((12, 5, 3), (4e-9, 4e-9, 3e-9)),
    ((24, 20, 2), (2e-9, 2e-9, 1.5e-9)),
    ((64, 48, 1), (4e-9, 4e-9, 3e-9)),
    ((33, 17, 5), (3e-9, 2e-9, 2e-9)),
    ((16, 16, 4), (2e-9, 2e-9, 2e-9)),      # power-of-two y: register y passes
    ((20, 64, 2), (2e-9, 2e-9, 2e-9)),
    ((8, 512, 3), (2e-9, 2e-9, 2e-9)),      # Ny = 1024 = 32 x 32 split
    ((6, 5, 32), (2e-9, 2e-9, 2e-9)),       # Nz = 64 register z pass
    ((100, 10, 3), (2e-9, 2e-9, 2e-9)),     # LX = 128 register x passes
    ((200, 6, 1), (2e-9, 2e-9, 1e-9)),      # LX = 256
    ((300, 3, 2), (2e-9, 2e-9, 1e-9)),      # LX = 384 (generic x kernel)
    ((512, 4, 1), (2e-9, 2e-9, 1e-9)),      # LX = 512
    ((1000, 2, 1), (2e-9, 2e-9, 1e-9)),     # LX = 1024
    ((1100, 2, 1), (2e-9, 2e-9, 1e-9)),     # LX = 1536 (beyond the register x kernels: generic)
    ((2000, 1, 1), (2e-9, 2e-9, 1e-9)),     # LX = 2048 (generic)
    ((4, 1024, 2), (2e-9, 2e-9, 2e-9)),     # Ny = 2048 (radix-16 Stockham or generic y passes)
    ((4, 3, 64), (2e-9, 2e-9, 2e-9)),       # Nz = 128 (generic z pass)
]


@pytest.mark.parametrize("n,h", DEMAG_CASES)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_hdemag(bm, n, h, prec):
    N = n[0] * n[1] * n[2]
    M = sphere_random(N, seed=1234 + N, Ms=8e5)
    Href, dot = orc_hdemag(M, n, h)
    with bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_material(0, Ms=8e5)
        c.set_m(M)
        H, e = c.demag_field(with_energy=True)
    tol = 1e-9 if prec == "fp64" else 1e-5
    assert _relmax(H, Href) < tol
    eref = -1.256637061435916e-6 * dot / (2 * N)
    assert abs(e - eref) <= (1e-9 if prec == "fp64" else 1e-5) * abs(eref)


@pytest.mark.parametrize("n,h", [((16, 8, 1), (5e-9, 5e-9, 3e-9)), ((10, 6, 4), (2e-9, 2e-9, 2e-9))])
def test_hdemag_vs_reference_build(bm, n, h):
    """Against the reference's own Convolution<., DemagKernel> (compiled CPU build)."""
    if reference() is None:
        pytest.skip("reference CPU build not available")
    N = n[0] * n[1] * n[2]
    M = sphere_random(N, seed=99, Ms=8e5)
    Href, _ = ref_hdemag(M, n, h)
    with bm.Context(precision=bm.FP64) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_m(M)
        H = c.demag_field()
    assert _relmax(H, Href) < 1e-9


def test_uniform_film_known_answer(bm):
    """Thin film magnetised along z: H ~ -M in the interior (N_zz -> 1)."""
    n = (128, 128, 1)
    h = (2e-9, 2e-9, 1e-9)
    M = np.zeros((n[0] * n[1], 3))
    M[:, 2] = 1e6
    with bm.Context(precision=bm.MIXED) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_m(M)
        H = c.demag_field().reshape(n[1], n[0], 3)
    centre = H[n[1] // 2, n[0] // 2]
    assert -1.0 < centre[2] / 1e6 < -0.97
    assert abs(centre[0]) < 1e-3 * 1e6 and abs(centre[1]) < 1e-3 * 1e6


FIELD_CASES = [
    ("exch", (12, 9, 1), 2),
    ("exch3d", (7, 6, 4), 2),
    ("idmi", (12, 9, 1), 4),
    ("idmi3d", (8, 5, 3), 4),
    ("all", (16, 12, 2), 1 | 4 | 8 | 16),
    ("all2", (20, 10, 1), 1 | 2 | 8 | 16),
]


@pytest.mark.parametrize("name,n,mods", FIELD_CASES)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_heff_terms(bm, name, n, mods, prec):
    h = (2e-9, 3e-9, 1.5e-9)
    N = n[0] * n[1] * n[2]
    rng = np.random.default_rng(7)
    Ms_map = 8e5 * (1 + 0.1 * rng.normal(size=N))
    K1_map = rng.uniform(0, 2e5, N)
    M = sphere_random(N, seed=5) * Ms_map[:, None]
    mesh = dict(n=n, h=h, Ms=8e5, A=1.3e-11, D=1.5e-3, alpha=0.1, K1=3e5, K2=1e4, ea=(0.3, 0.2, 1.0),
                Ms_map=Ms_map, K1_map=K1_map, modules=mods, Ha=(1e3, -2e3, 5e2))
    s = OracleSolver([mesh])
    s.set_m(M)
    Href = s.heff()
    s.close()
    with bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED) as c:
        c.add_mesh(n, h)
        c.set_material(0, Ms=8e5, A=1.3e-11, alpha=0.1, K1=3e5, K2=1e4, ea=(0.3, 0.2, 1.0), D=1.5e-3)
        c.set_material_maps(0, Ms_map=Ms_map, K1_map=K1_map)
        c.set_modules(0, mods)
        c.set_field(0, (1e3, -2e3, 5e2))
        c.set_m(M)
        H = c.update_field()
    tol = 1e-10 if prec == "fp64" else 1e-5
    assert _relmax(H, Href) < tol
