"""Periodic boundary conditions on cuda:0 (bm_set_pbc, C ABI) against the oracle, which restates the
reference's own PBC algorithm (cyclic convolution of period n with the image-summed tensor, the
wrapped stencils, SelfDemag_PBC) and is pinned to the compiled reference in test_oracle_pbc.py; and,
where the reference's field is the periodic convolution (an even cell count along the last
transformed axis), against the compiled reference directly.

Tolerances: tensor octant FP64 5e-11 absolute; H_demag and H_eff FP64 1e-9 (stencil-only 1e-10),
mixed 1e-5 relative to max |H_ref|; integration FP64 1e-9 of Ms after the run (RKDP54 1e-8 with the
same accepted / rejected counts), mixed 1e-4; adjoint FP64 gradients 1e-8 of their largest magnitude."""
import numpy as np
import pytest

import boris2_b200 as bmod
from oracle_libs import (OracleSolver, sphere_random, tilted_z, orc_hdemag_pbc, ref_hdemag_pbc, orc_tensor_pbc,
                         reference, orc_adjoint)
from test_oracle_pbc import symmetrise
from test_gpu_step import _make

pytestmark = pytest.mark.gpu


def _relmax(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def _ids(c):
    return "n%dx%dx%d_pbc%d,%d,%d" % (c[0] + c[2])


TENSOR_CASES = [
    ((16, 8, 1), (5e-9, 4e-9, 3e-9), (2, 3, 0)),
    ((7, 5, 1), (5e-9, 4e-9, 3e-9), (2, 2, 1)),
    ((6, 5, 4), (4e-9, 3e-9, 5e-9), (1, 2, 3)),
    ((10, 6, 3), (3e-9, 4e-9, 5e-9), (0, 2, 1)),
    ((48, 40, 1), (4e-9, 4e-9, 3e-9), (6, 6, 0)),   # offsets beyond the 40-cell far-field switch
    ((8, 6, 2), (5e-9, 5e-9, 3e-9), (-2, 1, -1)),
]


@pytest.mark.parametrize("case", TENSOR_CASES, ids=_ids)
def test_pbc_tensor_octant(bm, case):
    """The device's periodic octant equals the reference-style tensor made even / odd per periodic axis."""
    n, h, pbc = case
    dg, od = orc_tensor_pbc(n, h, pbc)
    S = symmetrise(dg, od, pbc)
    g = bm.debug_tensor(n, h, pbc=pbc)
    for c in range(6):
        if n[2] == 1 and c >= 4:
            continue
        assert np.abs(g[..., c] - S[c][:n[2], :n[1], :n[0]]).max() < 5e-11, c


DEMAG_CASES = [
    ((16, 8, 1), (5e-9, 5e-9, 3e-9), (3, 0, 0)),
    ((16, 8, 1), (5e-9, 4e-9, 3e-9), (2, 3, 0)),
    ((12, 10, 1), (5e-9, 5e-9, 2e-9), (0, 0, 4)),
    ((9, 8, 1), (5e-9, 4e-9, 3e-9), (2, 0, 0)),
    ((7, 5, 1), (5e-9, 4e-9, 3e-9), (2, 2, 1)),      # odd periodic y in 2D
    ((8, 8, 4), (4e-9, 4e-9, 4e-9), (2, 2, 0)),
    ((6, 5, 4), (4e-9, 3e-9, 5e-9), (1, 2, 3)),
    ((10, 6, 3), (3e-9, 4e-9, 5e-9), (0, 2, 1)),     # odd periodic z
    ((8, 6, 2), (5e-9, 5e-9, 3e-9), (-2, 1, -1)),    # negative counts: |images| for demag
    ((1, 8, 1), (5e-9, 5e-9, 3e-9), (3, 0, 0)),
    ((8, 1, 4), (5e-9, 5e-9, 3e-9), (0, 2, 2)),
    ((64, 64, 1), (4e-9, 4e-9, 3e-9), (10, 10, 0)),  # register y pass, two periodic axes
    ((100, 10, 3), (2e-9, 2e-9, 2e-9), (3, 0, 0)),   # LX = 128 register x pass
    ((32, 32, 8), (3e-9, 3e-9, 3e-9), (4, 4, 0)),
    ((16, 16, 16), (2e-9, 2e-9, 2e-9), (1, 1, 1)),   # periodic on every axis
]


@pytest.mark.parametrize("case", DEMAG_CASES, ids=_ids)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pbc_hdemag(bm, case, prec):
    n, h, pbc = case
    N = n[0] * n[1] * n[2]
    M = sphere_random(N, seed=300 + N, Ms=8e5)
    Href, dot = orc_hdemag_pbc(M, n, h, pbc)
    with bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_pbc(0, pbc)
        assert c.get_pbc(0) == tuple(pbc)
        c.set_m(M)
        H, e = c.demag_field(with_energy=True)
    tol = 1e-9 if prec == "fp64" else 1e-5
    assert _relmax(H, Href) < tol
    eref = -1.256637061435916e-6 * dot / (2 * N)
    assert abs(e - eref) <= tol * abs(eref)


@pytest.mark.parametrize("case", [c for c in DEMAG_CASES
                                  if not ((c[0][2] == 1 and c[2][1] and c[0][1] % 2) or
                                          (c[0][2] > 1 and c[2][2] and c[0][2] % 2)) and np.prod(c[0]) <= 4096],
                         ids=_ids)
def test_pbc_hdemag_vs_reference_build(bm, case):
    """Against the reference's own Convolution<., DemagKernel> set up with pbc_images."""
    if reference() is None:
        pytest.skip("reference CPU build not available")
    n, h, pbc = case
    N = n[0] * n[1] * n[2]
    M = sphere_random(N, seed=99, Ms=8e5)
    Href, _ = ref_hdemag_pbc(M, n, h, pbc)
    with bm.Context(precision=bm.FP64) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_pbc(0, pbc)
        c.set_m(M)
        H = c.demag_field()
    assert _relmax(H, Href) < 1e-9


def test_pbc_uniform_in_plane_film_has_no_field(bm):
    """Known answer: a film periodic in x and y, magnetised uniformly along x, is an infinite sheet up to
    the truncated image sum, so H_x is small and uniform (no edge charges anywhere)."""
    n, h = (64, 64, 1), (4e-9, 4e-9, 3e-9)
    M = np.zeros((n[0] * n[1], 3))
    M[:, 0] = 8e5
    with bm.Context(precision=bm.FP64) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_pbc(0, (20, 20, 0))
        c.set_m(M)
        H = c.demag_field()
    assert np.abs(H[:, 0]).max() < 2e-3 * 8e5
    assert np.abs(H[:, 0] - H[:, 0].mean()).max() < 1e-9 * 8e5
    with bm.Context(precision=bm.FP64) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_m(M)
        Hopen = c.demag_field()
    assert np.abs(Hopen[:, 0]).max() > 0.1 * 8e5   # without PBC the edges carry charge


FIELD_CASES = [
    ("exch", (12, 9, 1), 2, (2, 3, 0)),
    ("exch3d", (7, 6, 4), 2, (1, 0, 2)),
    ("idmi", (12, 9, 1), 4, (3, 0, 0)),
    ("idmi3d", (8, 5, 3), 4, (1, 2, 1)),
    ("idmi_neg", (10, 6, 2), 4, (-1, 2, 0)),
    ("all", (16, 12, 2), 1 | 4 | 8 | 16, (2, 2, 0)),
    ("all2", (20, 10, 1), 1 | 2 | 8 | 16, (0, 4, 0)),
]


@pytest.mark.parametrize("name,n,mods,pbc", FIELD_CASES)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pbc_heff_terms(bm, name, n, mods, pbc, prec):
    h = (2e-9, 3e-9, 1.5e-9)
    N = n[0] * n[1] * n[2]
    rng = np.random.default_rng(7)
    Ms_map = 8e5 * (1 + 0.1 * rng.normal(size=N))
    K1_map = rng.uniform(0, 2e5, N)
    M = sphere_random(N, seed=5) * Ms_map[:, None]
    mesh = dict(n=n, h=h, Ms=8e5, A=1.3e-11, D=1.5e-3, alpha=0.1, K1=3e5, K2=1e4, ea=(0.3, 0.2, 1.0),
                Ms_map=Ms_map, K1_map=K1_map, modules=mods, Ha=(1e3, -2e3, 5e2), pbc=pbc)
    s = OracleSolver([mesh])
    s.set_m(M)
    Href = s.heff()
    s.close()
    with bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED) as c:
        c.add_mesh(n, h)
        c.set_material(0, Ms=8e5, A=1.3e-11, alpha=0.1, K1=3e5, K2=1e4, ea=(0.3, 0.2, 1.0), D=1.5e-3)
        c.set_material_maps(0, Ms_map=Ms_map, K1_map=K1_map)
        c.set_modules(0, mods)
        c.set_pbc(0, pbc)
        c.set_field(0, (1e3, -2e3, 5e2))
        c.set_m(M)
        H = c.update_field()
    tol = (1e-9 if mods & 1 else 1e-10) if prec == "fp64" else 1e-5
    assert _relmax(H, Href) < tol


def test_pbc_exchange_wraps_a_uniform_twist(bm):
    """A spin spiral commensurate with the periodic x length has the same exchange field in every cell
    (no boundary cells), and the field differs from the Neumann one at the faces."""
    n, h = (32, 4, 1), (2e-9, 2e-9, 2e-9)
    N = n[0] * n[1]
    x = np.tile(np.arange(n[0]), n[1])
    th = 2 * np.pi * x / n[0]
    M = 8e5 * np.stack([np.cos(th), np.sin(th), np.zeros(N)], axis=1)
    with bm.Context(precision=bm.FP64) as c:
        c.add_mesh(n, h)
        c.set_modules(0, bm.EXCH)
        c.set_pbc(0, (1, 0, 0))
        c.set_m(M)
        H = c.update_field()
    # H = c * lap M: antiparallel to M with |H| = 2A/(mu0 Ms^2) * Ms * 2 (1 - cos(2 pi / n)) / h^2
    c0 = 2 * 1.3e-11 / (1.256637061435916e-6 * 8e5 ** 2) * 8e5 * 2 * (1 - np.cos(2 * np.pi / n[0])) / h[0] ** 2
    proj = (H * M).sum(axis=1) / 8e5
    assert np.abs(proj + c0).max() < 1e-9 * c0
    assert np.abs(np.cross(H, M)).max() < 1e-9 * c0 * 8e5


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_pbc_rk4_film(bm, prec, tol):
    mesh = dict(n=(32, 16, 1), h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, D=2e-3, alpha=0.5, modules=1 | 4 | 16,
                Ha=(1e3, 0, 0), pbc=(5, 5, 0))
    N = 32 * 16
    M = sphere_random(N, seed=1236, Ms=8e5)
    s = OracleSolver([mesh], evaluation=0, dt=1e-13)
    s.set_m(M)
    s.run(30)
    mref = s.get_m() / 8e5
    c = _make(bm, prec, mesh, M, "RK4", 1e-13)
    st = c.run(30)
    m = c.get_m() / 8e5
    c.close()
    assert st["accepted"] == 30
    assert np.abs(m - mref).max() < tol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pbc_rkdp54_adaptive_3d(bm, prec):
    n = (16, 12, 4)
    N = int(np.prod(n))
    mesh = dict(n=n, h=(2e-9, 2e-9, 2e-9), Ms=1.1e6, A=1.5e-11, D=1.5e-3, alpha=0.1, K1=5e5,
                modules=1 | 4 | 8 | 16, Ha=(0, 0, 0), pbc=(2, 3, 1))
    M = tilted_z(N, seed=18, Ms=1.1e6)
    ctrl = (1e-5, 2.0, 1e-15, 3e-12)
    s = OracleSolver([mesh], evaluation=1, dt=1e-14, tol=1e-5, dT_incr=2.0, dT_min=1e-15, dT_max=3e-12)
    s.set_m(M)
    sr = s.run(50)
    mref = s.get_m() / 1.1e6
    c = _make(bm, prec, mesh, M, "RKDP54", 1e-14, ctrl)
    st = c.run(50)
    m = c.get_m() / 1.1e6
    c.close()
    assert st["accepted"] == 50
    if prec == "fp64":
        assert st["rejected"] == sr["rejected"]
        assert abs(st["time"] - sr["time"]) <= 1e-9 * sr["time"]
        assert np.abs(m - mref).max() < 1e-8
    else:
        assert np.abs(m - mref).max() < 1e-4


@pytest.mark.parametrize("level", [2, 4])
def test_pbc_evalspeedup_rk4(bm, level):
    """The speedup's self term under PBC is SelfDemag_PBC (the images' far field added)."""
    mesh = dict(n=(32, 16, 1), h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16,
                Ha=(1e3, 0, 0), pbc=(4, 2, 0))
    N = 32 * 16
    M = sphere_random(N, seed=500 + level, Ms=8e5)
    s = OracleSolver([mesh], evaluation=0, dt=1e-13)
    s.evalspeedup(level)
    s.set_m(M)
    s.run(20)
    mref = s.get_m()
    s.close()
    c = _make(bm, "fp64", mesh, M, "RK4", 1e-13)
    c.evalspeedup(level)
    c.run(20)
    m = c.get_m()
    c.close()
    assert np.abs(m - mref).max() / 8e5 < 1e-9


def test_pbc_batched_equals_per_mesh(bm):
    """Meshes with different PBC in one batched launch match their per-mesh runs (FP64)."""
    systems = [((32, 16, 1), (3, 0, 0)), ((24, 24, 2), (2, 2, 0)), ((16, 8, 4), (0, 0, 1)), ((20, 12, 1), (0, 0, 0))]
    h = (4e-9, 4e-9, 3e-9)
    out = {}
    for batched in (False, True):
        c = bm.Context(precision=bm.FP64)
        for q, (n, pbc) in enumerate(systems):
            c.add_mesh(n, h, (0.0, 0.0, 1e-6 * q))
            c.set_material(q, Ms=8e5, A=1.3e-11, alpha=0.3, D=1e-3)
            c.set_modules(q, 1 | 4)
            c.set_pbc(q, pbc)
        c.set_batched(batched)
        c.setode("RK4", 1e-13)
        for q, (n, _) in enumerate(systems):
            c.set_m(sphere_random(int(np.prod(n)), seed=70 + q, Ms=8e5), q)
        c.run(15)
        out[batched] = [c.get_m(q) for q in range(len(systems))]
        c.close()
    for a, b in zip(out[False], out[True]):
        assert np.abs(a - b).max() / 8e5 < 1e-11


def test_pbc_adjoint_fp64_matches_oracle(bm):
    from test_gpu_adjoint import _case, _gpu, _rel
    mesh, m0, tgt, steps, dt = _case(n=(16, 12, 1))
    mesh["pbc"] = (3, 2, 0)
    lo, gMs_o, gK_o, gHa_o = orc_adjoint(mesh, m0, tgt, steps, dt)
    lg, gMs, gK, gHa, _ = _gpu(bm, mesh, m0, tgt, steps, dt, "fp64", 5)
    # the periodic kernels of the two agree to ~1e-11 (image sums of the device's and the CPU's libm
    # values), one decade above the open-boundary case
    assert abs(lg - lo) <= 1e-11 * abs(lo)
    assert _rel(gMs, gMs_o) < 1e-8
    assert _rel(gK, gK_o) < 1e-8
    assert _rel(gHa, gHa_o) < 1e-8


def test_pbc_refusals(bm):
    with bm.Context() as c:
        c.add_mesh((8, 8, 1), (4e-9, 4e-9, 3e-9))
        with pytest.raises(bmod.BorisError) as e:
            c.set_pbc(0, (bm.PBC_MAX_IMAGES + 1, 0, 0))
        assert e.value.code == bm.EINVAL
        with pytest.raises(bmod.BorisError):
            c.set_pbc(3, (1, 0, 0))
    # the periodic tensor build is bounded
    with bm.Context() as c:
        c.add_mesh((256, 256, 16), (4e-9, 4e-9, 3e-9))
        c.set_modules(0, bm.DEMAG)
        c.set_pbc(0, (400, 400, 0))
        with pytest.raises(bmod.BorisError) as e:
            c.set_m(np.tile([0.0, 0.0, 8e5], (256 * 256 * 16, 1)))
            c.demag_field()
        assert e.value.code == bm.EUNSUPPORTED
    # not with the multilayered convolution
    with bm.Context() as c:
        c.add_mesh((16, 16, 1), (4e-9, 4e-9, 3e-9), (0, 0, 0))
        c.add_mesh((16, 16, 1), (4e-9, 4e-9, 3e-9), (0, 0, 6e-9))
        c.set_pbc(0, (2, 2, 0))
        c.multiconvolution(bm.ML_3D)
        with pytest.raises(bmod.BorisError) as e:
            c.prepare()
        assert e.value.code == bm.EUNSUPPORTED
