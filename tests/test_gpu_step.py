"""GPU parity of the LLG RK4 / RKDP54 integration against the oracle (C ABI on cuda:0).

Tolerances: FP64 plain form <= 1e-9 max |m - m_ref| after the run; mixed precision
<= 1e-4 (the stated |dm| tolerance). RKDP54 step counts (accepted / rejected) and the
simulated time must agree with the oracle for the FP64 form.
"""
import numpy as np
import pytest

from oracle_libs import OracleSolver, sphere_random, tilted_z

pytestmark = pytest.mark.gpu


def _make(bm, prec, mesh, M, evaluation, dt, ctrl=None):
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    c.add_mesh(mesh["n"], mesh["h"])
    c.set_material(0, Ms=mesh.get("Ms", 8e5), A=mesh.get("A", 1.3e-11), alpha=mesh.get("alpha", 0.5),
                   grel=mesh.get("grel", 1.0), K1=mesh.get("K1", 0.0), K2=mesh.get("K2", 0.0),
                   ea=mesh.get("ea", (0, 0, 1)), D=mesh.get("D", 0.0))
    if mesh.get("Ms_map") is not None or mesh.get("K1_map") is not None:
        c.set_material_maps(0, Ms_map=mesh.get("Ms_map"), K1_map=mesh.get("K1_map"))
    c.set_modules(0, mesh["modules"])
    if mesh.get("pbc") is not None:
        c.set_pbc(0, mesh["pbc"])
    c.set_field(0, mesh.get("Ha", (0, 0, 0)), mesh.get("Ha_tspan", 0.0))
    c.setode(evaluation, dt)
    if ctrl:
        c.astepctrl(*ctrl)
    c.set_m(M)
    return c


CFG1_SMALL = dict(n=(32, 16, 1), h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5,
                  grel=2.211e5 / 2.212761569e5, modules=1 | 2 | 16, Ha=(1e3, 0, 0))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_rk4_film(bm, prec, tol):
    mesh = CFG1_SMALL
    N = 32 * 16
    M = sphere_random(N, seed=1235, Ms=8e5)
    s = OracleSolver([mesh], evaluation=0, dt=1e-13)
    s.set_m(M)
    s.run(40)
    mref = s.get_m() / 8e5
    c = _make(bm, prec, mesh, M, "RK4", 1e-13)
    st = c.run(40)
    m = c.get_m() / 8e5
    c.close()
    assert st["accepted"] == 40
    assert abs(st["time"] - 40e-13) < 1e-25
    assert np.abs(m - mref).max() < tol


def test_rk4_3d_iDMI_anisotropy_maps(bm):
    n = (12, 10, 4)
    N = n[0] * n[1] * n[2]
    rng = np.random.default_rng(3)
    Ms_map = 1.1e6 * (1 + 0.05 * rng.normal(size=N))
    K1_map = rng.uniform(0, 5e5, N)
    mesh = dict(n=n, h=(2e-9, 2e-9, 2e-9), Ms=1.1e6, A=1.5e-11, D=1.5e-3, alpha=0.1, K1=5e5,
                ea=(0, 0, 1), modules=1 | 4 | 8 | 16, Ha=(0, 0, 0), Ms_map=Ms_map, K1_map=K1_map)
    M = tilted_z(N, seed=11) * Ms_map[:, None]
    s = OracleSolver([mesh], evaluation=0, dt=2e-14)
    s.set_m(M)
    s.run(25)
    mref = s.get_m() / Ms_map[:, None]
    for prec, tol in (("fp64", 1e-9), ("mixed", 1e-4)):
        c = _make(bm, prec, mesh, M, "RK4", 2e-14)
        c.run(25)
        m = c.get_m() / Ms_map[:, None]
        c.close()
        assert np.abs(m - mref).max() < tol, prec


def test_zeeman_pulse_samples(bm):
    """Piecewise-constant applied field samples, evaluated at the step start time."""
    n = (16, 16, 1)
    N = 256
    rng = np.random.default_rng(8)
    Ha = rng.normal(0, 5e3, size=(8, 3))
    mesh = dict(n=n, h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.02, modules=1 | 2 | 16,
                Ha=Ha, Ha_tspan=8 * 5e-13)
    M = sphere_random(N, seed=4, Ms=8e5)
    s = OracleSolver([mesh], evaluation=0, dt=1e-13)
    s.set_m(M)
    s.run(50)
    mref = s.get_m()
    c = _make(bm, "fp64", mesh, M, "RK4", 1e-13)
    c.run(50)
    assert np.abs(c.get_m() - mref).max() / 8e5 < 1e-9
    c.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_rkdp54_adaptive(bm, prec):
    n = (16, 16, 2)
    N = n[0] * n[1] * n[2]
    mesh = dict(n=n, h=(2e-9, 2e-9, 2e-9), Ms=1.1e6, A=1.5e-11, D=1.5e-3, alpha=0.1, K1=5e5,
                modules=1 | 4 | 8 | 16, Ha=(0, 0, 0))
    M = tilted_z(N, seed=17, Ms=1.1e6)
    ctrl = (1e-5, 2.0, 1e-15, 3e-12)
    s = OracleSolver([mesh], evaluation=1, dt=1e-14, tol=1e-5, dT_incr=2.0, dT_min=1e-15, dT_max=3e-12)
    s.set_m(M)
    sr = s.run(60)
    mref = s.get_m() / 1.1e6
    c = _make(bm, prec, mesh, M, "RKDP54", 1e-14, ctrl)
    st = c.run(60)
    m = c.get_m() / 1.1e6
    c.close()
    assert st["accepted"] == 60
    if prec == "fp64":
        assert st["rejected"] == sr["rejected"]
        assert abs(st["time"] - sr["time"]) <= 1e-9 * sr["time"]
        assert abs(st["dT"] - sr["dT"]) <= 1e-6 * sr["dT"]
        assert np.abs(m - mref).max() < 1e-8
    else:
        assert abs(st["time"] - sr["time"]) <= 1e-3 * sr["time"]
        assert np.abs(m - mref).max() < 1e-4


def test_rkdp54_rejections(bm):
    """A large starting step forces rejections; the FP64 device controller must follow the
    oracle's accept/reject sequence exactly."""
    n = (16, 16, 1)
    N = 256
    mesh = dict(n=n, h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16, Ha=(1e4, 0, 0))
    M = sphere_random(N, seed=21, Ms=8e5)
    ctrl = (1e-6, 2.0, 1e-16, 1e-11)
    s = OracleSolver([mesh], evaluation=1, dt=2e-12, tol=1e-6, dT_incr=2.0, dT_min=1e-16, dT_max=1e-11)
    s.set_m(M)
    sr = s.run(30)
    assert sr["rejected"] > 0
    c = _make(bm, "fp64", mesh, M, "RKDP54", 2e-12, ctrl)
    st = c.run(30)
    m = c.get_m()
    c.close()
    assert st["accepted"] == 30
    assert st["rejected"] == sr["rejected"]
    assert abs(st["time"] - sr["time"]) <= 1e-9 * sr["time"]
    assert np.abs(m - s.get_m()).max() / 8e5 < 1e-8


def test_norm_preserved_and_energy_decreases(bm):
    n = (64, 64, 1)
    N = n[0] * n[1]
    mesh = dict(n=n, h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2, Ha=(0, 0, 0))
    M = sphere_random(N, seed=2, Ms=8e5)
    c = _make(bm, "mixed", mesh, M, "RK4", 5e-14)
    H0 = c.update_field()
    e0 = -(c.get_m() * H0).sum()
    c.run(200)
    m = c.get_m()
    H1 = c.update_field()
    e1 = -(m * H1).sum()
    c.close()
    assert np.abs(np.linalg.norm(m, axis=1) / 8e5 - 1).max() < 1e-5
    assert e1 < e0


@pytest.mark.parametrize("xv", ["0", "1"])
@pytest.mark.parametrize("staged", ["0", "1"])
@pytest.mark.parametrize("rows", [1, 3])
def test_stage_kernel_variants(bm, staged, rows, xv, monkeypatch):
    """Every stage-kernel variant (per-cell rows prefetched into shared memory or read from global
    memory; two-level or radix-8 Stockham x transform) and several rows per block, forced through
    BM_TILES / BM_STAGE_ROWS / BM_STAGE_XV, give the oracle's RKDP54 trajectory (exchange + iDMI +
    anisotropy + demag, 3D, LX = 128, 64 and 256). The 256-wide mesh makes the staged launches of
    one graph need different shared-memory sizes above 48 KB (the error-estimate launch stages the
    most rows)."""
    monkeypatch.setenv("BM_TILES", "1,4,8,%d" % rows)
    monkeypatch.setenv("BM_STAGE_ROWS", staged)
    monkeypatch.setenv("BM_STAGE_XV", xv)
    for n in [(100, 10, 3), (64, 12, 2), (256, 6, 2)]:
        N = n[0] * n[1] * n[2]
        rng = np.random.default_rng(5)
        Ms_map = 1.1e6 * (1 + 0.05 * rng.normal(size=N))
        mesh = dict(n=n, h=(2e-9, 2e-9, 2e-9), Ms=1.1e6, A=1.5e-11, D=1.5e-3, alpha=0.1, K1=5e5,
                    modules=1 | 4 | 8 | 16, Ha=(1e3, 0, 0), Ms_map=Ms_map)
        M = tilted_z(N, seed=23) * Ms_map[:, None]
        s = OracleSolver([mesh], evaluation=1, dt=1e-14, tol=1e-5, dT_incr=2.0, dT_min=1e-15, dT_max=3e-12)
        s.set_m(M)
        sr = s.run(8)
        mref = s.get_m() / Ms_map[:, None]
        c = _make(bm, "fp64", mesh, M, "RKDP54", 1e-14, (1e-5, 2.0, 1e-15, 3e-12))
        st = c.run(8)
        t = c.tiles()
        m = c.get_m() / Ms_map[:, None]
        c.close()
        assert abs(t["stage_rows"]) == rows and (t["stage_rows"] < 0) == (staged == "1")
        assert t["stage_xv"] == int(xv)
        assert st["rejected"] == sr["rejected"]
        assert np.abs(m - mref).max() < 1e-8


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
@pytest.mark.parametrize("nx", [16, 32, 64, 128, 256, 512, 1024, 24, 48, 96, 192, 384, 768])
def test_stage_xv_every_length(bm, nx, prec, tol, monkeypatch):
    """The Stockham x transform at every register length (power of two, radix 8 with tails 8x2,
    8x4, 8x8, 8x8x2, 8x8x4, 8x8x8, 8x8x8x2; 3 * 2^k, radix 4 / 2 with a last radix-3 pass; odd nx
    leaves a zero partner slot) against the oracle's RK4 trajectory with demag, exchange and
    Zeeman."""
    monkeypatch.setenv("BM_TILES", "1,4,8,1")
    monkeypatch.setenv("BM_STAGE_XV", "1")
    for n in [(nx, 3, 2), (nx - 1, 2, 1)]:
        N = n[0] * n[1] * n[2]
        mesh = dict(n=n, h=(3e-9, 3e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(2e3, 1e3, 0))
        M = sphere_random(N, seed=nx, Ms=8e5)
        s = OracleSolver([mesh], evaluation=0, dt=2e-14)
        s.set_m(M)
        s.run(10)
        c = _make(bm, prec, mesh, M, "RK4", 2e-14)
        c.run(10)
        t = c.tiles()
        m = c.get_m()
        c.close()
        assert t["stage_xv"] == 1
        assert np.abs(m - s.get_m()).max() / 8e5 < tol


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
@pytest.mark.parametrize("ny,W", [(128, 4), (256, 4), (512, 4), (1024, 2), (96, 2), (192, 1), (384, 1), (768, 1)])
def test_ypass_stockham_every_length(bm, ny, W, prec, tol, monkeypatch):
    """The Stockham y transform (3D; Ny = 256 .. 2048 with radix 16 and tails 16x16, 16x16x2,
    16x16x4, 16x16x8; Ny = 192 .. 1536 with radix 4 / 2 and a last radix-3 pass) against the
    oracle's RK4 trajectory with demag, exchange and Zeeman, for a ny that fills Ny / 2 and one that
    leaves zero rows below Ny / 2."""
    monkeypatch.setenv("BM_TILES", "1,%d,8,1" % W)
    monkeypatch.setenv("BM_Y_XV", "1")
    for n in [(8, ny, 2), (6, ny - 3, 3)]:
        N = n[0] * n[1] * n[2]
        mesh = dict(n=n, h=(3e-9, 3e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(2e3, 1e3, 0))
        M = sphere_random(N, seed=ny, Ms=8e5)
        s = OracleSolver([mesh], evaluation=0, dt=2e-14)
        s.set_m(M)
        s.run(10)
        c = _make(bm, prec, mesh, M, "RK4", 2e-14)
        c.run(10)
        t = c.tiles()
        m = c.get_m()
        c.close()
        assert t["ypass_yv"] == 1 and t["ypass_W"] == W
        assert np.abs(m - s.get_m()).max() / 8e5 < tol


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
@pytest.mark.parametrize("ny,W", [(4, 8), (8, 8), (16, 8), (32, 4), (64, 4), (128, 4), (256, 4), (512, 2)])
def test_ymid2d_register_every_length(bm, ny, W, prec, tol, monkeypatch):
    """The two-level register 2D y pass (forward, fused 2D kernel product, inverse) at every
    register length Ny = 8 .. 1024, with a power-of-two ny and one that leaves zero rows, against
    the oracle's RK4 trajectory with demag, exchange and Zeeman."""
    monkeypatch.setenv("BM_TILES", "%d,4,8,1" % W)
    for n in [(12, ny, 1), (9, max(ny - 1, 1), 1)]:
        N = n[0] * n[1] * n[2]
        mesh = dict(n=n, h=(3e-9, 3e-9, 2e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(2e3, 1e3, 0))
        M = sphere_random(N, seed=ny + 3, Ms=8e5)
        s = OracleSolver([mesh], evaluation=0, dt=2e-14)
        s.set_m(M)
        s.run(10)
        c = _make(bm, prec, mesh, M, "RK4", 2e-14)
        c.run(10)
        m = c.get_m()
        c.close()
        assert np.abs(m - s.get_m()).max() / 8e5 < tol


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
@pytest.mark.parametrize("nx", [256, 512, 1024])
@pytest.mark.parametrize("xv", ["2", "3"])
def test_stage_radix16_lengths(bm, nx, prec, tol, xv, monkeypatch):
    """The radix-16 Stockham x transform of the stage kernel (16 values and half the threads per
    line; radix tails 16x16, 16x16x2, 16x16x4) against the oracle with demag, exchange, iDMI,
    anisotropy and Zeeman, for a power-of-two nx and an odd one: RKDP54 with step control in FP64,
    fixed-step RK4 in mixed precision (an FP32 adaptive trajectory may choose other steps). Variant
    3 is the same kernel body compiled at the lower FP32 register cap."""
    monkeypatch.setenv("BM_TILES", "1,4,8,1")
    monkeypatch.setenv("BM_STAGE_XV", xv)
    for n in [(nx, 3, 2), (nx - 1, 2, 2)]:
        N = n[0] * n[1] * n[2]
        mesh = dict(n=n, h=(2e-9, 2e-9, 2e-9), Ms=1.1e6, A=1.5e-11, D=1.5e-3, alpha=0.1, K1=5e5,
                    modules=1 | 4 | 8 | 16, Ha=(1e3, 0, 0))
        M = tilted_z(N, seed=nx) * 1.1e6
        if prec == "fp64":
            s = OracleSolver([mesh], evaluation=1, dt=1e-14, tol=1e-5, dT_incr=2.0, dT_min=1e-15, dT_max=3e-12)
            c = _make(bm, prec, mesh, M, "RKDP54", 1e-14, (1e-5, 2.0, 1e-15, 3e-12))
        else:
            s = OracleSolver([mesh], evaluation=0, dt=2e-14)
            c = _make(bm, prec, mesh, M, "RK4", 2e-14)
        s.set_m(M)
        s.run(6)
        c.run(6)
        t = c.tiles()
        m = c.get_m()
        c.close()
        assert t["stage_xv"] == int(xv)
        assert np.abs(m - s.get_m()).max() / 1.1e6 < tol
