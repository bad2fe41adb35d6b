"""CPU tests of the oracle: the project's FP64 restatement (oracle/oracle.c) pinned against
the reference's own compiled CPU code (oracle/_ref), against the committed golden fixtures
(tests/golden/, made by tests/golden/make_golden.py from the reference build), and against
known answers (self-demag trace, DFT definition, far-field vs exact Newell)."""
import os

import numpy as np
import pytest

from oracle_libs import (oracle, reference, dp, orc_hdemag, ref_hdemag, OracleSolver, sphere_random, tilted_z)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden.npz")
MU0 = 1.256637061435916e-6


def need_ref():
    r = reference()
    if r is None:
        pytest.skip("reference CPU build unavailable")
    return r


# ---------------------------------------------------------------- FFT shim
@pytest.mark.parametrize("L", [1, 2, 3, 5, 6, 7, 8, 12, 15, 16, 30, 64, 96, 100, 128])
def test_fft_shim_matches_dft_definition(L):
    rng = np.random.default_rng(L)
    x = rng.normal(size=L) + 1j * rng.normal(size=L)
    buf = np.ascontiguousarray(np.stack([x.real, x.imag], axis=1).reshape(-1))
    oracle().bm_oracle_fft(L, dp(buf), -1)
    got = buf[0::2] + 1j * buf[1::2]
    k = np.arange(L)
    ref = (x[None, :] * np.exp(-2j * np.pi * np.outer(k, k) / L)).sum(axis=1)
    assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


# ---------------------------------------------------------------- Newell tensor
@pytest.mark.parametrize("h", [(5, 5, 3), (2, 2, 2), (4, 4, 3), (1, 2, 3.5), (1, 1, 0.2)])
def test_selfdemag_trace_is_minus_one(h):
    o = np.zeros(3)
    oracle().orc_selfdemag(h[0], h[1], h[2], dp(o))
    assert abs(o.sum() + 1.0) < 1e-13
    if h[0] == h[1] == h[2]:
        assert np.allclose(o, -1.0 / 3, atol=1e-14)


@pytest.mark.parametrize("h", [(5, 5, 3), (1, 2, 3.5)])
def test_selfdemag_vs_reference(h):
    R = need_ref()
    a = np.zeros(3)
    b = np.zeros(3)
    R.ref_selfdemag(h[0], h[1], h[2], dp(a))
    oracle().orc_selfdemag(h[0], h[1], h[2], dp(b))
    assert np.abs(a - b).max() < 1e-14


@pytest.mark.parametrize("h", [(1.0, 1.0, 1.0), (1.0, 1.0, 0.6), (0.5, 1.0, 0.75)])
def test_far_field_expansion_vs_exact_newell(h):
    """The project's far-field expansion agrees with exact Newell where both are accurate."""
    L = oracle()
    rng = np.random.default_rng(3)
    worst = 0.0
    for _ in range(40):
        d = rng.normal(size=3)
        d *= rng.uniform(8, 14) / np.linalg.norm(d)
        x, y, z = d[0] * h[0], d[1] * h[1], d[2] * h[2]
        a = np.zeros(6)
        L.orc_asymptotic(h[0], h[1], h[2], x, y, z, dp(a))
        # exact Newell at the same offset through the tensor fill of a tiny grid is index based;
        # compare with the 27-point formula via orc_tensor at integer offsets instead
        worst = max(worst, 0.0)
    # integer offsets: tensor cells at distance 8..14 computed exactly, far formula directly
    n = (16, 16, 16) if h[2] == 1.0 else (16, 16, 12)
    N = tuple(2 * v for v in n)
    dg = np.zeros(3 * N[0] * N[1] * N[2])
    od = np.zeros_like(dg)
    L.orc_tensor(n[0], n[1], n[2], N[0], N[1], N[2], h[0], h[1], h[2], dp(dg), dp(od))
    dg = dg.reshape(N[2], N[1], N[0], 3)
    od = od.reshape(N[2], N[1], N[0], 3)
    hm = max(h)
    hn = (h[0] / hm, h[1] / hm, h[2] / hm)
    for (i, j, k) in [(9, 3, 2), (4, 10, 1), (2, 5, 9), (8, 8, 8), (11, 0, 0), (0, 0, 11)]:
        if k >= n[2]:
            continue
        a = np.zeros(6)
        L.orc_asymptotic(hn[0], hn[1], hn[2], i * hn[0], j * hn[1], k * hn[2], dp(a))
        ex = np.concatenate([dg[k, j, i], od[k, j, i]])
        scale = np.abs(ex).max()
        worst = max(worst, np.abs(a - ex).max() / scale)
    assert worst < 1e-6


@pytest.mark.parametrize("n,h", [((8, 6, 1), (5, 5, 3)), ((6, 5, 4), (2, 2, 2)), ((50, 45, 1), (4, 4, 3)),
                                 ((45, 7, 3), (1, 2, 3.5)), ((64, 48, 2), (2, 2, 1))])
def test_tensor_vs_reference(n, h):
    R = need_ref()
    nx, ny, nz = n
    N = (2 * nx, 2 * ny, 2 * nz if nz > 1 else 1)
    npt = N[0] * N[1] * N[2]
    rd, ro, od_, oo = (np.zeros(3 * npt) for _ in range(4))
    R.ref_tensor(nx, ny, nz, *N, *h, dp(rd), dp(ro))
    oracle().orc_tensor(nx, ny, nz, *N, *h, dp(od_), dp(oo))
    assert np.abs(rd - od_).max() < 5e-11
    assert np.abs(ro - oo).max() < 5e-11


@pytest.mark.parametrize("n,h", [((8, 6, 1), (5, 5, 3)), ((6, 5, 4), (2, 2, 2)), ((50, 45, 1), (4, 4, 3)),
                                 ((12, 7, 3), (1, 2, 3.5))])
def test_kernels_vs_reference(n, h):
    R = need_ref()
    nx, ny, nz = n
    N = (2 * nx, 2 * ny, 2 * nz if nz > 1 else 1)
    nk = (N[0] // 2 + 1) * (N[1] // 2 + 1) * (N[2] // 2 + 1)
    rkd = np.zeros(3 * nk)
    rko = np.zeros(3 * nk if nz > 1 else nk)
    okd = np.zeros(3 * nk)
    oko = np.zeros(3 * nk)
    R.ref_kernels(nx, ny, nz, *h, dp(rkd), dp(rko))
    oracle().orc_kernels(nx, ny, nz, *N, *h, dp(okd), dp(oko))
    assert np.abs(rkd - okd).max() < 1e-9
    assert np.abs(rko - (oko if nz > 1 else oko[0::3])).max() < 1e-9


@pytest.mark.parametrize("n,h", [((16, 8, 1), (5e-9, 5e-9, 3e-9)), ((10, 6, 4), (2e-9, 2e-9, 2e-9)),
                                 ((64, 32, 1), (5e-9, 5e-9, 3e-9)), ((30, 20, 5), (4e-9, 4e-9, 3e-9)),
                                 ((5, 3, 1), (2e-9, 3e-9, 1e-9))])
def test_hdemag_vs_reference(n, h):
    need_ref()
    N = n[0] * n[1] * n[2]
    M = sphere_random(N, seed=1, Ms=8e5)
    Hr, er = ref_hdemag(M, n, h)
    Ho, dot = orc_hdemag(M, n, h)
    assert np.abs(Hr - Ho).max() / np.abs(Hr).max() < 1e-9
    assert abs(er - (-MU0 * dot / (2 * N))) < 1e-9 * abs(er)


def test_hdemag_fft_size_independent():
    """Any FFT size >= 2n gives the same linear convolution (the GPU pads to 2^p or 3*2^p)."""
    n, h = (5, 3, 3), (2e-9, 3e-9, 1e-9)
    M = sphere_random(45, seed=2, Ms=8e5)
    a, _ = orc_hdemag(M, n, h, N=(10, 6, 6))
    b, _ = orc_hdemag(M, n, h, N=(12, 8, 8))
    assert np.abs(a - b).max() / np.abs(a).max() < 1e-12


@pytest.mark.parametrize("n", [(7, 5, 1), (6, 5, 4), (1, 5, 3), (9, 1, 1), (5, 4, 2)])
def test_stencils_vs_reference(n):
    R = need_ref()
    nx, ny, nz = n
    N = nx * ny * nz
    h = (2e-9, 3e-9, 1.5e-9)
    rng = np.random.default_rng(2)
    Ms = rng.uniform(5e5, 1e6, N)
    M = np.ascontiguousarray((sphere_random(N, seed=3) * Ms[:, None]).reshape(-1))
    A = np.full(N, 1.3e-11)
    Dm = np.full(N, 1.5e-3)
    for which in ("exch", "idmi"):
        Hr = np.zeros(3 * N)
        Ho = np.zeros(3 * N)
        if which == "exch":
            R.ref_exchange(nx, ny, nz, *h, dp(M), dp(A), dp(Ms), dp(Hr))
            oracle().orc_field_exchange(nx, ny, nz, *h, dp(M), 1.3e-11, dp(Ms), dp(Ho))
        else:
            R.ref_idmi(nx, ny, nz, *h, dp(M), dp(A), dp(Dm), dp(Ms), dp(Hr))
            oracle().orc_field_idmi(nx, ny, nz, *h, dp(M), 1.3e-11, 1.5e-3, dp(Ms), dp(Ho))
        scale = max(np.abs(Hr).max(), 1e-300)
        assert np.abs(Hr - Ho).max() / scale < 1e-13, which


# ---------------------------------------------------------------- golden fixtures
def test_golden_fixtures():
    """The oracle reproduces the committed outputs of the reference build."""
    if not os.path.exists(GOLDEN):
        pytest.skip("golden fixtures not generated")
    g = np.load(GOLDEN)
    for key in [k for k in g.files if k.startswith("hdemag_")]:
        tag = key[len("hdemag_"):]
        n = tuple(int(v) for v in g["n_" + tag])
        h = tuple(float(v) for v in g["h_" + tag])
        Ho, _ = orc_hdemag(g["M_" + tag], n, h)
        assert np.abs(Ho - g[key]).max() / np.abs(g[key]).max() < 1e-9, tag
    for key in [k for k in g.files if k.startswith("kdiag_")]:
        tag = key[len("kdiag_"):]
        n = tuple(int(v) for v in g["kn_" + tag])
        h = tuple(float(v) for v in g["kh_" + tag])
        N = (2 * n[0], 2 * n[1], 2 * n[2] if n[2] > 1 else 1)
        nk = (N[0] // 2 + 1) * (N[1] // 2 + 1) * (N[2] // 2 + 1)
        okd = np.zeros(3 * nk)
        oko = np.zeros(3 * nk)
        oracle().orc_kernels(*n, *N, *h, dp(okd), dp(oko))
        assert np.abs(okd - g[key]).max() < 1e-9, tag
    s = g["selfdemag"]
    for row in s:
        o = np.zeros(3)
        oracle().orc_selfdemag(row[0], row[1], row[2], dp(o))
        assert np.abs(o - row[3:]).max() < 1e-14


# ---------------------------------------------------------------- integrators (oracle alone)
def test_oracle_rk4_norm_and_convergence():
    """RK4 keeps |M| = Ms and converges at 4th order in dt (self-consistency)."""
    n = (8, 8, 1)
    mesh = dict(n=n, h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16, Ha=(1e4, 0, 0))
    M = sphere_random(64, seed=7, Ms=8e5)
    res = {}
    for dt, steps in ((4e-14, 50), (2e-14, 100), (1e-14, 200)):
        s = OracleSolver([mesh], evaluation=0, dt=dt)
        s.set_m(M)
        s.run(steps)
        res[dt] = s.get_m() / 8e5
        s.close()
    assert np.abs(np.linalg.norm(res[1e-14], axis=1) - 1).max() < 1e-12
    e1 = np.abs(res[4e-14] - res[1e-14]).max()
    e2 = np.abs(res[2e-14] - res[1e-14]).max()
    assert e1 / e2 > 8.0   # ~ (2^4 - 1) / 1 for 4th order


def test_oracle_rkdp_rejects_and_recovers():
    n = (8, 8, 1)
    mesh = dict(n=n, h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16, Ha=(1e4, 0, 0))
    M = sphere_random(64, seed=21, Ms=8e5)
    s = OracleSolver([mesh], evaluation=1, dt=2e-12, tol=1e-6, dT_incr=2.0, dT_min=1e-16, dT_max=1e-11)
    s.set_m(M)
    st = s.run(20)
    assert st["accepted"] == 20 and st["rejected"] > 0
    assert np.abs(np.linalg.norm(s.get_m(), axis=1) / 8e5 - 1).max() < 1e-12


@pytest.mark.parametrize("modules", [1 | 4 | 8 | 16, 1 | 2 | 16])
def test_solver_with_reference_fields_matches_restatement(modules):
    """The CPU baseline's solver (demag and exchange / iDMI from the reference's compiled code,
    the rest restated) follows the pure restatement's RKDP54 trajectory to FP64 round-off."""
    if reference() is None:
        pytest.skip("reference build absent")
    n, h = (24, 16, 4), (2e-9, 2e-9, 2e-9)
    mesh = dict(n=n, h=h, Ms=1.1e6, A=1.5e-11, D=1.5e-3, K1=5e5, alpha=0.1, modules=modules, Ha=(1e3, 2e3, 0))
    M = tilted_z(n[0] * n[1] * n[2], seed=5, Ms=1.1e6)
    out = []
    for use_ref in (False, True):
        s = OracleSolver([mesh], evaluation=1, dt=1e-14, tol=1e-5, dT_incr=2.0, dT_min=1e-15, dT_max=3e-12)
        if use_ref:
            assert s.use_reference_fields(0)
        s.set_m(M)
        st = s.run(8)
        out.append((s.get_m(), st))
        s.close()
    (m0, s0), (m1, s1) = out
    assert s0["accepted"] == s1["accepted"] and s0["rejected"] == s1["rejected"]
    assert abs(s0["time"] - s1["time"]) <= 1e-9 * s0["time"]
    assert np.abs(m1 - m0).max() / 1.1e6 < 1e-9
