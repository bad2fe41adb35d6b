"""CPU tests of the oracle's multilayered convolution (SDemag multilayer mode): the project's
FP64 restatement (oracle/oracle.c, orc_ml_*) against the reference's own DemagKernelCollection,
Convolution and VEC mesh-transfer code compiled from its sources (oracle/_ref, ref_ml_*).

Covered: layer geometry (n_common, enlarged rectangles, transfer flags, kernel kinds incl. the
2D inverse z-shift reuse), the weighted mesh transfer in both directions, and H_demag in 3D,
2D and 2D-layered modes, with in-plane shifts (full complex kernels), unequal thicknesses
(irregular 2D kernels) and meshes wider than the 40-cell near-field radius."""
import numpy as np
import pytest

from oracle_libs import MultiLayer, reference, oracle, dp, sphere_random, orc_hdemag, OracleSolver

NM = 1e-9
# three stacked meshes of the multilayer configuration, scaled down (16 x 16 in-plane)
STACK3 = [((16, 16, 1), (2 * NM, 2 * NM, 1 * NM), (0, 0, 0)),
          ((8, 8, 2), (4 * NM, 4 * NM, 2 * NM), (0, 0, 2 * NM)),
          ((16, 16, 1), (2 * NM, 2 * NM, 1.5 * NM), (0, 0, 7 * NM))]
SHIFTED_XY = [((12, 10, 1), (3 * NM, 3 * NM, 2 * NM), (0, 0, 0)),
              ((12, 10, 1), (3 * NM, 3 * NM, 2 * NM), (9 * NM, 6 * NM, 3 * NM))]
SHIFTED_XY_IRR = [((12, 10, 1), (3 * NM, 3 * NM, 2 * NM), (0, 0, 0)),
                  ((12, 10, 1), (3 * NM, 3 * NM, 1 * NM), (9 * NM, 6 * NM, 3 * NM))]
WIDE_EQ = [((48, 44, 1), (2 * NM, 2 * NM, 1 * NM), (0, 0, 0)),
           ((48, 44, 1), (2 * NM, 2 * NM, 1 * NM), (0, 0, 2 * NM))]
WIDE_IRR = [((48, 44, 1), (2 * NM, 2 * NM, 1 * NM), (0, 0, 0)),
            ((48, 44, 1), (2 * NM, 2 * NM, 3 * NM), (0, 0, 2 * NM))]
WIDE_LAYERED = [((48, 44, 1), (2 * NM, 2 * NM, 1 * NM), (0, 0, 0)),
                ((24, 22, 2), (4 * NM, 4 * NM, 1 * NM), (0, 0, 2 * NM))]

CASES = [
    ("stack3_3d", STACK3, 0, None),
    ("stack3_2d", STACK3, 1, None),
    ("stack3_2d_layered", STACK3, 2, None),
    ("shifted_xy_3d", SHIFTED_XY, 0, None),
    ("shifted_xy_irregular_2d", SHIFTED_XY_IRR, 1, None),
    ("wide_equal", WIDE_EQ, 0, None),
    ("wide_irregular", WIDE_IRR, 0, None),
    ("wide_layered", WIDE_LAYERED, 2, None),
    ("stack3_ncommon_8_8_4", STACK3, 0, (8, 8, 4)),
    ("stack3_ncommon_16_16_1", STACK3, 0, (16, 16, 1)),
]


def need_ref():
    r = reference()
    if r is None:
        pytest.skip("reference CPU build unavailable")
    return r


@pytest.mark.parametrize("name,meshes,mode,nc", CASES, ids=[c[0] for c in CASES])
def test_ml_geometry_and_field_match_reference(name, meshes, mode, nc):
    need_ref()
    a = MultiLayer(meshes, mode, nc, which="reference")
    b = MultiLayer(meshes, mode, nc, which="oracle")
    ia, ib = a.info(), b.info()
    assert ia["L"] == ib["L"]
    assert ia["n_common"] == ib["n_common"]
    assert ia["layer_mesh"] == ib["layer_mesh"]
    assert ia["transfer"] == ib["transfer"]
    assert np.allclose(ia["rects"], ib["rects"], rtol=0, atol=1e-18)
    assert (ia["kinds"] == ib["kinds"]).all()
    n = sum(a.ncell)
    M = sphere_random(n, seed=11, Ms=8e5)
    Ha, Hb = a.eval(M), b.eval(M)
    # FP64 both; the reference tabulates f/g while the oracle evaluates them per point
    assert np.abs(Ha - Hb).max() <= 2e-9 * np.abs(Ha).max()


def test_ml_kernel_kinds_of_the_stack():
    """3D stack: one self kernel per layer and z-shifted kernels between layers; 2D-layered:
    the opposite z shift between equal-thickness layers reuses the kernel (kind 3)."""
    i3 = MultiLayer(STACK3, 0).info()
    assert i3["n_common"] == (16, 16, 2) and i3["transfer"] == [1, 1, 1]
    assert (np.diag(i3["kinds"]) == 1).all() and (i3["kinds"][~np.eye(3, dtype=bool)] == 2).all()
    il = MultiLayer(STACK3, 2).info()
    assert il["L"] == 4 and il["layer_mesh"] == [0, 1, 1, 2] and il["n_common"] == (16, 16, 1)
    assert il["kinds"][2, 1] == 3


@pytest.mark.parametrize("name,meshes,mode", [("stack3_3d", STACK3, 0), ("stack3_2d_layered", STACK3, 2),
                                              ("wide_layered", WIDE_LAYERED, 2)])
def test_ml_transfer_matches_reference(name, meshes, mode):
    need_ref()
    a = MultiLayer(meshes, mode, which="reference")
    b = MultiLayer(meshes, mode, which="oracle")
    info = a.info()
    ncc = int(np.prod(info["n_common"]))
    n = sum(a.ncell)
    M = sphere_random(n, seed=5, Ms=1.0)
    rng = np.random.default_rng(6)
    for layer in range(info["L"]):
        if not info["transfer"][layer]:
            continue
        Hc = rng.normal(size=(ncc, 3))
        Mc_a, Hm_a = a.transfer(layer, M, Hc, ncc)
        Mc_b, Hm_b = b.transfer(layer, M, Hc, ncc)
        assert np.abs(Mc_a - Mc_b).max() <= 1e-14
        assert np.abs(Hm_a - Hm_b).max() <= 1e-14 * max(1.0, np.abs(Hm_a).max())


def test_ml_transfer_known_weights():
    """3D stack: the 1 nm layer fills half of its first 2 nm common cell (weight 0.5), the 4 nm
    cells of the middle mesh map one-to-one onto the common cells they contain, and each
    mesh cell reads back the common cells inside it with equal weights."""
    b = MultiLayer(STACK3, 0)
    info = b.info()
    ncc = int(np.prod(info["n_common"]))
    n = sum(b.ncell)
    M = sphere_random(n, seed=9, Ms=1.0)
    Hc = np.random.default_rng(3).normal(size=(ncc, 3))
    Mc, Hm = b.transfer(0, M, Hc, ncc)
    Mc = Mc.reshape(2, 16, 16, 3)
    assert np.allclose(Mc[0].reshape(-1, 3), 0.5 * M[:256], atol=1e-15)
    assert np.abs(Mc[1]).max() == 0.0
    assert np.allclose(Hm, Hc.reshape(2, 16, 16, 3)[0].reshape(-1, 3), atol=1e-15)
    Mc1, Hm1 = b.transfer(1, M, Hc, ncc)
    M1 = M[256:256 + 128].reshape(2, 8, 8, 3)
    Mc1 = Mc1.reshape(2, 16, 16, 3)
    assert np.allclose(Mc1[:, ::2, ::2], M1, atol=1e-15) and np.allclose(Mc1[:, 1::2, 1::2], M1, atol=1e-15)
    H4 = Hc.reshape(2, 8, 2, 8, 2, 3).mean(axis=(2, 4))
    assert np.allclose(Hm1.reshape(2, 8, 8, 3), H4, atol=1e-14)


def test_ml_single_mesh_equals_plain_demag():
    """One mesh in multilayer mode is the plain demag convolution."""
    mesh = ((12, 8, 3), (5 * NM, 5 * NM, 3 * NM), (0, 0, 0))
    b = MultiLayer([mesh], 0)
    M = sphere_random(12 * 8 * 3, seed=2, Ms=8e5)
    H = b.eval(M)
    H0, _ = orc_hdemag(M, (12, 8, 3), (5e-9, 5e-9, 3e-9))
    assert np.abs(H - H0).max() <= 1e-11 * np.abs(H0).max()


def test_ml_solver_runs_stack():
    """The oracle solver with a multilayered demag advances the three-mesh stack."""
    meshes = [dict(n=m[0], h=m[1], Ms=Ms, A=1.5e-11, alpha=0.05, modules=1 | 2)
              for m, Ms in zip(STACK3, (1.4e6, 6e5, 1.1e6))]
    s = OracleSolver(meshes, evaluation=0, dt=1e-13)
    s.multilayer([m[2] for m in STACK3], mode=0)
    for q, m in enumerate(meshes):
        s.set_m(sphere_random(int(np.prod(m["n"])), seed=q, Ms=m["Ms"]), q)
    st = s.run(3)
    assert st["accepted"] == 3
    for q, m in enumerate(meshes):
        Mq = s.get_m(q)
        assert np.allclose(np.linalg.norm(Mq, axis=1), m["Ms"], rtol=1e-12)


def _box_tensor(i, j, hs, hd, shift, order=12):
    """D = -N between a source cell (hs, at the origin) and a destination cell (hd, at (i, j)
    cells and z offset shift) by Gauss-Legendre integration of the dipole kernel."""
    g, w = np.polynomial.legendre.leggauss(order)

    def box(a0, a1):
        return a0 + (a1 - a0) * (g + 1) / 2, w * (a1 - a0) / 2

    ax = [box(i * hd[0], (i + 1) * hd[0]), box(j * hd[1], (j + 1) * hd[1]), box(shift, shift + hd[2]),
          box(0, hs[0]), box(0, hs[1]), box(0, hs[2])]

    def e(a, k):
        return a.reshape([-1 if q == k else 1 for q in range(6)])

    X = e(ax[0][0], 0) - e(ax[3][0], 3)
    Y = e(ax[1][0], 1) - e(ax[4][0], 4)
    Z = e(ax[2][0], 2) - e(ax[5][0], 5)
    W = e(ax[0][1], 0) * e(ax[1][1], 1) * e(ax[2][1], 2) * e(ax[3][1], 3) * e(ax[4][1], 4) * e(ax[5][1], 5)
    R = np.sqrt(X * X + Y * Y + Z * Z)
    V = hd[0] * hd[1] * hd[2]
    f = lambda K: -(W * K).sum() / (4 * np.pi * V)
    return np.array([f(1 / R**3 - 3 * X * X / R**5), f(1 / R**3 - 3 * Y * Y / R**5), f(1 / R**3 - 3 * Z * Z / R**5),
                     f(-3 * X * Y / R**5), f(-3 * X * Z / R**5), f(-3 * Y * Z / R**5)])


def test_reference_irregular_2d_tensor_against_exact_integral():
    """Documents how the reference builds 2D kernels between layers of unequal thickness
    (DemagTFunc_Irregular.cpp): xx and yy agree with the exact cell-averaged dipole integral,
    zz and the off-diagonal terms use the source and destination thicknesses the other way
    round, and past 40 cells the far field is scaled by the destination thickness (in units
    of the largest cellsize). Equal thicknesses agree everywhere. The product reproduces the
    reference as it is."""
    R = need_ref()
    n, N = (48, 8, 1), (96, 16, 1)

    def ref_t(hs, hd, sz, asympt):
        d = np.zeros((96 * 16, 3))
        o = np.zeros((96 * 16, 3))
        rc = R.ref_tensor_shifted(1, *n, *N, dp(np.array(hs, float)), dp(np.array(hd, float)),
                                  dp(np.array([0.0, 0.0, sz])), asympt, dp(d), dp(o))
        assert rc == 0
        return np.concatenate([d, o], axis=1).reshape(16, 96, 6)

    hs, hd = (1.0, 1.0, 0.3), (1.0, 1.0, 0.6)
    t = ref_t(hs, hd, 1.0, 40)
    exact = _box_tensor(2, 1, hs, hd, 1.0)
    got = t[1, 2]
    rel = np.abs(got - exact) / np.abs(exact)
    assert rel[0] < 1e-6 and rel[1] < 1e-6            # xx, yy exact
    assert rel[2] > 0.5 and rel[3] > 0.1              # zz, xy differ
    # far field: 40 cells out, exact sums vs the asymptotic branch differ by d.z = 0.6
    near = ref_t(hs, hd, 1.0, 0)
    assert abs(t[0, 40, 0] / near[0, 40, 0] - 0.6) < 1e-3
    # equal thicknesses: everything exact and continuous
    he = (1.0, 1.0, 0.5)
    te = ref_t(he, he, 1.0, 40)
    ex = _box_tensor(2, 1, he, he, 1.0)
    assert (np.abs(te[1, 2] - ex) / np.abs(ex)).max() < 1e-6
    ne = ref_t(he, he, 1.0, 0)
    assert abs(te[0, 40, 0] / ne[0, 40, 0] - 1.0) < 1e-4
