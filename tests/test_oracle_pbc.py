"""CPU tests of periodic boundary conditions in the oracle, pinned against the reference's own compiled
PBC code (oracle/_ref: DemagTFunc_PBC.cpp, the convolution set up with pbc_images, VEC_VC::set_pbc,
SelfDemag_PBC), plus a numpy restatement of the product's formulation (the periodic kernel made even
or odd per axis and embedded in the zero-padded convolution) checked against the oracle.

The reference's kernel multiplication handles the last transformed axis (y for a one-cell-thick
mesh, z otherwise) as if its length were even (Boris/DemagKernel.cpp:52-82,84-167): with an odd
periodic cell count there, one spectrum index is left unmultiplied and its field is not the periodic
convolution. For those shapes the oracle is pinned to a direct periodic convolution built from the
reference's own tensor instead."""
import numpy as np
import pytest

from oracle_libs import (oracle, reference, dp, orc_hdemag_pbc, ref_hdemag_pbc, orc_tensor_pbc, ref_tensor_pbc,
                         orc_kernels_pbc, ref_kernels_pbc, orc_stencil_pbc, ref_stencil_pbc, pbc_dims, _i3)

# (n, h, pbc images)
CASES = [
    ((16, 8, 1), (5e-9, 5e-9, 3e-9), (3, 0, 0)),
    ((16, 8, 1), (5e-9, 4e-9, 3e-9), (2, 3, 0)),
    ((12, 10, 1), (5e-9, 5e-9, 2e-9), (0, 0, 4)),
    ((9, 8, 1), (5e-9, 4e-9, 3e-9), (2, 0, 0)),
    ((8, 8, 4), (4e-9, 4e-9, 4e-9), (2, 2, 0)),
    ((6, 5, 4), (4e-9, 3e-9, 5e-9), (1, 2, 3)),
    ((5, 7, 4), (4e-9, 4e-9, 4e-9), (2, 1, 1)),
    ((10, 6, 3), (3e-9, 4e-9, 5e-9), (0, 2, 0)),
    ((8, 6, 2), (5e-9, 5e-9, 3e-9), (-2, 1, -1)),
    ((1, 8, 1), (5e-9, 5e-9, 3e-9), (3, 0, 0)),
    ((8, 1, 4), (5e-9, 5e-9, 3e-9), (0, 2, 2)),
]
# odd periodic cell count along the last transformed axis
ODD_LAST = [
    ((7, 5, 1), (5e-9, 4e-9, 3e-9), (2, 2, 1)),
    ((16, 7, 1), (5e-9, 5e-9, 3e-9), (0, 3, 0)),
    ((10, 6, 3), (3e-9, 4e-9, 5e-9), (0, 2, 1)),
]

# parity of xx, yy, zz, xy, xz, yz along x, y, z
PARITY = [(1, 1, 1), (1, 1, 1), (1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, -1, -1)]


def need_ref():
    r = reference()
    if r is None:
        pytest.skip("reference CPU build unavailable")
    return r


def _ids(c):
    return "n%dx%dx%d_pbc%d,%d,%d" % (c[0] + c[2])


def symmetrise(dg, od, pbc):
    """Per-axis even / odd part of an N-grid tensor (Nz, Ny, Nx, 3) along its periodic axes:
    (D(i) + p D((N - i) mod N)) / 2, the part the reference's per-axis Re / Im extraction keeps."""
    comps = [dg[..., 0], dg[..., 1], dg[..., 2], od[..., 0], od[..., 1], od[..., 2]]
    out = []
    for c, A in enumerate(comps):
        for ax, arr_ax in ((0, 2), (1, 1), (2, 0)):
            if pbc[ax]:
                A = 0.5 * (A + PARITY[c][ax] * np.roll(np.flip(A, axis=arr_ax), 1, axis=arr_ax))
        out.append(A)
    return out


def periodic_direct(S, M, n, N):
    """H = S * M as a cyclic convolution on the N grid (M zero-padded), from six real-space planes."""
    Mg = np.zeros((3, N[2], N[1], N[0]))
    Mg[:, :n[2], :n[1], :n[0]] = M.reshape(n[2], n[1], n[0], 3).transpose(3, 0, 1, 2)
    F = np.fft.fftn(Mg, axes=(1, 2, 3))
    K = [np.fft.fftn(A) for A in S]
    idx = [[0, 3, 4], [3, 1, 5], [4, 5, 2]]
    H = np.stack([np.real(np.fft.ifftn(sum(K[idx[a][b]] * F[b] for b in range(3)))) for a in range(3)])
    return H[:, :n[2], :n[1], :n[0]].transpose(1, 2, 3, 0).reshape(-1, 3)


@pytest.mark.parametrize("case", CASES + ODD_LAST, ids=_ids)
def test_pbc_tensor_vs_reference(case):
    need_ref()
    n, h, pbc = case
    dg, od = orc_tensor_pbc(n, h, pbc)
    rdg, rod = ref_tensor_pbc(n, h, pbc)
    assert dg.shape == rdg.shape
    scale = max(np.abs(rdg).max(), np.abs(rod).max())   # off-diagonals can vanish analytically (n = 1 axes)
    assert np.abs(dg - rdg).max() <= 1e-9 * scale
    assert np.abs(od - rod).max() <= 1e-9 * scale


@pytest.mark.parametrize("case", CASES + ODD_LAST, ids=_ids)
def test_pbc_kernels_vs_reference(case):
    need_ref()
    n, h, pbc = case
    kd, ko = orc_kernels_pbc(n, h, pbc)
    rkd, rko = ref_kernels_pbc(n, h, pbc)
    assert np.abs(kd - rkd).max() <= 5e-9 * np.abs(rkd).max()
    assert np.abs(ko - rko).max() <= 5e-9 * max(np.abs(rkd).max(), 1e-30)


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_pbc_hdemag_vs_reference(case):
    need_ref()
    n, h, pbc = case
    rng = np.random.default_rng(sum(n))
    M = rng.normal(size=(int(np.prod(n)), 3)) * 8e5
    H, dot = orc_hdemag_pbc(M, n, h, pbc)
    Hr, er = ref_hdemag_pbc(M, n, h, pbc)
    assert np.abs(H - Hr).max() <= 1e-9 * np.abs(Hr).max()
    e = -1.256637061435916e-6 * dot / (2.0 * np.prod(n))
    assert abs(e - er) <= 1e-9 * abs(er)


@pytest.mark.parametrize("case", ODD_LAST, ids=_ids)
def test_pbc_hdemag_odd_last_axis_is_the_periodic_convolution(case):
    """Pinned to the cyclic convolution with the reference's own tensor (made even / odd per periodic
    axis); the reference's own field differs there (its last-axis multiplication assumes an even length)."""
    need_ref()
    n, h, pbc = case
    rng = np.random.default_rng(7 + sum(n))
    M = rng.normal(size=(int(np.prod(n)), 3)) * 8e5
    N = pbc_dims(n, pbc)
    rdg, rod = ref_tensor_pbc(n, h, pbc)
    Hd = periodic_direct(symmetrise(rdg, rod, pbc), M, n, N)
    H, _ = orc_hdemag_pbc(M, n, h, pbc)
    assert np.abs(H - Hd).max() <= 1e-9 * np.abs(Hd).max()
    Hr, _ = ref_hdemag_pbc(M, n, h, pbc)
    assert np.abs(Hr - Hd).max() > 1e-3 * np.abs(Hd).max()   # the reference's deviation, as documented


@pytest.mark.parametrize("case", CASES + ODD_LAST, ids=_ids)
@pytest.mark.parametrize("idmi", [False, True])
def test_pbc_stencils_vs_reference(case, idmi):
    need_ref()
    n, h, pbc = case
    rng = np.random.default_rng(11 + sum(n))
    M = rng.normal(size=(int(np.prod(n)), 3))
    M *= 8e5 / np.linalg.norm(M, axis=1, keepdims=True)
    H = orc_stencil_pbc(M, n, h, pbc, 1.3e-11, 8e5, D=3e-3, idmi=idmi)
    Hr = ref_stencil_pbc(M, n, h, pbc, 1.3e-11, 8e5, D=3e-3, idmi=idmi)
    scale = max(np.abs(Hr).max(), 1e-30)
    assert np.abs(H - Hr).max() <= 1e-13 * scale


@pytest.mark.parametrize("case", CASES + ODD_LAST, ids=_ids)
def test_pbc_selfdemag_vs_reference(case):
    """SelfDemag_PBC on normalised cellsizes (the reference's own function, fed h / max h)."""
    R = need_ref()
    n, h, pbc = case
    s = np.zeros(3)
    sr = np.zeros(3)
    hm = max(h)
    oracle().orc_selfdemag_pbc(h[0], h[1], h[2], _i3(n), _i3(pbc), dp(s))
    R.ref_selfdemag_pbc(h[0] / hm, h[1] / hm, h[2] / hm, n[0], n[1], n[2], _i3(pbc), dp(sr))
    assert np.abs(s - sr).max() <= 1e-12


def _free_tensor(h, ext):
    """Free-space D = -N at non-negative offsets [0, ext) per axis: (ext_z, ext_y, ext_x, 6)."""
    nx, ny, nz = ext
    N = (2 * nx, 2 * ny, 2 * nz if nz > 1 else 1)
    np_ = N[0] * N[1] * N[2]
    dg = np.zeros(3 * np_)
    od = np.zeros(3 * np_)
    oracle().orc_tensor(nx, ny, nz, N[0], N[1], N[2], h[0], h[1], h[2], dp(dg), dp(od))
    dg = dg.reshape(N[2], N[1], N[0], 3)[:nz, :ny, :nx]
    od = od.reshape(N[2], N[1], N[0], 3)[:nz, :ny, :nx]
    return np.concatenate([dg, od], axis=3)


def product_octant(n, h, pbc):
    """The product's periodic octant (tensor.cu, k_tensor_octant_pbc) restated in numpy: along a periodic
    axis with X images, Ds(0) = sum_{m=-X..X} T(m n) (odd components 0) and, for i0 > 0,
    Ds(i0) = sum_{m=-X-1..X} w_m T(m n + i0) with w = 1/2 at both ends; T of odd components carries the
    sign of each offset (sign(0) = 0)."""
    X = [abs(v) for v in pbc]
    two_d = n[2] == 1
    ext = [(X[a] + 2) * n[a] if X[a] else n[a] for a in range(3)]
    if two_d:
        ext[2] = X[2] + 1
    T = _free_tensor(h, ext)
    out = np.zeros((n[2], n[1], n[0], 6))
    rng_of = []
    for a in range(3):
        r = []
        for q in range(n[a]):
            if not X[a]:
                r.append([(q, 1.0)])
            elif q == 0:
                r.append([(m * n[a], 1.0) for m in range(-X[a], X[a] + 1)])
            else:
                r.append([(m * n[a] + q, 0.5 if m in (-X[a] - 1, X[a]) else 1.0) for m in range(-X[a] - 1, X[a] + 1)])
        rng_of.append(r)
    for k in range(n[2]):
        for j in range(n[1]):
            for i in range(n[0]):
                acc = np.zeros(6)
                for oi, wi in rng_of[0][i]:
                    for oj, wj in rng_of[1][j]:
                        for ok, wk in rng_of[2][k]:
                            v = T[abs(ok), abs(oj), abs(oi)]
                            si, sj, sk = np.sign(oi), np.sign(oj), np.sign(ok)
                            sg = np.array([1, 1, 1, si * sj, si * sk, sj * sk])
                            acc += wi * wj * wk * v * sg
                for a, q in enumerate((i, j, k)):
                    if X[a] and q == 0:
                        for c in range(3, 6):
                            if PARITY[c][a] < 0:
                                acc[c] = 0.0
                out[k, j, i] = acc
    return out


@pytest.mark.parametrize("case", [((6, 4, 1), (5e-9, 4e-9, 3e-9), (2, 1, 0)), ((5, 4, 1), (4e-9, 4e-9, 3e-9), (1, 0, 2)),
                                  ((4, 3, 4), (4e-9, 3e-9, 5e-9), (1, 2, 1))], ids=_ids)
def test_product_octant_formula_is_the_symmetrised_tensor(case):
    """The weighted image sum the product evaluates equals the reference-style tensor made even / odd
    about the origin along each periodic axis (both from the oracle's Newell / far-field values)."""
    n, h, pbc = case
    oc = product_octant(n, h, pbc)
    dg, od = orc_tensor_pbc(n, h, pbc)
    S = symmetrise(dg, od, pbc)
    for c in range(6):
        ref = S[c][:n[2], :n[1], :n[0]]
        if n[2] == 1 and c >= 4:
            continue
        assert np.abs(oc[..., c] - ref).max() <= 1e-13 * max(np.abs(S[c]).max(), 1e-30), c


@pytest.mark.parametrize("case", [((6, 4, 1), (5e-9, 4e-9, 3e-9), (2, 1, 0)), ((5, 4, 1), (4e-9, 4e-9, 3e-9), (1, 0, 2)),
                                  ((4, 3, 4), (4e-9, 3e-9, 5e-9), (1, 2, 1)), ((7, 5, 1), (5e-9, 4e-9, 3e-9), (2, 2, 1))],
                         ids=_ids)
def test_product_embedding_is_the_periodic_convolution(case):
    """The product's formulation: the periodic octant placed in the zero-padded grid (N = 2n on every
    axis, mirrored with the components' parity) gives the cyclic convolution of period n."""
    n, h, pbc = case
    oc = product_octant(n, h, pbc)
    N = (2 * n[0], 2 * n[1], 2 * n[2] if n[2] > 1 else 1)
    S = []
    for c in range(6):
        A = np.zeros((N[2], N[1], N[0]))
        for k in range(N[2]):
            ak, sz = (k, 1) if k <= N[2] // 2 else (N[2] - k, -1)
            for j in range(N[1]):
                aj, sy = (j, 1) if j <= N[1] // 2 else (N[1] - j, -1)
                for i in range(N[0]):
                    ai, sx = (i, 1) if i <= N[0] // 2 else (N[0] - i, -1)
                    if ai < n[0] and aj < n[1] and ak < n[2]:
                        p = PARITY[c]
                        sgn = (p[0] if sx < 0 else 1) * (p[1] if sy < 0 else 1) * (p[2] if sz < 0 else 1)
                        A[k, j, i] = oc[ak, aj, ai, c] * sgn
        S.append(A)
    rng = np.random.default_rng(5)
    M = rng.normal(size=(int(np.prod(n)), 3)) * 8e5
    H = periodic_direct(S, M, n, N)
    Ho, _ = orc_hdemag_pbc(M, n, h, pbc)
    assert np.abs(H - Ho).max() <= 1e-10 * np.abs(Ho).max()


def test_pbc_dims_follow_the_reference():
    assert pbc_dims((16, 8, 1), (3, 0, 0)) == (16, 16, 1)
    assert pbc_dims((16, 8, 4), (0, 2, 1)) == (32, 8, 4)
    assert pbc_dims((16, 8, 4), (0, 0, 0)) == (32, 16, 8)
