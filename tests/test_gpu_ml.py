"""GPU parity of the multilayered convolution (C ABI on cuda:0) against the oracle's
restatement and the reference's own DemagKernelCollection build.

Tolerances: H_demag FP64 <= 1e-9 of max |H|, mixed precision <= 1e-5 (the stated demag
tolerance); runs FP64 <= 1e-9 max |m - m_ref| / Ms, mixed <= 1e-4."""
import numpy as np
import pytest

from oracle_libs import MultiLayer, OracleSolver, reference, sphere_random, tilted_z
from test_oracle_ml import (STACK3, SHIFTED_XY, SHIFTED_XY_IRR, WIDE_EQ, WIDE_IRR, WIDE_LAYERED)

pytestmark = pytest.mark.gpu

NM = 1e-9
MS3 = (1.4e6, 6e5, 1.1e6)

GPU_CASES = [
    ("stack3_3d", STACK3, 0, None),
    ("stack3_2d", STACK3, 1, None),
    ("stack3_2d_layered", STACK3, 2, None),
    ("shifted_xy_3d", SHIFTED_XY, 0, None),
    ("shifted_xy_irregular_2d", SHIFTED_XY_IRR, 1, None),
    ("wide_equal", WIDE_EQ, 0, None),
    ("wide_irregular", WIDE_IRR, 0, None),
    ("wide_layered", WIDE_LAYERED, 2, None),
    ("stack3_ncommon_8_8_4", STACK3, 0, (8, 8, 4)),
]


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _ctx(bm, meshes, mode, nc, prec, modules=None):
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    for n, h, o in meshes:
        c.add_mesh(n, h, o)
    for i in range(len(meshes)):
        c.set_modules(i, bm.DEMAG if modules is None else modules)
    c.multiconvolution(mode, nc)
    return c


def _split(M, meshes):
    out, off = [], 0
    for n, _, _ in meshes:
        k = n[0] * n[1] * n[2]
        out.append(M[off:off + k])
        off += k
    return out


@pytest.mark.parametrize("name,meshes,mode,nc", GPU_CASES, ids=[c[0] for c in GPU_CASES])
def test_ml_geometry_matches_oracle(bm, name, meshes, mode, nc):
    o = MultiLayer(meshes, mode, nc).info()
    with _ctx(bm, meshes, mode, nc, "fp64") as c:
        g = c.ml_info()
    assert g["L"] == o["L"] and g["n_common"] == o["n_common"]
    assert g["layer_mesh"] == o["layer_mesh"] and g["transfer"] == o["transfer"]
    assert np.allclose(g["rects"], o["rects"], rtol=0, atol=1e-18)
    assert (g["kinds"] == o["kinds"]).all()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name,meshes,mode,nc", GPU_CASES, ids=[c[0] for c in GPU_CASES])
def test_ml_hdemag_matches_oracle(bm, name, meshes, mode, nc, prec):
    ntot = sum(int(np.prod(m[0])) for m in meshes)
    M = sphere_random(ntot, seed=21, Ms=8e5)
    Href = MultiLayer(meshes, mode, nc).eval(M)
    tol = 1e-9 if prec == "fp64" else 1e-5
    with _ctx(bm, meshes, mode, nc, prec) as c:
        for i, Mi in enumerate(_split(M, meshes)):
            c.set_m(Mi, i)
        H = np.concatenate([c.demag_field(i) for i in range(len(meshes))])
    assert _relmax(H, Href) < tol


@pytest.mark.parametrize("name,meshes,mode", [("stack3_3d", STACK3, 0), ("stack3_2d_layered", STACK3, 2),
                                              ("wide_irregular", WIDE_IRR, 0)])
def test_ml_hdemag_vs_reference_build(bm, name, meshes, mode):
    if reference() is None:
        pytest.skip("reference CPU build not available")
    ntot = sum(int(np.prod(m[0])) for m in meshes)
    M = sphere_random(ntot, seed=22, Ms=8e5)
    Href = MultiLayer(meshes, mode, which="reference").eval(M)
    with _ctx(bm, meshes, mode, None, "fp64") as c:
        for i, Mi in enumerate(_split(M, meshes)):
            c.set_m(Mi, i)
        H = np.concatenate([c.demag_field(i) for i in range(len(meshes))])
    assert _relmax(H, Href) < 2e-9


def _stack_run(bm, prec, evaluation, steps, mode=0, dt=5e-14, ctrl=None, start="sphere", es=0):
    """The three-mesh stack with exchange, anisotropy on the top mesh and an applied field;
    start "sphere" (random directions) or "tilted" (+z with up to 15 degree tilts); es: evaluation
    speedup level (both runs)."""
    descs = []
    for q, (m, Ms) in enumerate(zip(STACK3, MS3)):
        d = dict(n=m[0], h=m[1], Ms=Ms, A=1.5e-11, alpha=0.05, modules=1 | 2 | 16, Ha=(2e4, 0, 0))
        if q == 2:
            d.update(K1=3e5, modules=1 | 2 | 8 | 16)
        descs.append(d)
    gen = sphere_random if start == "sphere" else tilted_z
    Ms0 = [gen(int(np.prod(d["n"])), seed=30 + q, Ms=d["Ms"]) for q, d in enumerate(descs)]
    s = OracleSolver(descs, evaluation=evaluation, dt=dt, **({} if ctrl is None else
                                                            dict(tol=ctrl[0], dT_incr=ctrl[1], dT_min=ctrl[2], dT_max=ctrl[3])))
    s.multilayer([m[2] for m in STACK3], mode=mode)
    if es:
        s.evalspeedup(es)
    for q, M0 in enumerate(Ms0):
        s.set_m(M0, q)
    st_o = s.run(steps)
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    for q, (m, d) in enumerate(zip(STACK3, descs)):
        c.add_mesh(m[0], m[1], m[2])
        c.set_material(q, Ms=d["Ms"], A=d["A"], alpha=d["alpha"], K1=d.get("K1", 0.0), ea=(0, 0, 1))
        c.set_modules(q, d["modules"])
        c.set_field(q, d["Ha"])
    c.multiconvolution(mode)
    if es:
        c.evalspeedup(es)
    c.setode("RK4" if evaluation == 0 else "RKDP54", dt)
    if ctrl:
        c.astepctrl(*ctrl)
    for q, M0 in enumerate(Ms0):
        c.set_m(M0, q)
    st_g = c.run(steps)
    err = max(np.abs(c.get_m(q) - s.get_m(q)).max() / d["Ms"] for q, d in enumerate(descs))
    c.close()
    return err, st_g, st_o


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
@pytest.mark.parametrize("mode", [0, 2])
def test_ml_rk4_stack(bm, prec, tol, mode):
    err, st_g, st_o = _stack_run(bm, prec, 0, 20, mode=mode)
    assert st_g["accepted"] == st_o["accepted"] == 20
    assert err < tol


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_ml_rkdp54_stack(bm, prec, tol):
    err, st_g, st_o = _stack_run(bm, prec, 1, 15, dt=1e-13, ctrl=(1e-5, 2.0, 1e-15, 3e-12), start="tilted")
    if prec == "fp64":
        assert st_g["accepted"] == st_o["accepted"] and st_g["rejected"] == st_o["rejected"]
        assert abs(st_g["time"] - st_o["time"]) <= 1e-9 * st_o["time"]
    assert err < tol


# ---------------------------------------------------------------- evaluation speedup, per layer
@pytest.mark.parametrize("level", [1, 2, 3, 6])
@pytest.mark.parametrize("mode", [0, 2])
def test_ml_evalspeedup_rk4_stack(bm, level, mode):
    """The speedup on the multilayered convolution (SDemagCUDA::UpdateField, Boris/SDemagCUDA.cpp:
    587-930): each layer's common-grid field minus its self term saved and extrapolated; FP64 follows
    the oracle to 1e-9 of Ms (that the oracle's speedup changes the trajectory is checked on the CPU,
    test_oracle_evalspeedup.py)."""
    err, st_g, st_o = _stack_run(bm, "fp64", 0, 20, mode=mode, es=level)
    assert st_g["accepted"] == st_o["accepted"] == 20
    assert err < 1e-9


@pytest.mark.parametrize("level", [1, 3])
def test_ml_evalspeedup_rkdp54_stack(bm, level):
    """RKDP54 with the speedup on the multilayered convolution, the reference's rule decided on the
    device per evaluation: accepted / rejected counts, time and m follow the oracle (FP64)."""
    err, st_g, st_o = _stack_run(bm, "fp64", 1, 15, dt=1e-13, ctrl=(1e-5, 2.0, 1e-15, 3e-12), start="tilted", es=level)
    assert st_g["accepted"] == st_o["accepted"] and st_g["rejected"] == st_o["rejected"]
    assert abs(st_g["time"] - st_o["time"]) <= 1e-9 * st_o["time"]
    assert err < 1e-8


def test_ml_evalspeedup_mixed(bm):
    err, st_g, _ = _stack_run(bm, "mixed", 0, 20, es=3)
    assert st_g["accepted"] == 20
    assert err < 1e-4
