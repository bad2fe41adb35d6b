"""Supermesh demag on cuda:0 (bm_set_multiconvolution(BM_ML_SUPERMESH), C ABI) against the oracle's
restatement (pinned to the compiled reference in test_oracle_supermesh.py) and against the reference
build directly.

Tolerances: H_demag FP64 1e-9, mixed 1e-5 relative to max |H_ref|; integration FP64 1e-9 of Ms after
the run (RKDP54 1e-8 with the same accepted / rejected counts), mixed 1e-4."""
import numpy as np
import pytest

import boris2_b200 as bmod
from oracle_libs import SuperMesh, OracleSolver, sphere_random, tilted_z, reference
from test_oracle_supermesh import CASES, _ids

pytestmark = pytest.mark.gpu


def _relmax(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def _ctx(bm, prec, meshes, hr, pbc, modules=1):
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    for q, (n, h, o) in enumerate(meshes):
        c.add_mesh(n, h, o)
        c.set_modules(q, modules)
    c.multiconvolution(bm.ML_SUPERMESH)
    c.supermesh_cellsize(hr)
    c.supermesh_pbc(pbc)
    return c


@pytest.mark.parametrize("case", CASES, ids=_ids)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_supermesh_hdemag(bm, case, prec):
    meshes, hr, pbc = case
    sm = SuperMesh(meshes, hr, pbc, "oracle")
    M = np.concatenate([sphere_random(nc, seed=40 + q, Ms=8e5) for q, nc in enumerate(sm.ncell)])
    Href, _ = sm.eval(M)
    off = np.cumsum([0] + sm.ncell)
    with _ctx(bm, prec, meshes, hr, pbc) as c:
        for q in range(len(meshes)):
            c.set_m(M[off[q]:off[q + 1]], q)
        tol = 1e-9 if prec == "fp64" else 1e-5
        for q in range(len(meshes)):
            H = c.demag_field(q)
            assert _relmax(H, Href[off[q]:off[q + 1]]) < tol * np.abs(Href).max() / np.abs(Href[off[q]:off[q + 1]]).max()
        info = c.supermesh_info()
    io = sm.info()
    assert info["n"] == io["n"]
    assert np.allclose(info["h"], io["h"], rtol=1e-14, atol=0)
    assert np.allclose(info["rect"], io["rect"], rtol=0, atol=1e-20)
    assert info["nonempty"] == io["nonempty"]


@pytest.mark.parametrize("case", CASES[:3], ids=_ids)
def test_supermesh_hdemag_vs_reference_build(bm, case):
    if reference() is None:
        pytest.skip("reference CPU build not available")
    meshes, hr, pbc = case
    sm = SuperMesh(meshes, hr, pbc, "reference")
    M = np.concatenate([sphere_random(nc, seed=90 + q, Ms=8e5) for q, nc in enumerate(sm.ncell)])
    Href, _ = sm.eval(M)
    off = np.cumsum([0] + sm.ncell)
    with _ctx(bm, "fp64", meshes, hr, pbc) as c:
        for q in range(len(meshes)):
            c.set_m(M[off[q]:off[q + 1]], q)
        H = np.concatenate([c.demag_field(q) for q in range(len(meshes))])
    assert _relmax(H, Href) < 1e-9


BILAYER = [dict(n=(24, 16, 1), h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(2e3, 0, 0)),
           dict(n=(16, 16, 2), h=(5e-9, 4e-9, 2e-9), Ms=1.1e6, A=1.5e-11, alpha=0.1, modules=1 | 2 | 16, Ha=(0, 1e3, 0))]
ORIGINS = [(0.0, 0.0, 0.0), (10e-9, 0.0, 5e-9)]


def _gpu_run(bm, prec, evaluation, dt, steps, M, hr, pbc, ctrl=None):
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    for q, d in enumerate(BILAYER):
        c.add_mesh(d["n"], d["h"], ORIGINS[q])
        c.set_material(q, Ms=d["Ms"], A=d["A"], alpha=d["alpha"])
        c.set_modules(q, d["modules"])
        c.set_field(q, d["Ha"])
    c.multiconvolution(bm.ML_SUPERMESH)
    c.supermesh_cellsize(hr)
    c.supermesh_pbc(pbc)
    c.setode(evaluation, dt)
    if ctrl:
        c.astepctrl(*ctrl)
    for q in range(2):
        c.set_m(M[q], q)
    st = c.run(steps)
    out = [c.get_m(q) for q in range(2)]
    c.close()
    return out, st


def _oracle_run(evaluation, dt, steps, M, hr, pbc, ctrl=None):
    kw = {} if ctrl is None else dict(tol=ctrl[0], dT_incr=ctrl[1], dT_min=ctrl[2], dT_max=ctrl[3])
    meshes = [dict(d, pbc=pbc) for d in BILAYER]
    s = OracleSolver(meshes, evaluation=evaluation, dt=dt, **kw)
    s.supermesh(ORIGINS, h_request=hr, pbc=pbc)
    for q in range(2):
        s.set_m(M[q], q)
    st = s.run(steps)
    out = [s.get_m(q) for q in range(2)]
    s.close()
    return out, st


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
@pytest.mark.parametrize("pbc", [(0, 0, 0), (2, 2, 0)])
def test_supermesh_rk4_bilayer(bm, prec, tol, pbc):
    M = [sphere_random(int(np.prod(d["n"])), seed=60 + q, Ms=d["Ms"]) for q, d in enumerate(BILAYER)]
    hr = (4e-9, 4e-9, 1e-9)
    mref, _ = _oracle_run(0, 1e-13, 20, M, hr, pbc)
    m, st = _gpu_run(bm, prec, "RK4", 1e-13, 20, M, hr, pbc)
    assert st["accepted"] == 20
    for q, d in enumerate(BILAYER):
        assert np.abs(m[q] - mref[q]).max() / d["Ms"] < tol


def test_supermesh_rkdp54_bilayer(bm):
    M = [tilted_z(int(np.prod(d["n"])), seed=70 + q, Ms=d["Ms"]) for q, d in enumerate(BILAYER)]
    hr = (4e-9, 4e-9, 1e-9)
    ctrl = (1e-5, 2.0, 1e-15, 3e-12)
    mref, sr = _oracle_run(1, 1e-14, 30, M, hr, (0, 0, 0), ctrl)
    m, st = _gpu_run(bm, "fp64", "RKDP54", 1e-14, 30, M, hr, (0, 0, 0), ctrl)
    assert st["accepted"] == 30
    assert st["rejected"] == sr["rejected"]
    assert abs(st["time"] - sr["time"]) <= 1e-9 * sr["time"]
    for q, d in enumerate(BILAYER):
        assert np.abs(m[q] - mref[q]).max() / d["Ms"] < 1e-8


def test_supermesh_refusals(bm):
    meshes, hr, pbc = CASES[0]
    with _ctx(bm, "mixed", meshes, hr, pbc) as c:
        c.setode("RK4", 1e-13)
        c.evalspeedup(2)
        with pytest.raises(bmod.BorisError) as e:
            c.prepare()
        assert e.value.code == bm.EUNSUPPORTED
    with _ctx(bm, "mixed", meshes, hr, pbc) as c:
        c.set_batched(True)
        with pytest.raises(bmod.BorisError) as e:
            c.prepare()
        assert e.value.code == bm.EUNSUPPORTED
    with _ctx(bm, "mixed", meshes, hr, pbc) as c:
        with pytest.raises(bmod.BorisError) as e:
            c.ml_info()
        assert e.value.code == bm.ESTATE
        with pytest.raises(bmod.BorisError) as e:
            c.supermesh_cellsize((0.0, 1e-9, 1e-9))
        assert e.value.code == bm.EINVAL
