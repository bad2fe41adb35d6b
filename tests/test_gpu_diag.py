"""The torque and dm/dt diagnostics on cuda:0 (bm_get_mxh / bm_get_dmdt through the C ABI, the
reference's Get_mxh / Get_dmdt: Boris/DiffEq_CommonBase_Get.cpp:7,19 with the reductions of
Boris/DiffEqFM_EvalsLLGCUDA.cu:416-640 and Boris/DiffEqFM_EvalsCUDA_RKDP54.cu:15-53,188-232) against
the oracle's restatement: RK4 and RKDP54 (adaptive in FP64, fixed-step in mixed precision), FP64 to
1e-9 and mixed precision to 1e-4 relative; one mesh, several meshes with per-mesh and batched
launches, a mesh with grel = 0 left out; the request semantics (0 before any request, a value one
step behind the call that asked for it, one request serving one step)."""
import numpy as np
import pytest

from oracle_libs import OracleSolver, tilted_z

pytestmark = pytest.mark.gpu

H = (3e-9, 3e-9, 3e-9)
MESHES = [dict(n=(24, 16, 3), h=H, Ms=8e5, A=1.3e-11, D=1e-3, alpha=0.3, K1=2e5, modules=1 | 4 | 8 | 16,
               Ha=(1e3, 2e3, 0)),
          dict(n=(32, 12, 1), h=H, Ms=1.1e6, A=1.5e-11, alpha=0.1, modules=1 | 2 | 16, Ha=(5e3, 0, 0)),
          dict(n=(16, 16, 4), h=H, Ms=6e5, A=1.0e-11, alpha=0.5, modules=1 | 2, grel=0.0)]
EVALS = {"RK4": 0, "RKDP54": 1}


def _pair(bm, prec, meshes, evaluation, batched=False):
    dt = 2e-14
    fixed = evaluation == "RKDP54" and prec == "mixed"
    ctrl = (1e-5, 2.0, dt, dt) if fixed else (1e-5, 2.0, 1e-15, 3e-12)
    kw = dict(tol=ctrl[0], dT_incr=ctrl[1], dT_min=ctrl[2], dT_max=ctrl[3]) if evaluation == "RKDP54" else {}
    s = OracleSolver(meshes, evaluation=EVALS[evaluation], dt=dt, **kw)
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    for q, d in enumerate(meshes):
        c.add_mesh(d["n"], d["h"], (0.0, 0.0, 1e-6 * q))
        c.set_material(q, Ms=d["Ms"], A=d["A"], alpha=d["alpha"], grel=d.get("grel", 1.0), K1=d.get("K1", 0.0),
                       D=d.get("D", 0.0))
        c.set_modules(q, d["modules"])
        c.set_field(q, d.get("Ha", (0, 0, 0)))
    c.set_batched(batched)
    c.setode(evaluation, dt)
    if evaluation == "RKDP54":
        c.astepctrl(*ctrl)
    for q, d in enumerate(meshes):
        M = tilted_z(int(np.prod(d["n"])), seed=70 + q, Ms=d["Ms"])
        s.set_m(M, q)
        c.set_m(M, q)
    return s, c


def _check(s, c, tol):
    a, b = s.get_mxh(), c.get_mxh()
    assert a > 0 and abs(b / a - 1) < tol, (a, b)
    a, b = s.get_dmdt(), c.get_dmdt()
    assert a > 0 and abs(b / a - 1) < tol, (a, b)


@pytest.mark.parametrize("evaluation", ["RK4", "RKDP54"])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_diag_one_mesh(bm, evaluation, prec, tol):
    s, c = _pair(bm, prec, MESHES[:1], evaluation)
    assert c.get_mxh() == 0.0 and c.get_dmdt() == 0.0   # nothing computed yet; both now requested
    s.get_mxh(); s.get_dmdt()
    s.run(1); c.run(1)
    _check(s, c, tol)          # the values of step 1; step 2 is asked
    s.run(3); c.run(3)
    _check(s, c, tol)          # the values of step 2, the first of the three
    s.close(); c.close()


@pytest.mark.parametrize("batched", [False, True])
@pytest.mark.parametrize("evaluation", ["RK4", "RKDP54"])
def test_diag_meshes(bm, evaluation, batched):
    s, c = _pair(bm, "fp64", MESHES, evaluation, batched)
    c.get_mxh(); c.get_dmdt(); s.get_mxh(); s.get_dmdt()
    s.run(2); c.run(2)
    _check(s, c, 1e-9)         # maxima over the meshes, the grel = 0 mesh left out
    s.run(1); c.run(1)
    _check(s, c, 1e-9)
    s.close(); c.close()


@pytest.mark.parametrize("evaluation", ["RK4", "RKDP54"])
def test_diag_multilayer_stack(bm, evaluation):
    """The diagnostics over the meshes of a multilayered convolution: Heff carries the demag field the
    transfer brings back from the common grid."""
    from test_gpu_ml import STACK3, MS3
    descs = []
    for q, (m, Ms) in enumerate(zip(STACK3, MS3)):
        d = dict(n=m[0], h=m[1], Ms=Ms, A=1.5e-11, alpha=0.05, modules=1 | 2 | 16, Ha=(2e4, 0, 0))
        if q == 2:
            d.update(K1=3e5, modules=1 | 2 | 8 | 16)
        descs.append(d)
    dt = 5e-14
    ev = EVALS[evaluation]
    kw = dict(tol=1e-5, dT_incr=2.0, dT_min=1e-15, dT_max=3e-12) if ev == 1 else {}
    s = OracleSolver(descs, evaluation=ev, dt=dt, **kw)
    s.multilayer([m[2] for m in STACK3], mode=0)
    c = bm.Context(precision=bm.FP64)
    for q, (m, d) in enumerate(zip(STACK3, descs)):
        c.add_mesh(m[0], m[1], m[2])
        c.set_material(q, Ms=d["Ms"], A=d["A"], alpha=d["alpha"], K1=d.get("K1", 0.0), ea=(0, 0, 1))
        c.set_modules(q, d["modules"])
        c.set_field(q, d["Ha"])
    c.multiconvolution(0)
    c.setode(evaluation, dt)
    if ev == 1:
        c.astepctrl(1e-5, 2.0, 1e-15, 3e-12)
    for q, d in enumerate(descs):
        M = tilted_z(int(np.prod(d["n"])), seed=90 + q, Ms=d["Ms"])
        s.set_m(M, q)
        c.set_m(M, q)
    s.get_mxh(); s.get_dmdt(); c.get_mxh(); c.get_dmdt()
    s.run(2); c.run(2)
    _check(s, c, 1e-9)
    s.close(); c.close()
