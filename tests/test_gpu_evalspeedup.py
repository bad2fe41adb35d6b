"""Evaluation speedup on cuda:0 against the oracle's restatement of the reference's
(DemagCUDA::UpdateField, Boris/DemagCUDA.cpp:106-470): levels 1 (step) .. 6 (quintic), 2D and 3D
meshes, under RK4 and under RKDP54 (the reference's rule decided on the device per evaluation,
including the repeated first evaluation after a rejected step). FP64 <= 1e-9 of Ms after the run
(RKDP54: also the same accepted and rejected counts); mixed precision <= 1e-4. The runs must also
differ from the run without the speedup by more than those tolerances, so the extrapolating path is
the one measured."""
import numpy as np
import pytest

from oracle_libs import OracleSolver, sphere_random
from test_gpu_step import _make

pytestmark = pytest.mark.gpu

FILM = dict(n=(32, 16, 1), h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16, Ha=(1e3, 0, 0))
BOX = dict(n=(16, 12, 4), h=(3e-9, 3e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(0, 2e3, 0))


def _oracle(mesh, M, steps, dt, level, evaluation=0, ctrl=None):
    kw = {} if ctrl is None else dict(tol=ctrl[0], dT_incr=ctrl[1], dT_min=ctrl[2], dT_max=ctrl[3])
    s = OracleSolver([mesh], evaluation=evaluation, dt=dt, **kw)
    s.evalspeedup(level)
    s.set_m(M)
    st = s.run(steps)
    m = s.get_m()
    s.close()
    return (m, st) if evaluation else m


@pytest.mark.parametrize("mesh", [FILM, BOX], ids=["film2d", "box3d"])
@pytest.mark.parametrize("level", [1, 2, 3, 4, 5, 6])
def test_evalspeedup_fp64(bm, mesh, level):
    N = int(np.prod(mesh["n"]))
    M = sphere_random(N, seed=77 + level, Ms=8e5)
    steps, dt = 20, 1e-13
    mref = _oracle(mesh, M, steps, dt, level)
    mplain = _oracle(mesh, M, steps, dt, 0)
    c = _make(bm, "fp64", mesh, M, "RK4", dt)
    c.evalspeedup(level)
    st = c.run(steps)
    m = c.get_m()
    c.close()
    assert st["accepted"] == steps
    err = np.abs(m - mref).max() / 8e5
    assert err < 1e-9, err
    assert np.abs(mref - mplain).max() / 8e5 > 1e-8   # the speedup changes the trajectory


def test_evalspeedup_mixed_and_restart(bm):
    """Mixed precision follows the FP64 oracle; setting M drops the saved fields (the next steps
    compute in full again), as a restart of the reference does."""
    mesh = FILM
    N = int(np.prod(mesh["n"]))
    M = sphere_random(N, seed=5, Ms=8e5)
    dt = 5e-14
    c = _make(bm, "mixed", mesh, M, "RK4", dt)
    c.evalspeedup(3)
    c.run(12)
    m = c.get_m()
    assert np.abs(m - _oracle(mesh, M, 12, dt, 3)).max() / 8e5 < 1e-4
    # restart from M2: identical to a fresh run from M2
    M2 = sphere_random(N, seed=6, Ms=8e5)
    c.set_m(M2)
    c.run(8)
    m2 = c.get_m()
    c.close()
    assert np.abs(m2 - _oracle(mesh, M2, 8, dt, 3)).max() / 8e5 < 1e-4


def test_evalspeedup_refusals(bm):
    mesh = FILM
    M = sphere_random(int(np.prod(mesh["n"])), seed=3, Ms=8e5)
    c = _make(bm, "fp64", mesh, M, "RKDP54", 1e-13)
    with pytest.raises(bm.BorisError):
        c.evalspeedup(7)
    c.evalspeedup(0)
    c.run(2)                                        # the context stays usable
    c.close()


CTRL = (1e-5, 2.0, 1e-15, 3e-12)


@pytest.mark.parametrize("mesh", [FILM, BOX], ids=["film2d", "box3d"])
@pytest.mark.parametrize("level", [1, 2, 3, 4, 5, 6])
def test_evalspeedup_rkdp54_fp64(bm, mesh, level):
    """RKDP54 with the speedup: every accepted and rejected step, the simulated time and m follow the
    oracle."""
    N = int(np.prod(mesh["n"]))
    M = sphere_random(N, seed=31 + level, Ms=8e5)
    steps, dt = 25, 2e-14
    (mref, sref) = _oracle(mesh, M, steps, dt, level, evaluation=1, ctrl=CTRL)
    (mplain, _) = _oracle(mesh, M, steps, dt, 0, evaluation=1, ctrl=CTRL)
    c = _make(bm, "fp64", mesh, M, "RKDP54", dt, CTRL)
    c.evalspeedup(level)
    st = c.run(steps)
    m = c.get_m()
    c.close()
    assert st["accepted"] == steps and st["rejected"] == sref["rejected"]
    assert abs(st["time"] - sref["time"]) <= 1e-9 * sref["time"]
    err = np.abs(m - mref).max() / 8e5
    assert err < 1e-9, err
    assert np.abs(mref - mplain).max() / 8e5 > 1e-8


@pytest.mark.parametrize("level", [2, 3, 6])
def test_evalspeedup_rkdp54_rejections(bm, level):
    """A large first step forces rejections: the repeated first evaluation extrapolates, with the field
    saved at the rejected step's end kept in its slot, exactly as in the oracle (FP64 counts, time and
    m). The mixed-precision path completes with a finite state (from this random start with a tight
    tolerance FP32 takes its own accept / reject decisions, so it is not compared cell by cell)."""
    mesh = dict(n=(16, 16, 1), h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16, Ha=(1e4, 0, 0))
    M = sphere_random(256, seed=21, Ms=8e5)
    ctrl = (1e-6, 2.0, 1e-16, 1e-11)
    (mref, sref) = _oracle(mesh, M, 30, 2e-12, level, evaluation=1, ctrl=ctrl)
    assert sref["rejected"] > 0
    for prec, tol in (("fp64", 1e-8), ("mixed", 1e-4)):
        c = _make(bm, prec, mesh, M, "RKDP54", 2e-12, ctrl)
        c.evalspeedup(level)
        st = c.run(30)
        m = c.get_m()
        c.close()
        assert st["accepted"] == 30 and np.isfinite(m).all()
        if prec == "fp64":
            assert st["rejected"] == sref["rejected"]
            assert abs(st["time"] - sref["time"]) <= 1e-9 * sref["time"]
            assert np.abs(m - mref).max() / 8e5 < tol


def test_evalspeedup_rkdp54_batched(bm):
    """Batched uneven meshes under RKDP54 with quadratic extrapolation: the speedup kernels cover every
    mesh in one launch and the run follows the oracle (FP64, 1e-9 of each mesh's Ms)."""
    from test_gpu_batch import _descs, _ctx, _init
    descs = _descs(modules=1 | 2 | 16)
    M0 = _init(descs, "sphere")
    s = OracleSolver(descs, evaluation=1, dt=2e-14, tol=CTRL[0], dT_incr=CTRL[1], dT_min=CTRL[2], dT_max=CTRL[3])
    s.evalspeedup(3)
    for q, M in enumerate(M0):
        s.set_m(M, q)
    sref = s.run(10)
    c = _ctx(bm, "fp64", True, descs, "RKDP54", 2e-14)
    c.astepctrl(*CTRL)
    c.evalspeedup(3)
    for q, M in enumerate(M0):
        c.set_m(M, q)
    st = c.run(10)
    assert st["rejected"] == sref["rejected"]
    err = max(np.abs(c.get_m(q) - s.get_m(q)).max() / d["Ms"] for q, d in enumerate(descs))
    c.close()
    s.close()
    assert err < 1e-9, err


def test_evalspeedup_batched_uneven_systems(bm):
    """Batched uneven meshes (2D and 3D, 3 * 2^k FFT lengths) with quadratic extrapolation follow the
    oracle (FP64, 1e-9 of each mesh's Ms) and the same meshes run one launch per mesh."""
    from test_gpu_batch import _descs, _ctx, _init
    descs = _descs(modules=1 | 2 | 16)
    M0 = _init(descs, "sphere")
    s = OracleSolver(descs, evaluation=0, dt=5e-14)
    s.evalspeedup(3)
    for q, M in enumerate(M0):
        s.set_m(M, q)
    s.run(12)
    out = []
    for batched in (True, False):
        c = _ctx(bm, "fp64", batched, descs, "RK4", 5e-14)
        c.evalspeedup(3)
        for q, M in enumerate(M0):
            c.set_m(M, q)
        assert c.run(12)["accepted"] == 12
        out.append([c.get_m(q) for q in range(len(descs))])
        c.close()
    err = max(np.abs(a - s.get_m(q)).max() / d["Ms"] for q, (a, d) in enumerate(zip(out[0], descs)))
    assert err < 1e-9, err
    same = max(np.abs(a - b).max() / d["Ms"] for a, b, d in zip(out[0], out[1], descs))
    assert same < 1e-11, same



@pytest.mark.parametrize("mesh", [FILM, BOX], ids=["film2d", "box3d"])
def test_evalspeedup_self_term_in_metres(bm, mesh):
    """bm_set_evalspeedup_self(ctx, 1): the self term as the reference computes it, on the cellsize in
    metres; FP64 follows the oracle with the same choice to 1e-9 of Ms (RK4, quadratic)."""
    N = int(np.prod(mesh["n"]))
    M = sphere_random(N, seed=91, Ms=8e5)
    s = OracleSolver([mesh], evaluation=0, dt=1e-13)
    s.evalspeedup(3, metres=True)
    s.set_m(M)
    s.run(20)
    mref = s.get_m()
    s.close()
    c = _make(bm, "fp64", mesh, M, "RK4", 1e-13)
    c.evalspeedup_self(True)
    c.evalspeedup(3)
    c.run(20)
    m = c.get_m()
    c.close()
    assert np.abs(m - mref).max() / 8e5 < 1e-9


@pytest.mark.parametrize("evaluation", ["RK4", "RKDP54"])
def test_evalspeedup_folded_into_stage_kernel(bm, monkeypatch, evaluation):
    """BM_ES_FOLD=1: the extrapolated spectrum formed by the stage kernel instead of k_es_extrap (an
    opt-in variant, slower on the headline film); FP64 follows the oracle to 1e-9 (RK4) / 1e-8 with the
    same counts (RKDP54)."""
    monkeypatch.setenv("BM_ES_FOLD", "1")
    mesh = BOX
    N = int(np.prod(mesh["n"]))
    M = sphere_random(N, seed=93, Ms=8e5)
    if evaluation == "RK4":
        mref = _oracle(mesh, M, 20, 1e-13, 3)
        c = _make(bm, "fp64", mesh, M, "RK4", 1e-13)
        c.evalspeedup(3)
        c.run(20)
        assert np.abs(c.get_m() - mref).max() / 8e5 < 1e-9
    else:
        mref, sr = _oracle(mesh, M, 20, 1e-14, 3, evaluation=1, ctrl=CTRL)
        c = _make(bm, "fp64", mesh, M, "RKDP54", 1e-14, CTRL)
        c.evalspeedup(3)
        st = c.run(20)
        assert st["rejected"] == sr["rejected"]
        assert np.abs(c.get_m() - mref).max() / 8e5 < 1e-8
    c.close()
