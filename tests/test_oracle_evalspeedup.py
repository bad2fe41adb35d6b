"""CPU checks of the evaluation-speedup restatement in the oracle and of the host self-demag
coefficients of the library (DemagTFunc::SelfDemag, Boris/DemagTFunc_Self.cpp:6)."""
import numpy as np
import pytest

from oracle_libs import OracleSolver, sphere_random, reference, dp

FILM = dict(n=(16, 8, 1), h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16, Ha=(1e3, 0, 0))


def _run(level, steps=12, dt=5e-14, seed=4):
    M = sphere_random(16 * 8, seed=seed, Ms=8e5)
    s = OracleSolver([FILM], evaluation=0, dt=dt)
    s.evalspeedup(level)
    s.set_m(M)
    s.run(steps)
    return s.get_m()


def test_level0_is_plain():
    M = sphere_random(16 * 8, seed=4, Ms=8e5)
    s = OracleSolver([FILM], evaluation=0, dt=5e-14)
    s.set_m(M)
    s.run(12)
    assert np.array_equal(_run(0), s.get_m())


def test_higher_levels_approach_plain():
    """Extrapolation error shrinks with the polynomial order on a smooth trajectory."""
    plain = _run(0, steps=30, dt=2e-14)
    errs = [np.abs(_run(k, steps=30, dt=2e-14) - plain).max() / 8e5 for k in (1, 2, 3)]
    assert errs[0] > errs[1] > errs[2] > 0
    assert errs[2] < 1e-4


def test_warmup_steps_are_exact():
    """Until `level` fields are saved every evaluation is computed in full: with level 6 the first
    5 steps equal the plain run bit for bit."""
    assert np.array_equal(_run(6, steps=5), _run(0, steps=5))
    assert not np.array_equal(_run(6, steps=7), _run(0, steps=7))


def _run_dp(level, steps=20, dt=2e-14, ctrl=(1e-5, 2.0, 1e-15, 3e-12), seed=4, Ha=(1e3, 0, 0)):
    M = sphere_random(16 * 8, seed=seed, Ms=8e5)
    s = OracleSolver([dict(FILM, Ha=Ha)], evaluation=1, dt=dt, tol=ctrl[0], dT_incr=ctrl[1], dT_min=ctrl[2],
                     dT_max=ctrl[3])
    s.evalspeedup(level)
    s.set_m(M)
    st = s.run(steps)
    m = s.get_m()
    s.close()
    return m, st


def test_rkdp54_levels_approach_plain():
    """RKDP54 with the reference's rule (save while fewer than `level` are saved and at the first
    evaluation after a completed step, extrapolate otherwise), at a fixed step (dT_min = dT_max) so
    every run ends at the same time: the extrapolation error shrinks with the polynomial order up to
    quadratic and stays small beyond (measured 8e-5, 6e-7, 1e-8, 1e-8, 2e-8, 8e-8 of Ms for levels 1..6)."""
    ctrl = (1e-5, 2.0, 2e-14, 2e-14)
    plain, sp = _run_dp(0, ctrl=ctrl, steps=30)
    errs = [np.abs(_run_dp(k, ctrl=ctrl, steps=30)[0] - plain).max() / 8e5 for k in (1, 2, 3, 4, 5, 6)]
    assert errs[0] > errs[1] > errs[2] > 0
    assert max(errs[2:]) < 1e-6


def test_rkdp54_rejections_stay_finite():
    """With rejections (a large first step and a tight tolerance) the repeated first evaluation
    extrapolates from fields that include one saved at the rejected step's end; the run completes with
    finite m and rejections counted."""
    for level in (1, 2, 3, 6):
        m, st = _run_dp(level, steps=30, dt=2e-12, ctrl=(1e-6, 2.0, 1e-16, 1e-11), Ha=(1e4, 0, 0))
        assert st["rejected"] > 0 and st["accepted"] == 30
        assert np.isfinite(m).all()


@pytest.mark.parametrize("h", [(1.0, 1.0, 1.0), (1.0, 1.0, 0.6), (0.5, 1.0, 0.75), (5.0, 5.0, 3.0)])
def test_self_demag_matches_reference(h):
    import boris2_b200
    from boris2_b200 import build
    build.build()
    R = reference()
    if R is None:
        pytest.skip("reference build unavailable")
    want = np.zeros(3)
    R.ref_selfdemag(h[0], h[1], h[2], dp(want))
    got = boris2_b200.self_demag(h)
    assert np.abs(got - want).max() < 1e-13
    # scale invariance: the library normalises the cellsize, so nanometre cells give the same
    assert np.abs(boris2_b200.self_demag(np.asarray(h) * 1e-9) - want).max() < 1e-13


@pytest.mark.parametrize("h", [(5e-9, 5e-9, 3e-9), (2e-9, 2e-9, 2e-9), (4e-9, 3e-9, 1e-9), (1e-6, 1e-6, 5e-7)])
def test_self_demag_metres_matches_reference(h):
    """The reference's speedup self term, SelfDemag on the cellsize in metres with its zero thresholds:
    the library's host function and the oracle's agree with the reference's own build."""
    import boris2_b200
    from boris2_b200 import build
    build.build()
    from oracle_libs import oracle
    R = reference()
    if R is None:
        pytest.skip("reference build unavailable")
    want = np.zeros(3)
    R.ref_selfdemag(h[0], h[1], h[2], dp(want))
    got = boris2_b200.self_demag(h, metres=True)
    orc = np.zeros(3)
    oracle().orc_selfdemag_metres(h[0], h[1], h[2], dp(orc))
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    assert np.abs(orc - want).max() <= 1e-13 * np.abs(want).max()


def test_self_demag_metres_deviates_on_nanometre_cells():
    """The documented difference: on 5 x 5 x 3 nm cells the reference's thresholds drop terms, giving
    (-0.232, -0.232, -0.535) instead of the tensor's (-0.274, -0.274, -0.452); micrometre cells agree."""
    import boris2_b200
    m = boris2_b200.self_demag((5e-9, 5e-9, 3e-9), metres=True)
    n = boris2_b200.self_demag((5e-9, 5e-9, 3e-9))
    assert np.allclose(m, (-0.232, -0.232, -0.535), atol=2e-3)
    assert np.allclose(n, (-0.274, -0.274, -0.452), atol=2e-3)
    assert np.abs(boris2_b200.self_demag((5e-6, 5e-6, 3e-6), metres=True) - n).max() < 1e-12


def test_metres_self_term_trajectory_difference():
    """Size of the trajectory difference between the two self-term choices (RK4, quadratic speedup,
    12 steps of the film): both are consistent splittings of the same field, so they differ only by the
    extrapolation error of S M; measured 7e-8 of Ms, well under the 1e-4 mixed tolerance."""
    M = sphere_random(16 * 8, seed=4, Ms=8e5)
    out = []
    for metres in (False, True):
        s = OracleSolver([FILM], evaluation=0, dt=5e-14)
        s.evalspeedup(3, metres=metres)
        s.set_m(M)
        s.run(12)
        out.append(s.get_m() / 8e5)
        s.close()
    d = np.abs(out[0] - out[1]).max()
    assert 1e-12 < d < 1e-4


# ---------------------------------------------------------------- multilayered convolution
ML_MESHES = [dict(n=(24, 16, 1), h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(1e3, 0, 0)),
             dict(n=(16, 16, 1), h=(5e-9, 4e-9, 3e-9), Ms=1.1e6, A=1.5e-11, alpha=0.1, modules=1 | 2 | 16, Ha=(0, 1e3, 0))]
ML_ORIGINS = [(0.0, 0.0, 0.0), (10e-9, 0.0, 6e-9)]


def _run_ml(level, evaluation=0, steps=12, dt=5e-14, meshes=ML_MESHES, origins=ML_ORIGINS, mode=1):
    # RKDP54 at a fixed step (dT_min = dT_max), so every run ends at the same time
    kw = dict(tol=1e-5, dT_incr=2.0, dT_min=dt, dT_max=dt) if evaluation else {}
    s = OracleSolver(meshes, evaluation=evaluation, dt=dt, **kw)
    s.multilayer(origins, mode=mode)
    s.evalspeedup(level)
    for q, d in enumerate(meshes):
        s.set_m(sphere_random(int(np.prod(d["n"])), seed=30 + q, Ms=d["Ms"]), q)
    st = s.run(steps)
    out = [s.get_m(q) / d["Ms"] for q, d in enumerate(meshes)]
    s.close()
    return out, st


def test_multilayer_one_direct_layer_equals_mesh_speedup():
    """One mesh as the only layer of the multilayered convolution (its grid is the common grid): the
    per-layer speedup (SDemagCUDA) follows the per-mesh one (DemagCUDA) with the same self term."""
    mesh = [dict(n=(16, 12, 2), h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(1e3, 0, 0))]
    for level in (1, 3):
        a, _ = _run_ml(level, meshes=mesh, origins=[(0.0, 0.0, 0.0)], mode=0)
        s = OracleSolver(mesh, evaluation=0, dt=5e-14)
        s.evalspeedup(level)
        s.set_m(sphere_random(384, seed=30, Ms=8e5))
        s.run(12)
        b = s.get_m() / 8e5
        s.close()
        assert np.abs(a[0] - b).max() < 1e-12, level


@pytest.mark.parametrize("evaluation", [0, 1])
def test_multilayer_speedup_approaches_plain(evaluation):
    plain, _ = _run_ml(0, evaluation)
    errs = []
    for level in (1, 2, 3):
        m, st = _run_ml(level, evaluation)
        assert st["accepted"] == 12
        errs.append(max(np.abs(x - y).max() for x, y in zip(m, plain)))
    assert errs[0] > 1e-9                      # the extrapolating path is the one run
    assert errs[2] < errs[0] and errs[2] < 1e-4
