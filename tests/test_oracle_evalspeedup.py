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
