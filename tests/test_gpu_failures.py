"""Failure detection through the C ABI, with failures made on the host (no GPU fault):

  * a NaN planted in M by bm_set_m, and a state driven to overflow by an applied field of 1e300 A/m:
    bm_run returns BM_ENONFINITE; under RKDP54 the step is not accepted even when dT cannot shrink
    (dT_min = dT); the flag stays until a new M is set, after which the context runs normally
  * a device-memory limit below what the meshes need: set-up refuses with BM_ENOMEM before
    allocating, and the same context works once the limit is raised
"""
import numpy as np
import pytest

from oracle_libs import sphere_random

pytestmark = pytest.mark.gpu

N3 = (32, 16, 2)
NC = N3[0] * N3[1] * N3[2]


def _film(bm, prec, evaluation, Ha=(1e3, 0, 0), dt=1e-13, dT_min=1e-15):
    c = bm.Context(precision=prec)
    c.add_mesh(N3, (4e-9, 4e-9, 3e-9))
    c.set_material(0, Ms=8e5, A=1.3e-11, alpha=0.1)
    c.set_modules(0, bm.DEMAG | bm.EXCH | bm.ZEEMAN)
    c.set_field(0, Ha)
    c.setode(evaluation, dt)
    if evaluation == "RKDP54":
        c.astepctrl(1e-5, 2.0, dT_min, 3e-12)
    return c


@pytest.mark.parametrize("evaluation", ["RK4", "RKDP54"])
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_nan_in_m_is_reported_and_cleared(bm, evaluation, prec):
    c = _film(bm, bm.MIXED if prec == "mixed" else bm.FP64, evaluation)
    M = sphere_random(NC, seed=3, Ms=8e5)
    bad = M.copy()
    bad[77, 1] = np.nan
    c.set_m(bad)
    with pytest.raises(bm.BorisError) as e:
        c.run(5)
    assert e.value.code == bm.ENONFINITE
    st = c.stats()
    if evaluation == "RKDP54":
        assert st["accepted"] == 0
    # the flag is sticky: running again is refused until a new M is set
    with pytest.raises(bm.BorisError) as e:
        c.run(1)
    assert e.value.code == bm.ENONFINITE
    c.set_m(M)
    st = c.run(5)
    assert np.isfinite(c.get_m()).all()
    assert st["accepted"] >= 5
    c.close()


@pytest.mark.parametrize("evaluation", ["RK4", "RKDP54"])
def test_overflow_is_not_accepted(bm, evaluation):
    """A field of 1e300 A/m overflows the FP64 LLG rhs: RK4 reports it after the batch; RKDP54 refuses
    the step although dT_min = dT leaves no smaller step to try."""
    c = _film(bm, bm.FP64, evaluation, Ha=(1e300, 0, 0), dt=1e-13, dT_min=1e-13)
    c.set_m(sphere_random(NC, seed=9, Ms=8e5))
    with pytest.raises(bm.BorisError) as e:
        c.run(3)
    assert e.value.code == bm.ENONFINITE
    if evaluation == "RKDP54":
        assert c.stats()["accepted"] == 0
    c.close()


def test_memory_limit_refuses_before_allocating(bm):
    c = bm.Context(precision=bm.MIXED)
    c.add_mesh((512, 512, 16), (2e-9, 2e-9, 2e-9))
    c.set_material(0, Ms=1.1e6, A=1.5e-11, alpha=0.1)
    c.set_modules(0, bm.DEMAG | bm.EXCH)
    c.setode("RK4", 1e-14)
    c.set_memory_limit(64 << 20)
    M = sphere_random(512 * 512 * 16, seed=1, Ms=1.1e6)
    c.set_m(M)
    with pytest.raises(bm.BorisError) as e:
        c.demag_field()
    assert e.value.code == bm.ENOMEM
    assert "memory limit" in str(e.value) and "MB" in str(e.value)
    c.set_memory_limit(0)
    H = c.demag_field()
    assert np.isfinite(H).all() and np.abs(H).max() > 0
    c.close()
