"""Evaluation speedup of RK4 on cuda:0 against the oracle's restatement of the reference's
(DemagCUDA::UpdateField, Boris/DemagCUDA.cpp:106-470): levels 1 (step) .. 6 (quintic), 2D and 3D
meshes. FP64 <= 1e-9 of Ms after the run; mixed precision <= 1e-4. The runs must also differ from
the run without the speedup by more than those tolerances, so the extrapolating path is the one
measured."""
import numpy as np
import pytest

from oracle_libs import OracleSolver, sphere_random
from test_gpu_step import _make

pytestmark = pytest.mark.gpu

FILM = dict(n=(32, 16, 1), h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16, Ha=(1e3, 0, 0))
BOX = dict(n=(16, 12, 4), h=(3e-9, 3e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.3, modules=1 | 2 | 16, Ha=(0, 2e3, 0))


def _oracle(mesh, M, steps, dt, level):
    s = OracleSolver([mesh], evaluation=0, dt=dt)
    s.evalspeedup(level)
    s.set_m(M)
    s.run(steps)
    return s.get_m()


@pytest.mark.parametrize("mesh", [FILM, BOX], ids=["film2d", "box3d"])
@pytest.mark.parametrize("level", [1, 2, 3, 4, 6])
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
    c.evalspeedup(3)
    with pytest.raises(bm.BorisError):
        c.run(2)                                    # RKDP54 with the speedup is refused
    c.evalspeedup(0)
    c.run(2)                                        # and the context stays usable
    c.close()


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

