"""GPU parity of batched execution (many uneven meshes per launch, C ABI on cuda:0) against the
oracle and against per-mesh launches.

Tolerances: FP64 <= 1e-9 max |m - m_ref| / Ms after the run, mixed precision <= 1e-4; the
batched and per-mesh FP64 runs of the library agree to 1e-11 (the batched passes use the
generic-length FFT kernels, the per-mesh passes the register ones)."""
import numpy as np
import pytest

from oracle_libs import OracleSolver, sphere_random, tilted_z

pytestmark = pytest.mark.gpu

# uneven systems: 2D and 3D, lengths with 3 * 2^k FFT sizes, 4 x 4 x 3 nm cells
SYSTEMS = [((48, 32, 1), 8e5, 1.3e-11, 0.3), ((64, 24, 2), 1.2e6, 1.8e-11, 0.05), ((32, 96, 1), 5e5, 0.9e-11, 0.5),
           ((40, 16, 4), 1.0e6, 1.5e-11, 0.1), ((20, 20, 1), 7e5, 1.1e-11, 0.02), ((96, 64, 2), 1.4e6, 2.0e-11, 0.2)]
H = (4e-9, 4e-9, 3e-9)


def _descs(modules=1 | 2):
    return [dict(n=n, h=H, Ms=Ms, A=A, alpha=al, modules=modules) for n, Ms, A, al in SYSTEMS]


def _ctx(bm, prec, batched, descs, evaluation, dt, ctrl=None):
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    for q, d in enumerate(descs):
        c.add_mesh(d["n"], d["h"], (0.0, 0.0, 1e-6 * q))
        c.set_material(q, Ms=d["Ms"], A=d["A"], alpha=d["alpha"])
        c.set_modules(q, d["modules"])
    c.set_batched(batched)
    c.setode(evaluation, dt)
    if ctrl:
        c.astepctrl(*ctrl)
    return c


def _init(descs, start):
    gen = sphere_random if start == "sphere" else tilted_z
    return [gen(int(np.prod(d["n"])), seed=40 + q, Ms=d["Ms"]) for q, d in enumerate(descs)]


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_batched_rk4_matches_oracle(bm, prec, tol):
    descs = _descs()
    M0 = _init(descs, "sphere")
    s = OracleSolver(descs, evaluation=0, dt=5e-14)
    for q, M in enumerate(M0):
        s.set_m(M, q)
    s.run(20)
    c = _ctx(bm, prec, True, descs, "RK4", 5e-14)
    for q, M in enumerate(M0):
        c.set_m(M, q)
    st = c.run(20)
    assert st["accepted"] == 20
    err = max(np.abs(c.get_m(q) - s.get_m(q)).max() / d["Ms"] for q, d in enumerate(descs))
    # per RK stage: one launch per transform length with a register kernel plus one for the other
    # lengths: 2D y pass (Ny 64; 192 and 48 generic), y forward and y inverse (Ny 48 generic, 32,
    # 128), z pass (Nz 4, 8), stage (LX 24, 32, 48, 64, 96) -> 2 + 3 + 2 + 3 + 5 launches
    assert c.kernels_per_step() == 4 * 15
    c.close()
    assert err < tol


def test_batched_equals_per_mesh(bm):
    descs = _descs()
    M0 = _init(descs, "sphere")
    out = []
    for batched in (False, True):
        c = _ctx(bm, "fp64", batched, descs, "RK4", 5e-14)
        for q, M in enumerate(M0):
            c.set_m(M, q)
        c.run(10)
        out.append([c.get_m(q) for q in range(len(descs))])
        c.close()
    err = max(np.abs(a - b).max() / d["Ms"] for a, b, d in zip(out[0], out[1], descs))
    assert err < 1e-11


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-8), ("mixed", 1e-4)])
def test_batched_rkdp54_matches_oracle(bm, prec, tol):
    """The error norm is the maximum over every mesh of the batch and one controller steps them all."""
    descs = _descs(1 | 2 | 16)
    M0 = _init(descs, "tilted")
    ctrl = (1e-5, 2.0, 1e-15, 3e-12)
    s = OracleSolver(descs, evaluation=1, dt=1e-13, tol=ctrl[0], dT_incr=ctrl[1], dT_min=ctrl[2], dT_max=ctrl[3])
    for q, M in enumerate(M0):
        s.set_m(M, q)
    so = s.run(12)
    c = _ctx(bm, prec, True, descs, "RKDP54", 1e-13, ctrl)
    for q, M in enumerate(M0):
        c.set_m(M, q)
    sg = c.run(12)
    err = max(np.abs(c.get_m(q) - s.get_m(q)).max() / d["Ms"] for q, d in enumerate(descs))
    c.close()
    if prec == "fp64":
        assert sg["accepted"] == so["accepted"] and sg["rejected"] == so["rejected"]
        assert abs(sg["time"] - so["time"]) <= 1e-9 * so["time"]
    assert err < tol


def test_batched_wide_systems_equal_per_mesh(bm):
    """Systems 256 and 512 cells wide (the batched radix-16 stage kernel) and 384 wide (radix 4/3):
    batched and per-mesh FP64 runs agree to 1e-11 of Ms."""
    descs = [dict(n=n, h=H, Ms=Ms, A=1.3e-11, alpha=0.2, modules=1 | 2)
             for n, Ms in [((256, 24, 1), 8e5), ((512, 16, 2), 1.1e6), ((384, 12, 2), 6e5)]]
    M0 = _init(descs, "sphere")
    out = []
    for batched in (False, True):
        c = _ctx(bm, "fp64", batched, descs, "RK4", 5e-14)
        for q, M in enumerate(M0):
            c.set_m(M, q)
        c.run(6)
        out.append([c.get_m(q) for q in range(len(descs))])
        c.close()
    err = max(np.abs(a - b).max() / d["Ms"] for a, b, d in zip(out[0], out[1], descs))
    assert err < 1e-11
