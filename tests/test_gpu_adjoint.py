"""GPU parity of the discrete RK4 adjoint (bm_adjoint_rk4, C ABI on cuda:0) against the oracle's
FP64 CPU adjoint (itself checked against central finite differences on the CPU), against central
finite differences of the GPU's own loss, and through the torch.autograd wrapper.

Tolerances: FP64 loss 1e-12 relative, gradients 1e-8 of their largest magnitude; mixed precision
(FP32 stages and adjoint, FP64 accumulation) gradients 2e-3 of their largest magnitude; the
checkpoint interval changes nothing (FP64, 1e-12)."""
import numpy as np
import pytest

from oracle_libs import orc_adjoint

pytestmark = pytest.mark.gpu


def _case(seed=2, n=(16, 12, 1), nHa=4, steps=20, dt=1e-13):
    rng = np.random.default_rng(seed)
    N = int(np.prod(n))
    mesh = dict(n=n, h=(4e-9, 4e-9, 3e-9), Ms_map=8e5 * (1 + 0.1 * rng.normal(size=N)),
                K1_map=rng.uniform(0, 2e5, N), A=1.3e-11, alpha=0.02, Ha=rng.normal(0, 5e3, (nHa, 3)),
                Ha_tspan=steps * dt)
    m0 = rng.normal(size=(N, 3))
    m0 /= np.linalg.norm(m0, axis=1)[:, None]
    tgt = rng.normal(size=(N, 3))
    tgt /= np.linalg.norm(tgt, axis=1)[:, None]
    return mesh, m0, tgt, steps, dt


def _gpu(bm, mesh, m0, tgt, steps, dt, prec, ckpt, modules=1 | 2 | 8 | 16):
    c = bm.Context(precision=bm.FP64 if prec == "fp64" else bm.MIXED)
    c.add_mesh(mesh["n"], mesh["h"])
    c.set_material(0, Ms=8e5, A=mesh["A"], alpha=mesh["alpha"], ea=(0, 0, 1))
    c.set_material_maps(0, Ms_map=mesh["Ms_map"], K1_map=mesh["K1_map"])
    c.set_modules(0, modules)
    if mesh.get("pbc") is not None:
        c.set_pbc(0, mesh["pbc"])
    c.set_field(0, mesh["Ha"], mesh["Ha_tspan"])
    c.setode("RK4", dt)
    c.set_m(m0 * mesh["Ms_map"][:, None])
    out = c.adjoint_rk4(tgt, steps, ckpt, True)
    c.close()
    return out


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("n", [(16, 12, 1), (12, 10, 2)])
def test_adjoint_fp64_matches_oracle(bm, n):
    mesh, m0, tgt, steps, dt = _case(n=n)
    lo, gMs_o, gK_o, gHa_o = orc_adjoint(mesh, m0, tgt, steps, dt)
    lg, gMs, gK, gHa, tm = _gpu(bm, mesh, m0, tgt, steps, dt, "fp64", 5)
    assert abs(lg - lo) <= 1e-12 * abs(lo)
    assert _rel(gMs, gMs_o) < 1e-8
    assert _rel(gK, gK_o) < 1e-8
    assert _rel(gHa, gHa_o) < 1e-8
    assert tm[0] > 0 and tm[1] > 0


def test_adjoint_mixed_matches_oracle(bm):
    mesh, m0, tgt, steps, dt = _case()
    lo, gMs_o, gK_o, gHa_o = orc_adjoint(mesh, m0, tgt, steps, dt)
    lg, gMs, gK, gHa, _ = _gpu(bm, mesh, m0, tgt, steps, dt, "mixed", 10)
    assert abs(lg - lo) <= 1e-4 * abs(lo)
    assert _rel(gMs, gMs_o) < 2e-3
    assert _rel(gK, gK_o) < 2e-3
    assert _rel(gHa, gHa_o) < 2e-3


def test_adjoint_checkpoint_interval_is_transparent(bm):
    mesh, m0, tgt, steps, dt = _case()
    ref = _gpu(bm, mesh, m0, tgt, steps, dt, "fp64", 20)
    for ck in (1, 4, 10):
        out = _gpu(bm, mesh, m0, tgt, steps, dt, "fp64", ck)
        assert abs(out[0] - ref[0]) <= 1e-12 * abs(ref[0])
        for a, b in zip(out[1:4], ref[1:4]):
            assert _rel(a, b) < 1e-12


def test_adjoint_fp64_matches_gpu_central_differences(bm):
    mesh, m0, tgt, steps, dt = _case(seed=5, n=(10, 8, 1))
    _, gMs, gK, gHa, _ = _gpu(bm, mesh, m0, tgt, steps, dt, "fp64", 5)
    i = 17
    e = 1e-4 * mesh["Ms_map"][i]
    a, b = mesh["Ms_map"].copy(), mesh["Ms_map"].copy()
    a[i] += e
    b[i] -= e
    fd = (_gpu(bm, dict(mesh, Ms_map=a), m0, tgt, steps, dt, "fp64", 5)[0] -
          _gpu(bm, dict(mesh, Ms_map=b), m0, tgt, steps, dt, "fp64", 5)[0]) / (2 * e)
    assert abs(gMs[i] - fd) <= 1e-5 * abs(fd)
    H1, H2 = mesh["Ha"].copy(), mesh["Ha"].copy()
    H1[1, 2] += 10.0
    H2[1, 2] -= 10.0
    fd = (_gpu(bm, dict(mesh, Ha=H1), m0, tgt, steps, dt, "fp64", 5)[0] -
          _gpu(bm, dict(mesh, Ha=H2), m0, tgt, steps, dt, "fp64", 5)[0]) / 20.0
    assert abs(gHa[1, 2] - fd) <= 1e-5 * abs(fd)


def test_adjoint_torch_autograd(bm):
    import torch
    from boris2_b200.adjoint import Problem, rk4_loss
    mesh, m0, tgt, steps, dt = _case()
    p = Problem(n=mesh["n"], h=mesh["h"], m0=m0, target=tgt, steps=steps, dt=dt, ckpt_every=5, A=mesh["A"],
                alpha=mesh["alpha"], t_span=mesh["Ha_tspan"], precision=bm.FP64)
    Ms = torch.tensor(mesh["Ms_map"], requires_grad=True)
    K1 = torch.tensor(mesh["K1_map"], requires_grad=True)
    Ha = torch.tensor(mesh["Ha"], requires_grad=True)
    loss = rk4_loss(Ms, K1, Ha, p)
    (2.0 * loss).backward()
    lo, gMs_o, gK_o, gHa_o = orc_adjoint(mesh, m0, tgt, steps, dt)
    assert abs(loss.item() - lo) <= 1e-12 * abs(lo)
    assert _rel(Ms.grad.numpy(), 2.0 * gMs_o) < 1e-8
    assert _rel(K1.grad.numpy(), 2.0 * gK_o) < 1e-8
    assert _rel(Ha.grad.numpy(), 2.0 * gHa_o) < 1e-8
