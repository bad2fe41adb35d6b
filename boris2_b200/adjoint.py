"""Gradients of a final-magnetisation loss through RK4 micromagnetics, for torch.

``rk4_loss(Ms_map, K1_map, Ha, problem)`` returns the loss (1/n) sum_i |m_i(T) - target_i|^2 after
``problem.steps`` RK4 steps from m0, as a torch scalar whose backward gives the exact discrete
gradients with respect to the per-cell Ms map, the per-cell K1 map (uniaxial anisotropy) and the
applied-field samples. The forward and backward both run on the GPU through the C ABI
(``bm_adjoint_rk4``: checkpoints every ``problem.ckpt_every`` steps, recompute per segment); the
gradients are computed together with the loss and handed to autograd. Tensors may live on any
device; the library copies them through host memory.
"""
from dataclasses import dataclass, field
from typing import Tuple

import numpy as np
import torch

import boris2_b200 as bm


@dataclass
class Problem:
    """One film: mesh, fixed material, initial unit vectors m0 (M0 = Ms m0), target unit vectors."""
    n: Tuple[int, int, int]
    h: Tuple[float, float, float]
    m0: np.ndarray
    target: np.ndarray
    steps: int
    dt: float
    ckpt_every: int = 100
    A: float = 1.3e-11
    alpha: float = 0.02
    ea: Tuple[float, float, float] = (0.0, 0.0, 1.0)
    t_span: float = 0.0
    modules: int = bm.DEMAG | bm.EXCH | bm.ANIUNI | bm.ZEEMAN
    precision: int = bm.MIXED
    device: int = 0
    last: dict = field(default_factory=dict)


def _run(p, Ms, K1, Ha):
    c = bm.Context(device=p.device, precision=p.precision)
    try:
        c.add_mesh(p.n, p.h)
        c.set_material(0, Ms=float(np.mean(Ms)), A=p.A, alpha=p.alpha, ea=p.ea)
        c.set_material_maps(0, Ms_map=Ms, K1_map=K1)
        c.set_modules(0, p.modules)
        c.set_field(0, Ha, p.t_span)
        c.setode("RK4", p.dt)
        c.set_m(np.asarray(p.m0, dtype=np.float64).reshape(-1, 3) * np.asarray(Ms)[:, None])
        loss, dMs, dK1, dHa, tm = c.adjoint_rk4(p.target, p.steps, p.ckpt_every, True, nHa=len(Ha))
        p.last = {"m_final": c.get_m(0) / np.asarray(Ms)[:, None], "times_ms": tm}
    finally:
        c.close()
    return loss, dMs, dK1, dHa


class RK4Loss(torch.autograd.Function):
    """loss(Ms_map, K1_map, Ha) for a fixed Problem, with its exact discrete gradient."""

    @staticmethod
    def forward(ctx, Ms_map, K1_map, Ha, problem):
        Ms = Ms_map.detach().double().cpu().numpy().reshape(-1)
        K1 = K1_map.detach().double().cpu().numpy().reshape(-1)
        H = Ha.detach().double().cpu().numpy().reshape(-1, 3)
        loss, dMs, dK1, dHa = _run(problem, Ms, K1, H)
        ctx.save_for_backward(torch.as_tensor(dMs, dtype=Ms_map.dtype, device=Ms_map.device).reshape(Ms_map.shape),
                              torch.as_tensor(dK1, dtype=K1_map.dtype, device=K1_map.device).reshape(K1_map.shape),
                              torch.as_tensor(dHa, dtype=Ha.dtype, device=Ha.device).reshape(Ha.shape))
        return torch.tensor(loss, dtype=Ms_map.dtype, device=Ms_map.device)

    @staticmethod
    def backward(ctx, g):
        dMs, dK1, dHa = ctx.saved_tensors
        return g * dMs, g * dK1, g * dHa, None


def rk4_loss(Ms_map, K1_map, Ha, problem):
    return RK4Loss.apply(Ms_map, K1_map, Ha, problem)
