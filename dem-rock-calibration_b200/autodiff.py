"""Elastic macro-properties as a differentiable torch function of the
micro-parameters.

ElasticResponse.apply(p, case) runs the pre-failure uniaxial loading of a
specimen in the sensitivity build (precision 2: FP64 with forward-mode
tangents carried through the same pair and particle kernels, breakage off)
and returns its secant modulus and secant Poisson ratio at the last step;
backward multiplies the incoming gradient by the 2 x 5 Jacobian the run
produced.  The five parameters are, in order, the bond modulus E_bond (GPa),
kn/ks, the bond-radius factor, the particle modulus E (GPa) and the sliding
friction coefficient mu - the order of SENS_NAMES.  A batch p of shape (B, 5) runs as B
samples of one context.

This is the gradient path of a calibration: where the reference's conjugate
gradient (mp_determineconjgradient.cu:84-351, CalculateStepCG in mp_task.h)
spends one extra simulation per parameter on finite differences, one
sensitivity run gives the whole gradient.  The time step is held fixed (the
caller passes it), so the derivatives are those of a fixed-step run.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import SENS_NAMES, Context, Loading
from .workloads import rock_material

PARAMS = ("E_bond", "kn_ks", "bond_radius_factor", "E", "mu")


@dataclass
class ElasticCase:
    """A specimen (positions, radii, loading) and the run: steps at a fixed dt,
    and material values that are not differentiated (rock_material keywords)."""
    xyz: np.ndarray
    radii: np.ndarray
    loading: Loading
    steps: int
    dt: float
    fixed: dict | None = None
    device: int = 0
    deterministic: bool = True     # exact fixed-point force sums: repeatable values and derivatives


def _material(case: ElasticCase, row):
    kw = dict(case.fixed or {})
    kw.update(dict(zip(PARAMS, (float(v) for v in row))))
    kw.setdefault("nobreak", 1)
    kw.setdefault("Ec_sd", 0.0)
    kw.setdefault("Gc_sd", 0.0)
    return rock_material(float(case.radii.min()), float(case.radii.mean()), dt=case.dt, **kw)


def elastic_run(p: np.ndarray, case: ElasticCase):
    """(values (B, 2), Jacobians (B, 2, 5)) of (E_secant, nu_secant)."""
    P = np.atleast_2d(np.asarray(p, np.float64))
    ctx = Context(precision=2, device=case.device, deterministic=case.deterministic)
    try:
        ld = Loading.from_buffer_copy(case.loading)
        ld.max_steps = case.steps
        for row in P:
            ctx.add_sample(_material(case, row), ld, case.xyz, case.radii)
        ctx.setup()
        ctx.run(case.steps)
        out = [ctx.sensitivities(i) for i in range(len(P))]
    finally:
        ctx.close()
    assert list(SENS_NAMES) == ["E_bond", "kn_ks", "bond_radius", "E", "mu"]
    vals = np.array([[s["E_secant"], s["nu_secant"]] for s in out])
    jac = np.stack([np.stack([s["dE"], s["dnu"]]) for s in out])
    return vals, jac


class ElasticResponse(torch.autograd.Function):
    """p (5,) or (B, 5) float64 tensor -> (2,) or (B, 2): secant E (GPa) and
    secant Poisson ratio."""

    @staticmethod
    def forward(ctx, p: torch.Tensor, case: ElasticCase):
        vals, jac = elastic_run(p.detach().cpu().numpy(), case)
        J = torch.from_numpy(jac).to(p.dtype)
        ctx.save_for_backward(J)
        ctx.squeeze = p.dim() == 1
        out = torch.from_numpy(vals).to(p.dtype)
        return out[0] if ctx.squeeze else out

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        (J,) = ctx.saved_tensors
        g2 = g.reshape(-1, 2).to(J.dtype)
        grad = torch.einsum("bi,bij->bj", g2, J)
        return (grad[0] if ctx.squeeze else grad).to(g.dtype), None


def elastic_response(p: torch.Tensor, case: ElasticCase) -> torch.Tensor:
    return ElasticResponse.apply(p, case)
