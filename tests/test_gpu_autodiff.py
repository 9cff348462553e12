"""ElasticResponse (torch.autograd.Function over the sensitivity build)
against the sensitivities themselves and against central finite
differences of a calibration loss.

A polydisperse cylinder of about 3,000 spheres, unbreakable bonds, 2,000
steps of uniaxial loading at a fixed time step, rolling friction off (as in
test_gpu_sensitivity.py, whose docstring gives the reason).  Loss =
sum(((y - y*) / s)^2) over (secant E, secant nu) with y* the response at
1.1 x the bond modulus and 0.9 x kn/ks.  Runs in deterministic mode (exact
fixed-point force sums).  Tolerances: backward = g J with J's rows from
autograd on the same forward run, to 1e-12; a second run repeats the values
and the Jacobian exactly; against central differences with h = 1e-4 within
TOL_FD of the gradient's norm; a batch of two equals the two single runs
exactly.
"""
from __future__ import annotations

import importlib
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
AD = importlib.import_module("dem-rock-calibration_b200.autodiff")
W = importlib.import_module("dem-rock-calibration_b200.workloads")
pytestmark = pytest.mark.gpu

STEPS = 2000
BASE = [30.0, 2.5, 0.8, 50.0, 0.5]
TOL_FD = 1e-3


def _case():
    d = (3000 * 0.068068 / (0.58 * math.pi * 0.5)) ** (1 / 3)
    spec = W.uniaxial_cylinder(seed=3, diameter=d, height=2 * d)
    r_min = float(spec.radii.min())
    nu, rho, E = 0.25, 2.65, 50.0
    t_r = math.pi * r_min * math.sqrt(2 * rho * (1 + nu)) / (math.sqrt(E) * (0.163 * nu + 0.8766))
    return AD.ElasticCase(spec.xyz, spec.radii, spec.loading, STEPS, 0.2 * t_r, fixed={"mur": 0.0})


def test_autograd_gradient_matches_sensitivities_and_finite_differences():
    case = _case()
    tgt_p = np.array(BASE) * np.array([1.1, 0.9, 1.0, 1.0, 1.0])
    target = torch.from_numpy(AD.elastic_run(tgt_p, case)[0][0])
    scale = torch.tensor([1.0, 0.01], dtype=torch.float64)

    def loss_of(y):
        return (((y - target) / scale) ** 2).sum()

    p = torch.tensor(BASE, dtype=torch.float64, requires_grad=True)
    y = AD.elastic_response(p, case)
    # rows of the Jacobian through autograd itself (the same forward run)
    J = torch.stack([torch.autograd.grad(y, p, e, retain_graph=True)[0]
                     for e in torch.eye(2, dtype=torch.float64)])
    L = loss_of(y)
    L.backward()
    g_out = 2 * (y.detach() - target) / scale ** 2
    assert torch.allclose(p.grad, g_out @ J, rtol=1e-12, atol=0)
    vals, jac = AD.elastic_run(np.array(BASE), case)
    assert float(y[0]) == vals[0][0] and float(y[1]) == vals[0][1]      # deterministic runs repeat exactly
    assert torch.equal(J, torch.from_numpy(jac[0]))
    h = 1e-4
    fd = np.zeros(5)
    for k in range(5):
        up, dn = np.array(BASE), np.array(BASE)
        up[k] *= 1 + h
        dn[k] *= 1 - h
        fd[k] = (float(loss_of(torch.from_numpy(AD.elastic_run(up, case)[0][0]))) -
                 float(loss_of(torch.from_numpy(AD.elastic_run(dn, case)[0][0])))) / (2 * h * BASE[k])
    g = p.grad.numpy()
    scale = np.linalg.norm(fd * np.array(BASE))          # relative sensitivities p dL/dp
    for k in range(5):
        print(f"\np dL/dp[{k}]: autograd {g[k] * BASE[k]:+.6e}  central difference {fd[k] * BASE[k]:+.6e}  "
              f"|diff| / norm {abs(g[k] - fd[k]) * BASE[k] / scale:.2e}", end="")
    print()
    assert np.all(np.abs(g - fd) * np.array(BASE) <= TOL_FD * scale), (g, fd)


def test_batched_response_equals_single_runs():
    case = _case()
    P = torch.tensor([BASE, [40.0, 2.0, 0.7, 50.0, 0.4]], dtype=torch.float64)
    yb = AD.elastic_response(P, case)
    for i in range(2):
        ys = AD.elastic_response(P[i], case)
        assert torch.equal(yb[i], ys)
