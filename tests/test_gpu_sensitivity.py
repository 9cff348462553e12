"""Forward-mode sensitivities (precision 2) at the size of the gradient
configuration, against central finite differences and against the
reference's conjugate-gradient direction.

The run: a polydisperse cylinder of 20,000 spheres (radii U[0.20, 0.30] mm,
height twice the diameter) with the plain uniaxial configuration's physics
(particle E 50 GPa, nu 0.25, rho 2650 kg/m^3, friction 0.5; bond E 30 GPa,
kn/ks 2.5, bond radius 0.8 min(r_i, r_j)), unbreakable bonds, 4,000 steps of
uniaxial loading at a fixed time step (0.2 of the Rayleigh step), FP64.  The
sensitivity build carries the five tangents (bond modulus, kn/ks,
bond-radius factor, particle modulus, sliding friction) through the FP64
kernels; the differences use the plain FP64 build.  Deterministic mode
(exact fixed-point force sums): the two runs of a difference differ only by
the parameter change.

Rolling friction is off (mur = 0).  Its moment, -mur |F_n| w / |w|, flips
direction whenever a spin passes through zero; with it on (mur = 0.05, the
reference's value) the secant modulus of this run scatters by about 7e-7
(relative) around a smooth curve from one parameter value to the next (the
residual of a quadratic fit over eleven values within +-1e-4), so a central
difference with h = 1e-4 carries a noise of about 3e-3 and cannot check a
derivative to 1e-3.  With mur = 0 the scatter is about 2e-9.

1. Secant modulus E: relative sensitivities (p / E) dE/dp within 1e-3 of
   (E(p(1+h)) - E(p(1-h))) / (2 h E), h = 1e-4, for every parameter (the
   friction sensitivity, about 1e-7, against 1e-3 of 5% of the gradient's
   norm instead of its own size).
2. Secant Poisson ratio nu: the same comparison, within 2e-3 of the norm of
   the relative-sensitivity vector for every parameter (measured: up to
   1.5e-3; its smallest components, about 0.02, are known to only a few
   percent).
3. Conjugate-gradient direction: the first step of the reference's
   calibration update (CalculateNewParameters2, mp_task.h:253-300, as
   calibrate.descent_step) for a target (E, nu) of a stiffer bond and a
   softer kn/ks, with weights 1 / goal^2 (mp_task.h:133).  The direction from
   the tangents against the one from central differences (cosine above
   1 - 1e-5), and against the reference's own procedure: one-sided
   differences with each parameter raised by 10% (MaterialDeltaFactor 0.1,
   mp_task.h:144, one solve per parameter as in CalculateStepCG,
   mp_determineconjgradient.cu:84-145), cosine above 0.99 (the 10% steps
   see the curvature of the response).

Every comparison is printed (pytest -s).
"""
from __future__ import annotations

import importlib
import math

import numpy as np
import pytest

from dem_api import dem

W = importlib.import_module("dem-rock-calibration_b200.workloads")
cal = importlib.import_module("dem-rock-calibration_b200.calibrate")
pytestmark = pytest.mark.gpu

N_SPHERES = 20000
STEPS = 4000
H = 1e-4
BASE = dict(E_bond=30.0, kn_ks=2.5, bond_radius_factor=0.8, E=50.0, mu=0.5)
KEYS = ("E_bond", "kn_ks", "bond_radius_factor", "E", "mu")    # the order of dem.SENS_NAMES
RHO = 2.65
TOL_E = 1e-3
TOL_NU = 2e-3


@pytest.fixture(scope="module")
def case():
    d = (N_SPHERES * 0.068068 / (0.58 * math.pi * 0.5)) ** (1 / 3)
    spec = W.uniaxial_cylinder(seed=3, diameter=d, height=2 * d)
    r_min, r_mean = float(spec.radii.min()), float(spec.radii.mean())
    nu = 0.25
    t_r = math.pi * r_min * math.sqrt(2 * RHO * (1 + nu)) / (math.sqrt(BASE["E"]) * (0.163 * nu + 0.8766))

    def mat(p):
        return W.rock_material(r_min, r_mean, nobreak=1, dt=0.2 * t_r, Ec_sd=0.0, Gc_sd=0.0, rho=RHO, mur=0.0,
                               **dict(zip(KEYS, p)))

    def run(p, precision):
        ctx = dem.Context(precision=precision, deterministic=True)
        ld = dem.Loading.from_buffer_copy(spec.loading)
        ld.max_steps = STEPS
        ctx.add_sample(mat(p), ld, spec.xyz, spec.radii)
        ctx.setup()
        ctx.run(STEPS)
        s = ctx.sensitivities(0)
        r = ctx.result(0)
        ctx.close()
        return s, r

    p0 = np.array([BASE[k] for k in KEYS])
    s, r = run(p0, 2)
    plain, _ = run(p0, 1)
    # central differences of the plain FP64 build, h = 1e-4 relative
    fd = np.zeros((5, 2))
    for k in range(5):
        up, dn = p0.copy(), p0.copy()
        up[k] *= 1 + H
        dn[k] *= 1 - H
        su, _ = run(up, 1)
        sd, _ = run(dn, 1)
        fd[k] = [(su["E_secant"] - sd["E_secant"]) / (2 * H * p0[k]),
                 (su["nu_secant"] - sd["nu_secant"]) / (2 * H * p0[k])]
    return dict(spec=spec, run=run, p0=p0, s=s, r=r, plain=plain, fd=fd)


def test_run_is_the_gradient_configuration(case):
    s, r, spec = case["s"], case["r"], case["spec"]
    assert abs(spec.n - N_SPHERES) <= 0.05 * N_SPHERES
    assert r["steps"] == STEPS and r["bonds_now"] == r["bonds_initial"] and r["stale"] == 0
    assert s["stress"] > 0 and 1.0 < s["E_secant"] < 50.0 and 0.0 < s["nu_secant"] < 0.5
    # the sensitivity build's values are those of the plain FP64 build
    assert s["E_secant"] == pytest.approx(case["plain"]["E_secant"], rel=1e-9)
    assert s["nu_secant"] == pytest.approx(case["plain"]["nu_secant"], rel=1e-9)


def _relative(case, which):
    s, p0, fd = case["s"], case["p0"], case["fd"]
    f = s["E_secant"] if which == 0 else s["nu_secant"]
    tg = np.array(s["dE"] if which == 0 else s["dnu"]) * p0 / f
    return tg, fd[:, which] * p0 / f


def test_modulus_sensitivities_within_1e3_of_central_differences(case):
    tg, fd = _relative(case, 0)
    scale = np.maximum(np.abs(fd), 0.05 * np.linalg.norm(fd))
    for name, a, b, sc in zip(dem.SENS_NAMES, tg, fd, scale):
        print(f"\n(p/E) dE/d{name}: tangent {a:+.7f}  central difference {b:+.7f}  |diff| / scale {abs(a - b) / sc:.2e}",
              end="")
    print()
    assert np.all(np.abs(tg - fd) <= TOL_E * scale), (tg, fd)


def test_poisson_sensitivities_against_central_differences(case):
    tg, fd = _relative(case, 1)
    norm = np.linalg.norm(fd)
    for name, a, b in zip(dem.SENS_NAMES, tg, fd):
        print(f"\n(p/nu) dnu/d{name}: tangent {a:+.7f}  central difference {b:+.7f}  |diff| / norm {abs(a - b) / norm:.2e}",
              end="")
    print()
    assert np.all(np.abs(tg - fd) <= TOL_NU * norm), (tg, fd)


def test_cg_direction_matches_the_reference_procedure(case):
    run, p0, s = case["run"], case["p0"], case["s"]
    R0 = np.array([s["E_secant"], s["nu_secant"]])
    target = p0 * np.array([1.1, 0.9, 1.0, 1.0, 1.0])
    st, _ = run(target, 1)
    goal = np.array([st["E_secant"], st["nu_secant"]])
    weight = 1.0 / goal ** 2
    J_tan = np.stack([s["dE"], s["dnu"]], axis=1)                 # dR[i, j] = dR_j / dp_i
    J_cd = case["fd"]
    # the reference's procedure: one solve per parameter raised by 10%, one-sided differences
    var = 0.1 * p0
    Rv = np.zeros((5, 2))
    for k in range(5):
        p = p0.copy()
        p[k] += var[k]
        sv, _ = run(p, 1)
        Rv[k] = [sv["E_secant"], sv["nu_secant"]]
    J_ref = cal.finite_difference_jacobian(R0, Rv, var)
    d_tan, t_tan = cal.descent_step(R0, J_tan, goal, weight)
    d_cd, t_cd = cal.descent_step(R0, J_cd, goal, weight)
    d_ref, t_ref = cal.descent_step(R0, J_ref, goal, weight)
    cos = lambda a, b: float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
    print(f"\nCG direction: cosine(tangent, central differences) {cos(d_tan, d_cd):.9f}, "
          f"cosine(tangent, reference 10% one-sided) {cos(d_tan, d_ref):.6f}; step p - t d: "
          f"tangent {p0 - t_tan * d_tan}, reference {p0 - t_ref * d_ref}")
    assert cos(d_tan, d_cd) > 1 - 1e-5
    assert cos(d_tan, d_ref) > 0.99
    # the step lengths agree as the directions do
    assert t_tan * np.linalg.norm(d_tan) == pytest.approx(t_cd * np.linalg.norm(d_cd), rel=5e-3)
