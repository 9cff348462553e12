"""Forward-mode sensitivities (precision 2) against central finite
differences of the plain FP64 engine.

A polydisperse cylinder of about 3,000 spheres (diameter 7.2 mm, height
14.4 mm), unbreakable bonds, the uniaxial loading of the cylinder workload
for 2,000 steps with a fixed time step.  Secant modulus and secant Poisson
ratio at the last step and their derivatives with respect to the bond
modulus, kn/ks, the bond-radius factor, the particle modulus and the density,
against (f(p(1+h)) - f(p(1-h))) / (2 h p) with h = 1e-3.

Contact events (spheres touching a platen one step earlier or later) make
finite differences with much smaller h noisy in a DEM run; with h = 1e-3 the
bond and modulus derivatives agree within 3% (measured 0.03-1.1%), the
density derivative - inertia at this loading rate, where the tangent leaves
out the overlap dependence of the contact damping - within 25% (measured 19%).
"""
from __future__ import annotations

import importlib
import math

import numpy as np
import pytest

from dem_api import dem

W = importlib.import_module("dem-rock-calibration_b200.workloads")
pytestmark = pytest.mark.gpu

STEPS = 2000
BASE = dict(E_bond=30.0, kn_ks=2.5, bond_radius_factor=0.8, E=50.0, rho=2.65)
TOL = dict(E_bond=0.03, kn_ks=0.03, bond_radius_factor=0.03, E=0.03, rho=0.25)


def _run(spec, mat, precision):
    ctx = dem.Context(precision=precision)
    ld = dem.Loading.from_buffer_copy(spec.loading)
    ld.max_steps = STEPS
    ctx.add_sample(mat, ld, spec.xyz, spec.radii)
    ctx.setup()
    ctx.run(STEPS)
    s = ctx.sensitivities(0)
    r = ctx.result(0)
    ctx.close()
    return s, r


def test_sensitivities_match_central_differences():
    d = (3000 * 0.068068 / (0.58 * math.pi * 0.5)) ** (1 / 3)
    spec = W.uniaxial_cylinder(seed=3, diameter=d, height=2 * d)
    r_min, r_mean = float(spec.radii.min()), float(spec.radii.mean())
    nu = 0.25
    t_r = math.pi * r_min * math.sqrt(2 * BASE["rho"] * (1 + nu)) / (math.sqrt(BASE["E"]) * (0.163 * nu + 0.8766))

    def mat(**over):
        kw = dict(BASE)
        kw.update(over)
        return W.rock_material(r_min, r_mean, nobreak=1, dt=0.2 * t_r, Ec_sd=0.0, Gc_sd=0.0, **kw)

    s, r = _run(spec, mat(), 2)
    assert r["stale"] == 0 and r["bonds_now"] == r["bonds_initial"]
    assert s["stress"] > 0 and 1.0 < s["E_secant"] < 50.0 and 0.0 < s["nu_secant"] < 0.5
    plain, _ = _run(spec, mat(), 1)
    assert s["E_secant"] == pytest.approx(plain["E_secant"], rel=1e-3)
    h = 1e-3
    for k, name in enumerate(dem.SENS_NAMES):
        key = "bond_radius_factor" if name == "bond_radius" else name
        v = BASE[key]
        up, _ = _run(spec, mat(**{key: v * (1 + h)}), 1)
        dn, _ = _run(spec, mat(**{key: v * (1 - h)}), 1)
        fd_E = (up["E_secant"] - dn["E_secant"]) / (2 * h * v)
        fd_nu = (up["nu_secant"] - dn["nu_secant"]) / (2 * h * v)
        assert abs(s["dE"][k] - fd_E) <= TOL[key] * abs(fd_E), (name, s["dE"][k], fd_E)
        assert abs(s["dnu"][k] - fd_nu) <= TOL[key] * abs(fd_nu), (name, s["dnu"][k], fd_nu)
