"""Forward-mode sensitivities (precision 2) against central finite
differences of the plain FP64 engine.

A polydisperse cylinder of about 3,000 spheres (diameter 7.2 mm, height
14.4 mm), unbreakable bonds, the uniaxial loading of the cylinder workload
for 2,000 steps with a fixed time step.  Secant modulus and secant Poisson
ratio at the last step and their derivatives with respect to the bond
modulus, kn/ks, the bond-radius factor, the particle modulus and the sliding
friction coefficient, against (f(p(1+h)) - f(p(1-h))) / (2 h p) with h = 1e-3.

All runs in deterministic mode (exact fixed-point force sums), so the two
runs of a central difference differ only by the parameter change and not by
the order of floating-point atomic adds, which contact events would amplify
into the difference quotient.  Compared as relative sensitivities
(p / f) df/dp: within 6% of the finite difference plus 1e-4 (measured
0.3-4.5% over specimens and parameters): the tangent drops the derivatives
of the non-Lipschitz contact terms (the overlap factor of the contact
damping, the Coulomb and rolling directions) and follows each contact's own
history, while the difference quotient also sees contact onsets moving by a
step.  Every comparison is printed.  Contact events (spheres touching a platen one step earlier or
later) make finite differences with much smaller h noisy in a DEM run.  With
bonds unbreakable, few unbonded contacts slide before the secant point, so
the friction sensitivity is small; the absolute floor covers it.
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
BASE = dict(E_bond=30.0, kn_ks=2.5, bond_radius_factor=0.8, E=50.0, mu=0.5)
# the particle modulus acts through Hertz contacts (platens, unbonded pairs)
# whose onset steps shift with it: the tangent follows each contact history,
# the difference quotient also sees onsets moving by a step
TOL = 0.06
FLOOR = 1e-4
RHO = 2.65


def _run(spec, mat, precision):
    ctx = dem.Context(precision=precision, deterministic=True)
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
    t_r = math.pi * r_min * math.sqrt(2 * RHO * (1 + nu)) / (math.sqrt(BASE["E"]) * (0.163 * nu + 0.8766))

    def mat(**over):
        kw = dict(BASE)
        kw.update(over)
        return W.rock_material(r_min, r_mean, nobreak=1, dt=0.2 * t_r, Ec_sd=0.0, Gc_sd=0.0, rho=RHO, **kw)

    s, r = _run(spec, mat(), 2)
    assert r["stale"] == 0 and r["bonds_now"] == r["bonds_initial"]
    assert s["stress"] > 0 and 1.0 < s["E_secant"] < 50.0 and 0.0 < s["nu_secant"] < 0.5
    plain, _ = _run(spec, mat(), 1)
    assert s["E_secant"] == pytest.approx(plain["E_secant"], rel=1e-3)
    h = 1e-3
    rows = []
    for k, name in enumerate(dem.SENS_NAMES):
        key = "bond_radius_factor" if name == "bond_radius" else name
        v = BASE[key]
        up, _ = _run(spec, mat(**{key: v * (1 + h)}), 1)
        dn, _ = _run(spec, mat(**{key: v * (1 - h)}), 1)
        # relative sensitivities (v / f) df/dv
        fd_E = (up["E_secant"] - dn["E_secant"]) / (2 * h) / s["E_secant"]
        fd_nu = (up["nu_secant"] - dn["nu_secant"]) / (2 * h) / s["nu_secant"]
        tg_E = s["dE"][k] * v / s["E_secant"]
        tg_nu = s["dnu"][k] * v / s["nu_secant"]
        rows.append((name, "E", tg_E, fd_E))
        rows.append((name, "nu", tg_nu, fd_nu))
    for name, what, tg, fd in rows:
        print(f"d{what}/d{name} (relative): tangent {tg:+.5f}  central difference {fd:+.5f}  "
              f"rel.diff {abs(tg - fd) / max(abs(fd), 1e-12):.4f}")
    bad = [r for r in rows if abs(r[2] - r[3]) > TOL * abs(r[3]) + FLOOR]
    assert not bad, bad
