"""Deterministic mode (dem_options.deterministic): FP32 force, moment and
platen sums in exact 64-bit fixed point.

  * the same context run twice gives bit-identical results and records;
  * a case run inside a batch of four equals the same case run alone, bit for
    bit (a sample's results do not depend on the other samples of its
    context), which the float-atomic mode does not give;
  * one step's forces match the oracle and the reference kernels as in the
    float-atomic mode (test_gpu_parity.py runs its step cases in both modes);
  * whole loading tests agree with the float-atomic mode within the latter's
    own run-to-run scatter (UCS 10%, E and nu 3%).
"""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from dem_api import dem

S = importlib.import_module("dem-rock-calibration_b200.surrogate")
sweep = importlib.import_module("dem-rock-calibration_b200.sweep")
pytestmark = pytest.mark.gpu

KEYS = ("FractureStress", "FractureStrain", "E_chord", "nu", "steps", "bonds_now", "Destruction")


def _params(k):
    lo = np.array([v[0] for v in sweep.SWEEP_SPACE.values()])
    hi = np.array([v[1] for v in sweep.SWEEP_SPACE.values()])
    return S.latin_box(k, lo, hi, 4)


def _run(J, P, det=True):
    r_min, r_mean = float(J.rad.min()), float(J.rad.mean())
    ctx = dem.Context(deterministic=det)
    for row in P:
        ld = dem.loading(dem.TEST_UNIAXIAL, J.box, J.size_real, J.center_real, velocity=-0.1 / dem.VELOCITY,
                         min_stress=0.010, max_strain=0.01, cond_fracture=0.7, dNsave=100, max_steps=400000,
                         p_r_platen=r_mean)
        ctx.add_sample(sweep.material_for(dict(zip(J.keys, row)), r_min, r_mean, 7), ld, J.xyz, J.rad)
    ctx.setup()
    ctx.run(400000)
    out = [(ctx.result(i), ctx.record(i)[0]) for i in range(len(P))]
    ctx.close()
    return out


def test_runs_are_bit_reproducible_and_independent_of_the_batch():
    J = S.UniaxialJudge(n=2000, seed=5)
    P = _params(4)
    a = _run(J, P)
    b = _run(J, P)
    for (ra, ca), (rb, cb) in zip(a, b):
        assert all(ra[k] == rb[k] for k in KEYS)
        assert np.array_equal(ca, cb)
    for i in (0, 3):
        (rs, cs), = _run(J, P[i:i + 1])
        assert all(a[i][0][k] == rs[k] for k in KEYS), (i, {k: (a[i][0][k], rs[k]) for k in KEYS})
        assert np.array_equal(a[i][1], cs)


def test_deterministic_mode_agrees_with_float_atomics():
    J = S.UniaxialJudge(n=2000, seed=5)
    P = _params(4)
    d = _run(J, P, det=True)
    f = _run(J, P, det=False)
    for (rd, _), (rf, _) in zip(d, f):
        assert rd["FractureStress"] == pytest.approx(rf["FractureStress"], rel=0.10)
        assert rd["E_chord"] == pytest.approx(rf["E_chord"], rel=0.03)
        assert rd["nu"] == pytest.approx(rf["nu"], rel=0.03, abs=2e-3)
