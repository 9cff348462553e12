"""Conjugate-gradient calibration driver: the parameter update against the
reference's own mp_task_data::CalculateStartParameters and
CalculateNewParameters2 (mp_task.h:129-311, compiled into oracle/_ref), which
are host code and run here without a GPU; and (GPU) one batched CG step."""
from __future__ import annotations

import ctypes as C
import importlib

import numpy as np
import pytest

from dem_api import dem  # noqa: F401
from oracle import lib as L

cal = importlib.import_module("dem-rock-calibration_b200.calibrate")
needs_ref = pytest.mark.skipif(not L.ref_available(), reason="reference harness not built")


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _ref_start(params, goal, mult, calc_u, calc_b, vtype, delta):
    g = np.array(goal, np.float64)
    w = np.zeros(4)
    var = np.zeros(30)
    L.ref().refh_cg_start_parameters(_p(np.array(params, np.float64)), _p(g), _p(np.array(mult, np.float64)),
                                     int(calc_u), int(calc_b), vtype, delta, _p(w), _p(var))
    return g, w, var.reshape(6, 5)


@needs_ref
@pytest.mark.parametrize("calc_u,calc_b,vtype", [(True, False, 7), (True, True, 2), (False, True, 0)])
def test_start_parameters_match_reference(calc_u, calc_b, vtype):
    params = np.array([17.1, 0.618, 0.503, 1.64e-3, 5.9e-2])
    goal = [0.0048, 0.104, 0.0105, 1.0]
    mult = [50.0, 100.0, 1.0, 10000.0]
    t = cal.CGTask(params=params, goal=np.array(goal), weight_multiplier=np.array(mult), variation_type=vtype,
                   calc_u=calc_u, calc_b=calc_b)
    t.start_parameters()
    g, w, var = _ref_start(params, goal, mult, calc_u, calc_b, vtype, 0.1)
    assert np.array_equal(t.goal, g) and np.array_equal(t.weight, w) and np.array_equal(t.variation, var)


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_new_parameters_match_reference(seed):
    rng = np.random.default_rng(seed)
    params = np.array([rng.uniform(5, 60), rng.uniform(0.02, 0.9), rng.uniform(0.02, 0.9),
                       rng.uniform(0.05, 0.4), rng.uniform(0.005, 0.1)])
    if seed == 5:
        params[1] = 1e-7  # drives the update below a SetMaterialContractions floor
    t = cal.CGTask(params=params, goal=np.array([0.005, 0.1, 0.01, 1.0]),
                   weight_multiplier=np.array([50.0, 100.0, 1.0, 1e4]), variation_type=int(seed % 8))
    t.start_parameters()
    t.rfun[:] = rng.uniform(0.5, 1.5, (6, 4)) * np.array([0.005, 0.1, 0.01, 1.0])
    t.dfun[1:] = rng.normal(0, 1e3, 5) if seed % 2 else 0.0
    t.ddfun[1:] = rng.normal(0, 1e3, 5) if seed % 2 else 0.0
    var = t.variation.reshape(-1).copy()
    dfun, ddfun = t.dfun.copy(), t.ddfun.copy()
    new_ref, fun_ref = np.zeros(5), np.zeros(4)
    L.ref().refh_cg_new_parameters2(_p(t.params), _p(var), _p(t.rfun.reshape(-1).copy()), _p(t.goal), _p(t.weight),
                                    _p(dfun), _p(ddfun), t.variation_type, t.delta_factor, _p(new_ref), _p(fun_ref))
    new = t.new_parameters()
    assert np.array_equal(new, new_ref)
    assert np.array_equal(t.variation.reshape(-1), var)
    assert np.array_equal(t.dfun, dfun) and np.array_equal(t.ddfun, ddfun)
    assert np.array_equal(t.functional, fun_ref)


def test_solve_parameters_skip_unvaried_rows():
    t = cal.CGTask(params=np.array([17.1, 0.6, 0.5, 0.16, 0.06]), goal=np.ones(4), weight_multiplier=np.ones(4),
                   variation_type=6)  # type 6 varies E only
    t.start_parameters()
    assert np.allclose(t.solve_parameters(1), t.params + [1.71, 0, 0, 0, 0])
    assert all(t.solve_parameters(i) is None for i in range(2, 6))
    assert np.array_equal(t.solve_parameters(0), t.params)


@pytest.mark.gpu
def test_cg_step_runs_its_solves_in_one_context(tmp_path):
    """Two CG steps on a small reference-mode cylinder (about 800 spheres of
    0.5 mm): six uniaxial solves per step in one batched context (bounded to
    3000 steps each), then the update."""
    import dem_testlib as T
    from test_gpu_parity import _loading

    # p_r 0.5 mm: the particle radius SetVariationParameters uses
    c = T.ref_case(seed=2, lsi=(0.009, 0.009, 0.014), space=(0.018, 0.018, 0.026), p_r_si=0.5e-3, jitter_frac=0.1,
                   lattice_gap=0.5)
    uni = cal.Specimen(xyz=c.R, loading=_loading(c))
    p0 = np.array([30.0, 0.040, 0.040, 0.2, 0.025])  # E, Ec, Gc (GPa), b_r, gap (mm)
    task = cal.CGTask(params=p0, goal=np.array([0.006, 0.045, 0.01, 1.0]),
                      weight_multiplier=np.array([50.0, 100.0, 1.0, 1e4]), variation_type=0)
    # type 0 varies E, Ec, Gc only: an update of the bond gap could exceed the
    # engine's 48 partners per sphere (DEM_ERR_CAPACITY), as it would overflow
    # the reference's 32 interaction slots
    out = tmp_path / "CalculationResults.dat"
    cal.calibrate(task, uni, None, steps=2, max_steps=3000, results_file=str(out))
    assert len(task.history) == 2
    for h in task.history:
        assert np.all(np.isfinite(h["params"])) and h["results"][1] > 0
    assert np.all(np.isfinite(task.params)) and not np.array_equal(task.params, p0)
    assert out.read_text().count("Step:") == 2


def test_descent_step_is_the_first_cg_update():
    """descent_step (any Jacobian, any sizes) reproduces the first update of
    CGTask.new_parameters (the reference's CalculateNewParameters2 with no
    previous direction) when given the reference's finite-difference Jacobian."""
    rng = np.random.default_rng(4)
    params = np.array([17.1, 0.618, 0.503, 1.64e-3, 5.9e-2])
    goal = np.array([0.0048, 0.104, 0.0105, 1.0])
    t = cal.CGTask(params=params, goal=goal, weight_multiplier=np.array([50.0, 100.0, 1.0, 1e4]), variation_type=2,
                   calc_u=True, calc_b=True)
    t.start_parameters()
    t.rfun[:] = goal[None, :] * (1.0 + 0.2 * rng.standard_normal((6, 4)))
    var = np.array([t.variation[i + 1, i] for i in range(5)])
    dR = cal.finite_difference_jacobian(t.rfun[0], t.rfun[1:], var)
    dfun, step = cal.descent_step(t.rfun[0], dR, t.goal, t.weight)
    new = t.new_parameters()
    want = params - step * dfun
    want = np.maximum(want, np.array(cal.FLOORS))
    assert np.allclose(new, want, rtol=1e-12, atol=0)
    assert np.allclose(t.dfun[1:], dfun, rtol=1e-12, atol=0)
