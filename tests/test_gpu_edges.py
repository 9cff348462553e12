"""Edge cases of the engine through the public API (GPU).

  * argument and state errors come back as error codes, never as a fault:
    zero particles, null arrays, adding a sample after set-up, results of a
    sample that does not exist, running before set-up;
  * degenerate specimens run: a single sphere (no pairs at all), a specimen
    with no bonds (gap below any neighbour distance: contacts only), a
    specimen whose spheres all start outside the escape box (all parked);
  * ragged batches: 300 samples of very different sizes (1 to 3,000 spheres)
    in one context, each giving the result it gives alone (deterministic
    mode, so exactly).
"""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from dem_api import dem

W = importlib.import_module("dem-rock-calibration_b200.workloads")
S = importlib.import_module("dem-rock-calibration_b200.surrogate")
sweep = importlib.import_module("dem-rock-calibration_b200.sweep")
pytestmark = pytest.mark.gpu

KEYS = ("FractureStress", "FractureStrain", "E_chord", "nu", "steps", "bonds_now", "Destruction")


def _spec(n=2000, seed=5):
    J = S.UniaxialSolver(n=n, seed=seed)
    return J


def _loading(J, max_steps=2000):
    r_mean = float(J.rad.mean())
    return dem.loading(dem.TEST_UNIAXIAL, J.box, J.size_real, J.center_real, velocity=-0.1 / dem.VELOCITY,
                       min_stress=0.010, max_strain=0.01, cond_fracture=0.7, dNsave=100, max_steps=max_steps,
                       p_r_platen=r_mean)


def _mat(J, **over):
    p = dict(zip(J.keys, [40.0, 2.5, 0.04, 0.15, 0.5, 0.8]))
    m = sweep.material_for(p, float(J.rad.min()), float(J.rad.mean()), 7)
    for k, v in over.items():
        setattr(m, k, v)
    return m


def test_errors_are_codes_not_faults():
    J = _spec(800)
    L = dem.lib()
    ctx = dem.Context()
    h = ctx._h
    sid = dem.C.c_int32()
    ld = _loading(J)
    m = _mat(J)
    assert L.dem_add_sample(h, dem.C.byref(m), dem.C.byref(ld), dem._p(J.xyz), dem._p(J.rad), 0,
                            dem.C.byref(sid)) == -1                      # no particles
    assert L.dem_add_sample(h, dem.C.byref(m), dem.C.byref(ld), None, None, 10, dem.C.byref(sid)) == -1
    with pytest.raises(dem.DemError):
        ctx.run(10)                                                      # before set-up
    ctx.add_sample(m, ld, J.xyz, J.rad)
    ctx.setup()
    with pytest.raises(dem.DemError):
        ctx.add_sample(m, ld, J.xyz, J.rad)                              # after set-up
    with pytest.raises(dem.DemError):
        ctx.result(5)                                                    # no such sample
    ctx.run(50)
    assert ctx.result(0)["steps"] == 50
    ctx.close()


def test_single_sphere_runs():
    J = _spec(800)
    ctx = dem.Context()
    ld = _loading(J, max_steps=200)
    xyz = np.array([J.box.center[0], J.box.center[1], J.box.center[2]], np.float32)
    rad = np.array([0.25], np.float32)
    ctx.add_sample(_mat(J), ld, xyz, rad)
    ctx.setup()
    ctx.run(200)
    r = ctx.result(0)
    assert r["bonds_initial"] == 0 and r["steps"] == 200
    p = ctx.particles(0)
    assert np.all(np.isfinite(p["R"])) and np.all(np.isfinite(p["V"]))
    ctx.close()


def test_specimen_without_bonds_runs_on_contacts():
    J = _spec(2000)
    ctx = dem.Context()
    ctx.add_sample(_mat(J, gap=-1.0), _loading(J, max_steps=3000), J.xyz, J.rad)
    ctx.setup()
    assert ctx.counts()["bonds"] == 0
    ctx.run(3000)
    r = ctx.result(0)
    assert r["bonds_initial"] == 0 and r["stale"] == 0
    p = ctx.particles(0)
    assert np.all(np.isfinite(p["R"]))
    ctx.close()


def test_specimen_outside_the_box_is_parked():
    J = _spec(800)
    ctx = dem.Context()
    xyz = J.xyz.copy()
    xyz[2 * J.rad.size:] += 1000.0                                      # every sphere far above the box
    ctx.add_sample(_mat(J), _loading(J, max_steps=50), xyz, J.rad)
    ctx.setup()
    ctx.run(50)
    p = ctx.particles(0)
    R = p["R"].reshape(3, -1)
    hide = np.array(J.box.hidden_point, np.float32)
    assert np.allclose(R, hide[:, None], atol=1e-3)
    assert np.all(p["V"] == 0)
    ctx.close()


def test_ragged_batch_equals_single_runs():
    sizes = [1, 7, 60, 500, 3000]
    specs = [_spec(n, seed=11 + k) if n >= 100 else None for k, n in enumerate(sizes)]
    base = _spec(500, seed=11)

    def case(k):
        n = sizes[k]
        if specs[k] is not None:
            return specs[k], specs[k].xyz, specs[k].rad
        # tiny specimens: the first n spheres of a packed cylinder
        xyz = base.xyz.reshape(3, -1)[:, :n].reshape(-1).copy()
        return base, xyz, base.rad[:n].copy()

    order = [k % len(sizes) for k in range(300)]
    ctx = dem.Context(deterministic=True)
    for k in order:
        J, xyz, rad = case(k)
        ctx.add_sample(_mat(J), _loading(J, max_steps=400), xyz, rad)
    ctx.setup()
    ctx.run(400)
    batched = [ctx.result(i) for i in range(len(order))]
    ctx.close()
    for k in range(len(sizes)):
        J, xyz, rad = case(k)
        one = dem.Context(deterministic=True)
        one.add_sample(_mat(J), _loading(J, max_steps=400), xyz, rad)
        one.setup()
        one.run(400)
        r = one.result(0)
        one.close()
        for i in [i for i, kk in enumerate(order) if kk == k][:3]:
            assert all(batched[i][key] == r[key] or (np.isnan(batched[i][key]) and np.isnan(r[key]))
                       for key in KEYS), (sizes[k], i)


def test_non_finite_state_stops_its_sample_and_is_reported():
    """A NaN velocity put into one of two specimens (host-side injection):
    that specimen stops at the step where its state became non-finite
    (done, numeric flag), the call returns DEM_ERR_NUMERIC, the other
    specimen runs on unaffected; later calls succeed, and positions given
    with a NaN are refused up front."""
    J = _spec(800)
    ld = _loading(J, max_steps=10 ** 6)
    ctx = dem.Context()
    s0 = ctx.add_sample(_mat(J), ld, J.xyz, J.rad)
    s1 = ctx.add_sample(_mat(J), ld, J.xyz, J.rad)
    ctx.setup()
    p = ctx.particles(s0)
    V = p["V"].copy()
    V[7] = np.nan
    ctx.set_particles(s0, V=V)
    with pytest.raises(dem.DemError) as e:
        ctx.step(30)
    assert e.value.code == -8
    r0, r1 = ctx.result(s0), ctx.result(s1)
    assert r0["numeric"] == 1 and r0["done"] == 1 and r0["steps"] == 1, r0
    assert r1["numeric"] == 0 and r1["done"] == 0 and r1["steps"] == 30, r1
    ctx.step(10)                                   # no new non-finite state: no error
    assert ctx.result(s1)["steps"] == 40 and ctx.result(s0)["steps"] == 1
    ctx.close()
    bad = J.xyz.copy()
    bad[3] = np.inf
    ctx = dem.Context()
    with pytest.raises(dem.DemError) as e:
        ctx.add_sample(_mat(J), ld, bad, J.rad)
    assert e.value.code == -1
    ctx.close()


def test_contexts_reusing_cached_memory_repeat_exactly():
    """A closed context's device memory is reused by the next one (the
    library's block cache): every reused block starts zeroed, so the same
    run repeats bit for bit in a context of reused memory, after the cache
    went back to the driver (dem_release_cached_memory), and in a fresh one."""
    J = _spec(n=2000, seed=8)
    out = []
    for k in range(3):
        ctx = dem.Context(deterministic=True)
        sid = ctx.add_sample(_mat(J), _loading(J, max_steps=1500), J.xyz, J.rad)
        ctx.setup()
        ctx.run(10 ** 6)
        rec, _ = ctx.record(sid)
        out.append((ctx.result(sid)["FractureStress"], ctx.particles(sid)["R"].copy(), rec))
        ctx.close()
        if k == 1:
            dem.release_cached_memory()
    for fs, R, rec in out[1:]:
        assert fs == out[0][0] and np.array_equal(R, out[0][1]) and np.array_equal(rec, out[0][2])
