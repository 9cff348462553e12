"""Multi-step and macro parity of the CUDA engine.

* trajectory: 40 steps from the same bonded state (no platens), engine vs the
  CPU oracle: bond topology identical, positions within 1e-5 of the
  displacement scale, velocities within 1e-4 of the velocity scale;
* macro: the full uniaxial test through dem_calculation_test against the
  reference's own driver h_CalculationUniaxialCompression (compiled from the
  reference sources, oracle/_ref) on the same sample file: peak stress (UCS)
  and strain at peak within 1%, secant modulus within 1%.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

import dem_testlib as T
from dem_api import dem
from oracle import lib as L
from oracle import sim
from test_gpu_parity import _loading, _material, load_state
from test_oracle_golden import SMALL, load

pytestmark = pytest.mark.gpu


def test_trajectory_matches_oracle():
    c = T.ref_case(seed=11, **SMALL)
    g = load("step_u_plain")
    st = sim.RefState.from_dict(g, "in_")
    ctx = dem.Context()
    sid = ctx.add_sample(_material(c), _loading(c, test=dem.TEST_NONE), c.R)
    ctx.setup()
    load_state(ctx, sid, c, st)
    orc = st.copy()
    stages = sim.STAGE_ALL & ~sim.STAGE_PLATEN
    nsteps = 40
    for _ in range(nsteps):
        sim.oracle_step(orc, c.sc, stages=stages)
    ctx.step(nsteps)
    p = ctx.particles(sid)
    # positions: relative to the displacement of the run, plus two ulp of the
    # coordinates themselves (only the force summation order differs)
    dx = np.abs(orc.R.astype(np.float64) - st.R).max()
    err_r = np.abs(p["R"].astype(np.float64) - orc.R)
    ulp = np.spacing(np.abs(orc.R)).astype(np.float64)
    assert np.all(err_r <= 1e-4 * dx + 2 * ulp), (err_r.max(), dx)
    vs = np.abs(orc.V).max()
    assert np.abs(p["V"] - orc.V).max() <= 1e-4 * vs
    ws = np.abs(orc.W).max()
    assert np.abs(p["W"] - orc.W).max() <= 1e-4 * ws
    pr = ctx.pairs(sid)
    intact = {(int(i), int(j)) for i, j, k in zip(pr["i"], pr["j"], pr["kind"]) if k == 1}
    IL = orc.IL.reshape(orc.N, 32)
    ty = orc.ILtype.reshape(orc.N, 32)
    ref = {(i, int(IL[i, k])) for i in range(orc.N) for k in range(32)
           if IL[i, k] != L.EMPTY and ty[i, k] == 1 and i < IL[i, k]}
    assert intact == ref
    assert ctx.result(sid)["stale"] == 0


def _write_sample(tmp, name, xyz):
    os.makedirs(tmp / "result", exist_ok=True)
    dem.save_cylinder_sample(str(tmp / "result" / name), xyz)


@pytest.mark.skipif(not L.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("seed", [1, 2])
def test_uniaxial_macro_matches_reference_driver(tmp_path, seed):
    # reference-mode specimen: equal radii 0.25 mm, lattice packing, the
    # reference's loading protocol (0.1 m/s, MinStress 10 MPa, MaxStrain 1%)
    lsi, space = (0.0045, 0.0045, 0.007), (0.009, 0.009, 0.013)
    c = T.ref_case(seed=seed, lsi=lsi, space=space, jitter_frac=0.02)
    _write_sample(tmp_path, f"Sample_0_{seed}.txt", c.R)
    k = c.kw
    q = L.TestParams(E=k["E"], Ec=k["Ec"], Gc=k["Gc"], b_r=k["br_si"], gap=k["gap_si"], p_r_m=k["p_r_si"],
                     rho=2610.0, nu=0.247, p_e=0.6, p_mu=0.45, p_mur=0.05, farcut_factor=3.2,
                     velocity_si=-0.1, minstress_si=10e6, maxstrain=0.01, condfract=0.1, dNsave=100, fileN=seed,
                     isample=0)
    for d in range(3):
        q.space_si[d] = space[d]
        q.lsi[d] = lsi[d]
    out = L.TestResult()
    rc = L.ref().refh_run_test(0, str(tmp_path).encode(), f"_{seed}".encode(), C.byref(q), C.byref(out))
    assert rc == 0
    ref_rec = np.loadtxt(tmp_path / "result" / f"Uniaxial_{seed}.txt", skiprows=1).reshape(-1, 3)
    # the same file through the product's loader and driver
    xyz, size_real, center_real = dem.load_cylinder_sample(str(tmp_path / "result" / f"Sample_0_{seed}.txt"),
                                                           c.pot.p_r)
    box = dem.reference_space(space, lsi, c.pot.p_r, 3.2)
    ld = dem.loading(dem.TEST_UNIAXIAL, box, size_real, center_real, velocity=-0.1 / dem.VELOCITY,
                     min_stress=10e6 / dem.STRESS, max_strain=0.01, cond_fracture=0.1, dNsave=100)
    res, rec, rb = dem.calculation_test(_material(c), ld, xyz)
    ucs_ref, ucs = out.FractureStress, res["FractureStress"]
    assert ucs_ref > 0 and ucs > 0
    assert abs(ucs - ucs_ref) <= 0.01 * ucs_ref, (ucs, ucs_ref)
    assert abs(res["FractureStrain"] - out.FractureStrain) <= 0.01 * out.FractureStrain
    # secant modulus at half the peak stress from both stress-strain records
    def secant(r):
        eps = -r[:, 0]
        sig = 0.5 * (np.abs(r[:, 1]) + np.abs(r[:, 2]))
        if sig.size < 3:
            return np.nan
        kk = int(np.argmax(sig >= 0.5 * sig.max()))
        return sig[kk] / eps[kk] if eps[kk] > 0 else np.nan
    e_ref = secant(np.column_stack([ref_rec[:, 0], ref_rec[:, 1] / 1e9, ref_rec[:, 2] / 1e9]))
    e_b = secant(rec)
    assert abs(e_b - e_ref) <= 0.01 * e_ref, (e_b, e_ref)
