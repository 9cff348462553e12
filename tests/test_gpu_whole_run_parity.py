"""Whole loading tests, engine against the oracle, bit for bit, to fracture.

The engine's deterministic mode sums every particle's pair forces and
moments, and the platen and lateral-surface force sums, exactly (64-bit fixed
point).  The oracle runs the reference's loop body and host controller
(oracle/drive.py: md_calculationuniaxialcompression.cu:265-314,
md_calculationbraziltest.cu:185-231, md_results.cu:56-145,
md_data_types.h:347-494) with the same exact sums (fixsum=True).  Every
per-pair quantity of both is the reference's (the per-step tests pin the
oracle to the reference's kernels); the one difference from the reference
left is that it adds a particle's slots one after another in float
(md_calculateforcesdem3.cu:20-486), an order the engine's one-pass-per-pair
design does not have.  With exact sums nothing in a run depends on the order
in which pairs are visited, so the two complete runs - elastic loading, bond
breakage, Hertz-Mindlin contacts of broken and new pairs, contact-list
rebuilds, the loading controller, fracture and the post-peak record - must be
the same bit for bit: the same number of steps, the same stress-strain and
lateral records, and so the same uniaxial compressive strength, strain at
peak, Young's modulus, Poisson ratio and Brazilian tensile strength.

Five seeds each of (and the FP64 build on three of the physics cases):
* the configurations' physics: polydisperse radii U[0.20, 0.30] mm (4 x 8 mm
  cylinders, 30% post-peak stress drop) and U[0.18, 0.30] mm (6 x 3 mm
  discs, to the Brazilian controller's fracture), bond modulus 30 GPa, kn/ks
  2.5, bond radius 0.8 min r, per-bond strengths N(40, 8) MPa;
* reference-mode specimens (equal 0.25 mm spheres on a jittered FCC lattice,
  scalar 40 MPa strengths, the reference's monodisperse formulas in the
  oracle): the specimens the reference's own drivers run in
  test_gpu_macro.py.
"""
from __future__ import annotations

import importlib

import numpy as np
import pytest

import dem_testlib as T
from dem_api import dem
from oracle import drive
from oracle import physics as PH
from oracle import sim
from test_gpu_dynamics import LSI, SPACE
from test_gpu_parity import _loading, _material

pytestmark = pytest.mark.gpu

W = importlib.import_module("dem-rock-calibration_b200.workloads")
SEEDS = (1, 2, 3, 4, 5)
PK = dict(growth_stages=20, steps_per_stage=150, max_fire_steps=4000)


def _engine(mat, ld, xyz, radii=None, precision=0):
    fp64 = precision == 1
    ctx = dem.Context(deterministic=True, precision=precision)
    sid = ctx.add_sample(mat, ld, xyz, radii)
    ctx.setup()
    init = (ctx.particles(sid, double=fp64), ctx.pairs(sid, double=fp64), ctx.result(sid))
    ctx.run(10 ** 7)
    res = ctx.result(sid)
    rec, _ = ctx.record(sid)
    lat = ctx.lateral_record(sid)
    ctx.close()
    # (a contact list that went stale inside a chunk holds its sample until the
    # list is rebuilt, so res["stale"] > 0 changes nothing in the run)
    assert res["done"] and not res["numeric"]
    return init, res, rec, lat


def _oracle(st, sc, ld, dt, p_r, lateral=None, axis_center=None, **kw):
    """p_r: the sphere radius of the platen set-up (the uniaxial test's
    loaded area is pi (size/2 + p_r)^2, md_data_types.h:227-228)."""
    return drive.loading_run(st, sc, brazil=ld.test == dem.TEST_BRAZIL, size_real=list(ld.size_real),
                             center_real=list(ld.center_real), p_r=p_r, min_stress=ld.min_stress,
                             max_strain=ld.max_strain, cond_fracture=ld.cond_fracture, velocity=ld.velocity, dt=dt,
                             dNsave=ld.dNsave, max_steps=10 ** 7, fixsum=True, lateral=lateral,
                             axis_center=axis_center, **kw)


def _same(name, res, rec, o, lat=None):
    """Identical runs: step count, records, controller results."""
    print(f"{name}: {res['steps']} steps ({res['rebuilds']} list builds, {res['stale']} stale), "
          f"bonds {res['bonds_initial']} -> {res['bonds_now']}, "
          f"strength {res['FractureStress'] * 1e3:.6g} MPa at strain {res['FractureStrain']:.6g}; "
          f"oracle {o['steps']} steps, {o['FractureStress'] * 1e3:.6g} MPa at {o['FractureStrain']:.6g}")
    assert res["steps"] == o["steps"]
    assert rec.shape == o["rec"].shape and np.array_equal(rec, o["rec"])
    assert res["FractureStress"] == o["FractureStress"] and res["FractureStrain"] == o["FractureStrain"]
    # the run went through failure: at least 5% of the bonds broke
    assert res["bonds_now"] < 0.95 * res["bonds_initial"]
    if lat is not None:
        assert np.array_equal(lat, o["lat"])


def _physics(kind, seed):
    if kind == "uniaxial":
        sp = W.uniaxial_cylinder(seed=seed, diameter=4.0, height=8.0, pack_kw=PK)
    else:
        sp = W.brazilian_disc(seed=seed, diameter=6.0, thickness=3.0, velocity_m_s=0.1, pack_kw=PK)
    mat = dem.Material.from_buffer_copy(sp.material)
    ld = dem.Loading.from_buffer_copy(sp.loading)
    if kind == "uniaxial":
        ld.cond_fracture = 0.7       # to a 30% stress drop after the peak
    return sp, mat, ld


def _physics_runs_are_identical(kind, seed, precision):
    sp, mat, ld = _physics(kind, seed)
    (p0, pr0, r0), res, rec, lat = _engine(mat, ld, sp.xyz, sp.radii, precision)
    pc = PH.physics_case(mat, ld, sp.radii, dt=r0["dt"], dtype=np.float64 if precision == 1 else np.float32)
    # the oracle starts from the engine's bonded state (the bond set and 1/L0
    # are pinned separately, test_gpu_physics_parity.py)
    st, sbr, ssn, sst = PH.ref_state_from_pairs(p0["R"], p0["V"], p0["W"], p0["Oiwt"], pr0, pc)
    lateral = axis = None
    if kind == "uniaxial":
        lateral = drive.lateral_spheres(sp.xyz, sp.radii.astype(np.float64), ld.center_real, ld.size_real,
                                        float(np.mean(sp.radii.astype(np.float64))))
        axis = np.float32(np.array(ld.center_real[:2])).astype(np.float64)
    o = _oracle(st, pc.sc, ld, r0["dt"], ld.p_r_platen, lateral, axis, **pc.kw(sbr, ssn, sst))
    _same(f"\n{kind} seed {seed} ({sp.n} spheres, {'FP64' if precision == 1 else 'FP32'})", res, rec, o,
          lat if kind == "uniaxial" else None)
    if kind == "uniaxial":
        E_e, nu_e = drive.chord_moduli(rec, lat)
        E_o, nu_o = drive.chord_moduli(o["rec"], o["lat"])
        assert E_e == E_o and nu_e == nu_o and E_e == pytest.approx(res["E_chord"], rel=1e-12)
        print(f"  E {E_e:.6g} GPa, nu {nu_e:.6g} (both)")


@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("kind", ["uniaxial", "brazilian"])
def test_configuration_physics_runs_are_identical(kind, seed):
    _physics_runs_are_identical(kind, seed, 0)


@pytest.mark.parametrize("kind,seed", [("uniaxial", 1), ("uniaxial", 2), ("brazilian", 2)])
def test_fp64_runs_are_identical(kind, seed):
    """The FP64 build (double state and arithmetic, pair sums in 2^-50 fixed
    point) against the oracle's double path with the same sums."""
    _physics_runs_are_identical(kind, seed, 1)


def _ref_specimen(kind, seed):
    if kind == "uniaxial":
        c = T.ref_case(seed=seed, lsi=LSI, space=SPACE, jitter_frac=0.1, lattice_gap=0.5, Ec=40e6, Gc=40e6,
                       condfract=0.7)
    else:
        c = T.ref_case(seed=seed, lsi=(0.006, 0.006, 0.003), space=(0.012, 0.012, 0.006), jitter_frac=0.1,
                       lattice_gap=0.5, Ec=40e6, Gc=40e6, brazil=True, minstress_si=1e6, maxstrain=0.015)
    ld = _loading(c)
    ld.dNsave = 50
    return c, ld


@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("kind", ["uniaxial", "brazilian"])
def test_reference_mode_runs_are_identical(kind, seed):
    c, ld = _ref_specimen(kind, seed)
    (p0, pr0, r0), res, rec, _ = _engine(_material(c), ld, c.R)
    st = sim.RefState.empty(c.N)
    st.R[:] = c.R
    sim.oracle_setup_bonds(st, c.sc)
    assert int(np.sum((st.ILtype == 1) & (st.IL != 0xFFFFFFFF))) == 2 * r0["bonds_initial"]
    o = _oracle(st, c.sc, ld, r0["dt"], c.pot.p_r)
    _same(f"\nreference-mode {kind} seed {seed} ({c.N} spheres)", res, rec, o)
