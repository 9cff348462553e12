"""Per-step parity of the engine with the CPU oracle on the configurations'
own physics, in FP32 (float atomics and deterministic sums) and in the FP64
build.

The configurations run polydisperse specimens (radii U[0.20, 0.30] mm or
U[0.18, 0.30] mm), a bond modulus (30 GPa) and kn/ks (2.5) of their own
beside the particle modulus (50 GPa), bond radius 0.8 min(r_i, r_j), bonds
for gaps below 0.1 r_min, and per-bond normal and shear strengths drawn from
N(40, 8) MPa.  The reference kernels are monodisperse with scalar strengths
(md_calculateforcesdem3.cu:20-486), so the oracle's physics mode
(oracle/physics.py: per-sphere radii and masses, per-slot bond radius and
strengths, the polydisperse Hertz-Mindlin form that reduces to the
reference's when radii are equal) is the checker here.

For each specimen the engine and the oracle build bonds from the same
positions (bond set exact, 1/L0 bit-exact, bond radius and strengths as the
law gives them); then, from a perturbed state, the engine advances step by
step and before every step its full state (spheres and pair table) is
loaded into the oracle, which advances the same step:

* bond and contact histories after the step: bit-exact (the same operation
  order and rounding; only the force sums differ in order);
* bond-break decisions: identical;
* forces and moments of the step: within 1e-5 (FP32) / 1e-12 (FP64) of the
  per-particle sum of |contributions| (deterministic FP32 sums add the
  fixed-point quantum, 2^-36 kN or kN mm);
* positions, velocities and spins after the step: the force tolerance
  carried through the integration.

Cases: a uniaxial cylinder and a Brazilian disc whose bonds break under the
perturbation (bonds, breaks, and the Hertz-Mindlin contacts of broken
touching pairs, platens), and a cylinder with no bonds (every touching pair a
Hertz-Mindlin contact, with Coulomb slip and rolling friction).
"""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from dem_api import dem
from oracle import lib as L
from oracle import physics as PH
from oracle import sim

pytestmark = pytest.mark.gpu

W = importlib.import_module("dem-rock-calibration_b200.workloads")
STAGES = dem.STAGE_PAIRS | dem.STAGE_PARTICLES | dem.STAGE_KEEP_FORCES
RTOL = {0: 1e-5, 1: 1e-12}
_SPECIMENS = {}


def _specimen(name):
    if name not in _SPECIMENS:
        pk = dict(growth_stages=20, steps_per_stage=150, max_fire_steps=4000)
        if name == "brazilian":
            sp = W.brazilian_disc(seed=4, diameter=6.0, thickness=3.0, pack_kw=pk)
        else:
            sp = W.uniaxial_cylinder(seed=3, diameter=4.0, height=8.0, pack_kw=pk)
        _SPECIMENS[name] = sp
    return _SPECIMENS[name]


CASES = {
    # name: (specimen, material overrides, displacement / velocity / spin perturbation)
    "uniaxial_bonds": ("uniaxial", {}, (6e-4, 2e-4, 2e-3)),
    "brazilian_bonds": ("brazilian", {}, (6e-4, 2e-4, 2e-3)),
    "uniaxial_contacts": ("uniaxial", {"gap": -1.0}, (3e-3, 5e-4, 5e-3)),
}
# precision, deterministic sums, pair-kernel register budget (0: the default)
MODES = {"fp32": (0, False, 0), "fp32_det": (0, True, 0), "fp64": (1, False, 0)}


def _engine(sp, mat, precision, det, pair_min_blocks=0):
    ctx = dem.Context(precision=precision, deterministic=det, pair_min_blocks=pair_min_blocks)
    sid = ctx.add_sample(mat, sp.loading, sp.xyz, sp.radii)
    ctx.setup()
    return ctx, sid


def _oracle_bonds(pc, xyz, mat):
    n = xyz.size // 3
    st = sim.RefState.empty(n, IonP=pc.IonP, dtype=pc.dtype)
    st.R[:] = xyz
    ov = sim.oracle_setup_bonds(st, pc.sc, rad=pc.rad, gap=mat.gap)
    assert ov == 0
    IL = st.IL.reshape(n, pc.IonP)
    ty = st.ILtype.reshape(n, pc.IonP)
    r, c = np.nonzero((IL != L.EMPTY) & (ty == 1))
    j = IL[r, c]
    keep = r < j
    slots = (r * pc.IonP + c)[keep]
    return {(int(a), int(b)): float(st.invL0[s]) for a, b, s in zip(r[keep], j[keep], slots)}


def _slot_table(st: sim.RefState):
    """oracle slots i -> j with i < j: {(i, j): (type, 12 history values)}."""
    n, P = st.N, st.IonP
    IL = st.IL.reshape(n, P)
    r, c = np.nonzero(IL != L.EMPTY)
    j = IL[r, c]
    keep = r < j
    r, c, j = r[keep], c[keep], j[keep]
    s = r * P + c
    hist = np.concatenate([st.Rij.reshape(-1, 3)[s], st.Oijt.reshape(-1, 3)[s], st.Mijn.reshape(-1, 3)[s],
                           st.Mijt.reshape(-1, 3)[s]], axis=1)
    return {(int(a), int(b)): (int(t), h) for a, b, t, h in zip(r, j, st.ILtype[s], hist)}


def _compare_pairs(pr, st: sim.RefState):
    """Engine pair table after a step against the oracle's slots: bit-exact
    histories, identical bond states.  Returns (intact, broken, touching contacts)."""
    tab = _slot_table(st)
    counts = [0, 0, 0]
    seen = set()
    for i, j, k, s in zip(pr["i"], pr["j"], pr["kind"], pr["state"]):
        key = (int(i), int(j))
        assert key in tab, key
        t, h = tab[key]
        seen.add(key)
        if k == 1:
            assert t == 1, (key, "intact in the engine, broken in the oracle")
            assert np.array_equal(s[1:13], h), (key, s[1:13], h)
            counts[0] += 1
        else:
            assert t == 0, (key, "broken in the engine, intact in the oracle")
            assert np.array_equal(s[4:7], h[3:6]), (key, s[4:7], h[3:6])
            if k == 2:
                counts[1] += 1
            if np.any(h[3:6]):
                counts[2] += 1
    for key, (t, h) in tab.items():
        if key not in seen:
            assert t == 0 and not np.any(h[3:6]), (key, "pair with state missing from the engine")
    return counts


@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("case", list(CASES))
def test_steps_match_oracle_physics_mode(case, mode):
    precision, det, pmb = MODES[mode]
    name, over, (dx, dv, dw) = CASES[case]
    sp = _specimen(name)
    mat = dem.Material.from_buffer_copy(sp.material)
    for k, v in over.items():
        setattr(mat, k, v)
    dtype = np.float64 if precision == 1 else np.float32
    fp64 = precision == 1
    ctx, sid = _engine(sp, mat, precision, det, pmb)
    n = sp.n
    res = ctx.result(sid)
    assert res["dt"] == pytest.approx(PH.time_step(mat, sp.radii), rel=1e-15)
    pc = PH.physics_case(mat, sp.loading, sp.radii, dt=res["dt"], dtype=dtype)
    # bonds from the same positions: same set, 1/L0 bit-exact, law-given radius and strengths
    pr = ctx.pairs(sid, double=fp64)
    bonds = pr["kind"] == 1
    want = _oracle_bonds(pc, sp.xyz, mat)
    got = {(int(a), int(b)): s for a, b, s in zip(pr["i"][bonds], pr["j"][bonds], pr["state"][bonds])}
    assert set(got) == set(want)
    if over.get("gap", 0) >= 0:
        assert len(got) > n
    for key, s in got.items():
        assert s[0] == want[key], key
    if got:
        st_b = np.array(list(got.values()))
        ij = np.array(list(got.keys()), np.int64)
        rad = sp.radii.astype(dtype)
        br = dtype(mat.bond_radius_factor) * np.minimum(rad[ij[:, 0]], rad[ij[:, 1]])
        assert np.array_equal(st_b[:, 15], br.astype(dtype))
        sn, stt = PH.bond_strengths(mat, ij[:, 0], ij[:, 1], dtype)
        np.testing.assert_allclose(st_b[:, 13], sn, rtol=4 * np.finfo(dtype).eps)
        np.testing.assert_allclose(st_b[:, 14], stt, rtol=4 * np.finfo(dtype).eps)
        assert abs(np.mean(st_b[:, 13]) - mat.Ec) < 0.1 * mat.Ec and abs(np.std(st_b[:, 13]) - mat.Ec_sd) < 0.2 * \
            mat.Ec_sd
    # perturbed state (float32 values, exact in both precisions); platens 2 um inside the specimen
    rng = np.random.default_rng(17)
    R = (sp.xyz + rng.normal(0.0, dx, 3 * n)).astype(np.float32)
    V = rng.normal(0.0, dv, 3 * n).astype(np.float32)
    Wv = rng.normal(0.0, dw, 3 * n).astype(np.float32)
    ctx.set_particles(sid, R=R, V=V, W=Wv)
    ax = 1 if sp.loading.test == dem.TEST_BRAZIL else 2
    top = float(np.float32(sp.loading.center_real[ax] + 0.5 * sp.loading.size_real[ax] - 0.002))
    bot = float(np.float32(sp.loading.center_real[ax] - 0.5 * sp.loading.size_real[ax] + 0.002))
    ctx.set_platens(sid, top, bot, float(np.float32(sp.loading.velocity)))
    rtol = RTOL[precision]
    totals = np.zeros(3, np.int64)
    breaks = 0
    worst = 0.0
    for step in range(4):
        p = ctx.particles(sid, double=fp64)
        pr = ctx.pairs(sid, double=fp64)
        r = ctx.result(sid)
        st, slot_br, slot_sn, slot_st = PH.ref_state_from_pairs(p["R"], p["V"], p["W"], p["Oiwt"], pr, pc)
        intact_before = int(np.sum(pr["kind"] == 1))
        pc.sc.wall_top = float(np.float32(r["platen_top"]))
        pc.sc.wall_bot = float(np.float32(r["platen_bottom"]))
        pc.sc.wall_V = float(np.float32(r["platen_velocity"]))
        st_in = st.copy()
        out = sim.oracle_step(st, pc.sc, sim.STAGE_ALL, want_abs=True, **pc.kw(slot_br, slot_sn, slot_st))
        assert out.overflow == 0
        ctx.step_stages(STAGES)
        q = ctx.particles(sid, double=fp64)
        pr2 = ctx.pairs(sid, double=fp64)
        counts = _compare_pairs(pr2, st)
        totals += counts
        breaks += intact_before - counts[0]
        # deterministic sums carry every contribution in 2^-40 fixed point: a
        # rounding of up to 2^-41 per contribution (about 16 per sphere)
        quantum = 2.0 ** -36 if det else 1e-30
        fs = rtol * (out.Fabs + np.abs(st.F)) + quantum
        ms = rtol * (out.Mabs + np.abs(st.M)) + quantum
        eF = np.abs(q["F"] - st.F) / fs
        eM = np.abs(q["M"] - st.M) / ms
        worst = max(worst, float(eF.max()), float(eM.max()))
        assert np.all(eF <= 1.0), (step, float(eF.max()))
        assert np.all(eM <= 1.0), (step, float(eM.max()))
        dtm = pc.dtm[np.tile(np.arange(n), 3)]
        dtI = pc.dtI[np.tile(np.arange(n), 3)]
        eps = np.finfo(dtype).eps
        tolV = fs * dtm + 2 * eps * (np.abs(st_in.V) + np.abs(st.V)) + 1e-30
        tolR = tolV * pc.sc.dt + 2 * eps * np.abs(st.R)
        tolW = ms * dtI + 2 * eps * (np.abs(st_in.W) + np.abs(st.W)) + 1e-30
        for key, tol in (("V", tolV), ("R", tolR), ("W", tolW)):
            assert np.all(np.abs(q[key] - getattr(st, key)) <= tol), (step, key)
    print(f"\n{case}/{mode}: {n} spheres, intact {totals[0] // 4}, breaks {breaks}, "
          f"touching contacts {totals[2]} over 4 steps, worst |dF|,|dM| / tolerance {worst:.3g}")
    if case.endswith("bonds"):
        assert breaks > 0
    else:
        assert totals[2] > 0
    ctx.close()
