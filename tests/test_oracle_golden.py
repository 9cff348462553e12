"""Pin the CPU oracle to the reference's OWN CUDA kernels.

The fixtures in tests/golden/ were produced by tests/golden/make_golden.py,
which runs the reference kernels (compiled from the reference sources into
oracle/_ref/) on a B200.  Here the oracle replays the same inputs on the CPU:

* cell lists and interaction lists must agree bit for bit, slot for slot;
* bond creation (type, 1/L0) and bond-break topology must agree exactly;
* forces, moments and histories must agree within 1e-5 relative, measured
  against the sum of |contributions| of each particle (the reference
  contracts a*b+c into FMAs, the oracle rounds each operation), plus, for
  forces, the forward error of 6 ulp in each pair distance through the bond
  normal stiffness: the reference's norm3df is not correctly rounded, the
  oracle's norm is, and the bond strain (r - L0)/L0 amplifies one ulp of r
  by 1/strain.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import dem_testlib as T
from oracle import lib as L
from oracle import sim

GOLD = Path(__file__).resolve().parent / "golden"
SMALL = dict(lsi=(0.0035, 0.0035, 0.005), space=(0.008, 0.008, 0.011))
# make_golden.py STEP_CASES (case kwargs only)
CASES = {
    "u_plain": dict(seed=11),
    "b_plain": dict(seed=12, brazil=True),
    "u_break": dict(seed=13),
    "u_contact": dict(seed=14, gap_si=-0.01e-3, jitter_frac=0.05),
}
RTOL = 1e-5


def load(name):
    return dict(np.load(GOLD / f"{name}.npz"))


@pytest.mark.parametrize("seed", [1, 2])
def test_cells_and_il_bit_exact(seed):
    g = load(f"cells_il_s{seed}")
    c = T.ref_case(seed=seed, **SMALL)
    assert np.array_equal(c.R, g["R"]), "the seeded specimen must be reproducible"
    CI, CIs, pnC = sim.oracle_cells(c.R, c.N, c.sc)
    assert np.array_equal(CI, g["CI"])
    assert np.array_equal(CIs, g["CIs"])
    assert np.array_equal(pnC, g["pnC"])
    st = sim.RefState.empty(c.N)
    st.R[:] = c.R
    ov = sim.oracle_setup_bonds(st, c.sc)
    assert ov == 0
    # slot-exact interaction list and bond flags
    assert np.array_equal(st.IL, g["IL"])
    used = st.IL != L.EMPTY
    assert np.array_equal(st.ILtype[used], g["ILtype"][used])
    # 1/L0 = rsqrt(r^2): the reference may fuse r^2 into FMAs; allow 2 ulp
    b = used & (st.ILtype == 1)
    a, r = st.invL0[b], g["invL0"][b]
    ulp = np.abs(a.view(np.int32).astype(np.int64) - r.view(np.int32).astype(np.int64))
    assert ulp.max() <= 2, ulp.max()


def _case(name):
    c = T.ref_case(**SMALL, **CASES[name])
    g = load(f"step_{name}")
    c.sc.wall_top = float(g["wall_top"])
    c.sc.wall_bot = float(g["wall_bot"])
    return c, g


def _close(a, b, scale, rtol=RTOL, floor=1e-30):
    err = np.abs(a.astype(np.float64) - b.astype(np.float64))
    lim = rtol * (np.abs(scale.astype(np.float64)) + floor)
    return err <= lim, err, lim


@pytest.mark.parametrize("name", list(CASES))
def test_step_matches_reference(name):
    c, g = _case(name)
    st = sim.RefState.from_dict(g, "in_")
    ref = sim.RefState.from_dict(g, "out_")
    out = sim.oracle_step(st, c.sc, want_abs=True)
    assert out.overflow == 0
    # topology: interaction list (slot for slot) and bond-break decisions exact
    assert np.array_equal(st.IL, ref.IL)
    used = st.IL != L.EMPTY
    assert np.array_equal(st.ILtype[used], ref.ILtype[used])
    # forces and moments after the increments stage are the pre-integration
    # values (the reference integrates from the same F/M), compared per component
    # against the per-particle sum of |contributions| (plus the platen force)
    err = np.abs(st.F.astype(np.float64) - ref.F)
    lim = out.f_tol(ref.F)
    assert (err <= lim).all(), f"F worst {np.max(err / lim):.3g} of tolerance"
    err = np.abs(st.M.astype(np.float64) - ref.M)
    lim = out.m_tol(ref.M)
    assert (err <= lim).all(), f"M worst {np.max(err / lim):.3g} of tolerance"
    # platen sums
    assert np.allclose(out.sFL, g["sFL"], rtol=1e-5, atol=1e-12)
    # kinematics after one step: the force/moment tolerances carried through
    # v += F dt/m, x += v dt, w += M dt/I, plus rtol of the values themselves
    st_in = sim.RefState.from_dict(g, "in_")
    tolV = out.f_tol(ref.F) * c.sc.dt_d_m + RTOL * (np.abs(st_in.V) + np.abs(ref.V))
    tolW = out.m_tol(ref.M) * c.sc.dt_d_I + RTOL * (np.abs(st_in.W) + np.abs(ref.W))
    tolR = tolV * c.sc.dt + RTOL * np.abs(ref.R) * 1e-2
    for k, tol in (("V", tolV), ("W", tolW), ("R", tolR)):
        err = np.abs(getattr(st, k).astype(np.float64) - getattr(ref, k))
        assert (err <= tol + 1e-30).all(), f"{k} worst {np.max(err / (tol + 1e-30)):.3g}"
    # per-slot histories of live slots.  Contact (type 0) histories in Coulomb
    # slip are proportional to the overlap d = 2 r_p - r, so a distance ulp
    # enters relative to d: their tolerance adds DIST_ULPS * ulp(r) / d.
    N, IonP = st.N, st.IonP
    Rin = st_in.R.reshape(3, N).astype(np.float64)
    ii = np.repeat(np.arange(N), IonP)
    jj = np.where(used, st.IL, 0).astype(np.int64)
    r = np.linalg.norm(Rin[:, jj] - Rin[:, ii], axis=0)
    overlap = np.maximum(2.0 * c.sc.p_r - r, 1e-12)
    ulp_r = np.spacing(r.astype(np.float32)).astype(np.float64)
    hm = used & (st.ILtype == 0)
    extra = np.where(hm, sim.DIST_ULPS * ulp_r / overlap, 0.0)
    for k in ("Rij", "Oijt", "Mijn", "Mijt"):
        a = getattr(st, k).reshape(-1, 3).astype(np.float64)
        b = getattr(ref, k).reshape(-1, 3).astype(np.float64)
        mag = np.abs(b).max(1)
        floor = np.abs(b[used]).max() * 1e-3 if used.any() else 0.0
        tol = (1e-4 + extra) * np.maximum(mag, floor) + 1e-30
        err = np.abs(a - b).max(1)
        bad = used & (err > tol)
        assert not bad.any(), f"{k}: {int(bad.sum())} slots, worst {np.max(err[used] / tol[used]):.3g}"


def test_rsqrt_rn_is_correctly_rounded():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(1e-3, 4.0, 20000), rng.uniform(1e-12, 1e6, 20000)]).astype(np.float32)
    f = L.lib().orc_rsqrt_rn_f
    for x in xs[:4000]:
        y = np.float32(f(float(x)))
        exact = 1.0 / np.sqrt(np.float64(x))  # close to exact; correct rounding lies within 0.5 ulp
        ulp = np.spacing(y)
        assert abs(np.float64(y) - exact) <= 0.5 * np.float64(ulp) * (1 + 1e-6)


def _shuffle_slots(st: sim.RefState, rng) -> sim.RefState:
    """The same state with every particle's interaction-list slots in another
    order (each slot's partner, type, 1/L0 and histories move together)."""
    s = st.copy()
    N, P = st.N, st.IonP
    perm = np.argsort(rng.random((N, P)), axis=1)
    src = (np.arange(N)[:, None] * P + perm).reshape(-1)
    for k in ("IL", "ILtype", "invL0"):
        getattr(s, k)[:] = getattr(st, k)[src]
    for k in ("Rij", "Oijt", "Mijn", "Mijt"):
        getattr(s, k)[:] = getattr(st, k).reshape(-1, 3)[src].reshape(-1)
    return s


@pytest.mark.parametrize("name", list(CASES))
def test_fixed_point_sums_change_only_the_summation(name):
    """oracle_step(fixsum=True), the sums of the engine's deterministic mode:
    the same step as the reference's running float sums up to the rounding of
    the sums (topology and histories identical, forces, moments and platen
    sums within the reordering tolerance), and a result that does not depend
    on the order of a particle's slots (bit for bit after shuffling them)."""
    c, g = _case(name)
    stages = sim.STAGE_FORCES | sim.STAGE_PLATEN | sim.STAGE_INCR
    a = sim.RefState.from_dict(g, "in_")
    b = a.copy()
    out_a = sim.oracle_step(a, c.sc, stages, want_abs=True)
    out_b = sim.oracle_step(b, c.sc, stages, fixsum=True)
    used = a.IL != L.EMPTY
    assert np.array_equal(a.ILtype[used], b.ILtype[used])
    for k in ("Rij", "Oijt", "Mijn", "Mijt"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert (np.abs(a.F.astype(np.float64) - b.F) <= out_a.f_tol(a.F)).all()
    assert (np.abs(a.M.astype(np.float64) - b.M) <= out_a.m_tol(a.M)).all()
    assert np.allclose(out_b.sFL, out_a.sFL, rtol=1e-5, atol=1e-12)
    # order independence: shuffled slots give the same bits
    s = _shuffle_slots(sim.RefState.from_dict(g, "in_"), np.random.default_rng(3))
    out_s = sim.oracle_step(s, c.sc, stages, fixsum=True)
    for k in ("F", "M", "V", "R", "W", "Oiwt"):
        assert np.array_equal(getattr(s, k), getattr(b, k)), k
    assert np.array_equal(out_s.sFL, out_b.sFL)


@pytest.mark.parametrize("name", ["u_break", "u_contact"])
def test_fixed_point_sums_are_order_independent_in_fp64(name):
    """The FP64 path of the fixed-point sums (2^-50 resolution): the same
    step from the same state with every particle's slots shuffled gives the
    same bits."""
    c, g = _case(name)
    stages = sim.STAGE_FORCES | sim.STAGE_PLATEN | sim.STAGE_INCR
    base = sim.RefState.from_dict(g, "in_")
    d = sim.RefState(N=base.N, IonP=base.IonP, dtype=np.float64)
    for k in sim.RefState.ARRAYS:
        a = getattr(base, k)
        setattr(d, k, a.astype(np.float64) if a.dtype == np.float32 else a.copy())
    e = _shuffle_slots(d, np.random.default_rng(5))
    out_d = sim.oracle_step(d, c.sc, stages, fixsum=True)
    out_e = sim.oracle_step(e, c.sc, stages, fixsum=True)
    for k in ("F", "M", "V", "R", "W", "Oiwt"):
        assert np.array_equal(getattr(d, k), getattr(e, k)), k
    assert np.array_equal(out_d.sFL, out_e.sFL)
    assert np.abs(d.F).max() > 0


def test_fixed_point_whole_run_does_not_depend_on_slot_order():
    """A whole loading run of the oracle with exact sums (the mode the
    engine's deterministic runs are compared with, bit for bit, on the GPU):
    6,000 steps of a small reference-mode cylinder with weak (5 MPa) bonds, so
    that bonds break and broken pairs become Hertz-Mindlin contacts, the
    interaction list rebuilt every step.  Started once from the list as built
    and once with every particle's slots shuffled, the two runs give the same
    record, the same break topology and the same final state bit for bit."""
    from test_gpu_parity import _loading
    from oracle import drive

    c = T.ref_case(seed=3, **SMALL, Ec=5e6, Gc=5e6, condfract=0.7, jitter_frac=0.1, lattice_gap=0.5)
    ld = _loading(c)
    st = sim.RefState.empty(c.N)
    st.R[:] = c.R
    sim.oracle_setup_bonds(st, c.sc)
    bonds0 = int(np.sum((st.ILtype == 1) & (st.IL != L.EMPTY)))
    runs = []
    for s in (st.copy(), _shuffle_slots(st, np.random.default_rng(11))):
        o = drive.loading_run(s, c.sc, brazil=False, size_real=list(ld.size_real), center_real=list(ld.center_real),
                              p_r=c.pot.p_r, min_stress=ld.min_stress, max_strain=ld.max_strain,
                              cond_fracture=ld.cond_fracture, velocity=ld.velocity, dt=float(np.float32(c.sc.dt)),
                              dNsave=50, max_steps=6000, fixsum=True)
        bonds = int(np.sum((s.ILtype == 1) & (s.IL != L.EMPTY)))
        runs.append((o, s, bonds))
    (oa, sa, ba), (ob, sb, bb) = runs
    assert ba == bb and ba < bonds0 - 100          # the same breaks, and many of them
    assert oa["steps"] == ob["steps"] == 6000
    assert np.array_equal(oa["rec"], ob["rec"]) and oa["FractureStress"] == ob["FractureStress"]
    for k in ("R", "V", "W", "Oiwt"):
        assert np.array_equal(getattr(sa, k), getattr(sb, k)), k
