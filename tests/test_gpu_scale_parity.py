"""Parity with the reference's own CUDA kernels at the configurations' sizes.

Two reference-mode specimens (equal radii 0.25 mm on a jittered FCC lattice
spaced 2 r + gap/2, scalar micro-parameters, so the reference kernels run
them unchanged; compiled from the reference sources into oracle/_ref):

* the Brazilian disc 40 mm x 20 mm (about 2.5e5 spheres), the size of the
  Brazilian configuration;
* the uniaxial cylinder 8 mm x 16 mm (about 8e3 spheres), the size of the
  plain uniaxial configuration.

For each, against the reference (md_cell_distribution.cu:130-172,
md_interaction_list_construct.cu:204-317, md_boundinteractions_construct.cu:35-106,
and one pass of the loading loop body, md_calculationbraziltest.cu:185-231 /
md_calculationuniaxialcompression.cu:265-314):

* cell lists (CI, CIs, pnC): bit-exact;
* interaction sets of every sphere: identical;
* bond set: identical;
* one step from a perturbed state of the same bonded specimen: forces and
  moments within the reference-test tolerance (1e-5 of the per-particle sum
  of |contributions| plus the distance-rounding term, oracle/sim.py
  StepOut.f_tol), bond-break topology identical, velocities, positions and
  spins within the force tolerance carried through the integration.

The worst error as a fraction of its tolerance is printed (pytest -s).
"""
from __future__ import annotations

import numpy as np
import pytest

import dem_testlib as T
from dem_api import dem
from oracle import lib as L
from oracle import sim
from test_gpu_parity import _loading, _material

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not L.ref_available(), reason="reference harness not built")]

SPECIMENS = {
    "brazilian_disc_40x20": dict(seed=4, lsi=(0.040, 0.040, 0.020), space=(0.052, 0.052, 0.030), jitter_frac=0.1,
                                 lattice_gap=0.5, brazil=True, velocity_si=-0.02, minstress_si=2.1e6, maxstrain=0.03),
    "uniaxial_cylinder_8x16": dict(seed=5, lsi=(0.008, 0.008, 0.016), space=(0.0104, 0.0104, 0.024),
                                   jitter_frac=0.1, lattice_gap=0.5),
}


def _keys(i, j, n):
    return np.asarray(i, np.int64) * n + np.asarray(j, np.int64)


def _ref_bond_keys(IL, ILtype, n, P):
    M = IL.reshape(n, P)
    t = ILtype.reshape(n, P)
    r, c = np.nonzero((M != L.EMPTY) & (t == 1))
    j = M[r, c].astype(np.int64)
    keep = r < j
    return np.sort(_keys(r[keep], j[keep], n)), (r * P + c)[keep][np.argsort(_keys(r[keep], j[keep], n))]


@pytest.mark.parametrize("name", list(SPECIMENS))
def test_reference_kernels_parity_at_configuration_size(name):
    c = T.ref_case(**SPECIMENS[name])
    n, P = c.N, 32
    cells = (c.cells.a, c.cells.nx, c.cells.ny, c.cells.nz)
    # cell lists
    got = dem.ref_cells(c.R, *cells)
    want = sim.ref_cells(c.R, n, c.sc)
    for g, w, what in zip(got, want, ("CI", "CIs", "pnC")):
        assert np.array_equal(g, w), what
    # reference set-up: cells, interaction list, bonds, far-link deletion
    st = sim.RefState.empty(n)
    st.R[:] = c.R
    sim.ref_setup_bonds(st, c.sc)
    # interaction sets: the reference's rows sorted, against the engine's sorted sets
    sets, ovf = dem.ref_neighbor_sets(c.R, *cells, c.sc.il_aacut, c.sc.aa_farcut, P)
    assert ovf == 0
    assert np.array_equal(sets, np.sort(st.IL.reshape(n, P), axis=1))
    # bonds
    ctx = dem.Context()
    sid = ctx.add_sample(_material(c), _loading(c), c.R)
    ctx.setup()
    pr = ctx.pairs(sid)
    b = pr["kind"] == 1
    ref_keys, ref_slots = _ref_bond_keys(st.IL, st.ILtype, n, P)
    eng_keys = np.sort(_keys(pr["i"][b], pr["j"][b], n))
    assert np.array_equal(eng_keys, ref_keys)
    assert ref_keys.size > 5 * n
    # one step from a perturbed state: positions, velocities and spins
    rng = np.random.default_rng(9)
    T.perturb(st, rng, dx=1e-4, v=1e-4, w=1e-3)
    top, bot = float(np.float32(c.sc.wall_top - 0.002)), float(np.float32(c.sc.wall_bot + 0.002))
    c.sc.wall_top, c.sc.wall_bot = top, bot
    ctx.set_particles(sid, R=st.R, V=st.V, W=st.W)
    ctx.set_platens(sid, top, bot, c.sc.wall_V)
    st_in = st.copy()
    # the oracle steps the same state with its own bond lengths (1/L0 = rsqrt(r^2)
    # correctly rounded, as the engine computes them; the reference's FMA-contracted
    # r^2 may differ by an ulp or two, which the bond strain amplifies)
    own = sim.RefState.empty(n)
    own.R[:] = c.R
    sim.oracle_setup_bonds(own, c.sc)
    assert np.array_equal(own.IL, st.IL)
    orc = st.copy()
    orc.invL0[:] = own.invL0
    out = sim.oracle_step(orc, c.sc, want_abs=True)      # tolerance scales (and a third opinion)
    ref = st.copy()
    sim.ref_step(ref, c.sc)
    ctx.step_stages(dem.STAGE_PAIRS | dem.STAGE_PARTICLES | dem.STAGE_KEEP_FORCES)
    p = ctx.particles(sid)
    ftol = out.f_tol(ref.F) + 1e-12
    mtol = out.m_tol(ref.M) + 1e-15
    eF = np.abs(p["F"] - ref.F) / ftol
    eM = np.abs(p["M"] - ref.M) / mtol
    print(f"\n{name}: {n} spheres, {ref_keys.size} bonds; worst |dF|/tol {eF.max():.3g}, |dM|/tol {eM.max():.3g} "
          f"against the reference kernels")
    assert np.all(eF <= 1.0), float(eF.max())
    assert np.all(eM <= 1.0), float(eM.max())
    # against the oracle only the summation order differs
    fs = 1e-5 * (out.Fabs + np.abs(orc.F)) + 1e-12
    assert np.all(np.abs(p["F"] - orc.F) <= fs)
    # bond-break topology after the step
    pr2 = ctx.pairs(sid)
    b2 = pr2["kind"] == 1
    ref_keys2, _ = _ref_bond_keys(ref.IL, ref.ILtype, n, P)
    assert np.array_equal(np.sort(_keys(pr2["i"][b2], pr2["j"][b2], n)), ref_keys2)
    # kinematics after the step
    tolV = out.f_tol(ref.F) * c.sc.dt_d_m + 1e-5 * (np.abs(st_in.V) + np.abs(ref.V)) + 1e-12
    tolW = out.m_tol(ref.M) * c.sc.dt_d_I + 1e-5 * (np.abs(st_in.W) + np.abs(ref.W)) + 1e-12
    tolR = tolV * c.sc.dt + 2 * np.spacing(np.abs(ref.R))     # two ulp of the coordinates themselves
    for k, tol in (("V", tolV), ("R", tolR), ("W", tolW)):
        assert np.all(np.abs(p[k] - getattr(ref, k)) <= tol), k
    ctx.close()
