"""Reference-layout simulation state and the loading-step drivers used by the
parity tests (test infrastructure only).

`RefState` holds one specimen in the reference layout.  Two drivers advance
it through the same sequence of the reference hot loop
(md_calculationuniaxialcompression.cu:265-314, md_calculationbraziltest.cu:185-231):

* `oracle_*`  - the CPU restatement (oracle/_build/libdemoracle.so);
* `ref_*`     - the reference's own CUDA kernels (oracle/_ref/libdemref.so),
                usable only on a GPU box.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import lib as L
from . import params as prm

STAGE_IL, STAGE_FORCES, STAGE_PLATEN, STAGE_INCR, STAGE_CUT, STAGE_DELETE = 1, 2, 4, 8, 16, 32
STAGE_ALL = 63
# Pair distances computed by different norm routines (CUDA's norm3df against a
# correctly rounded norm) may differ by this many ulp; force tolerances carry
# that forward error through the normal stiffness (StepOut.Fsens).
DIST_ULPS = 6.0


@dataclass
class StepOut:
    sFL: np.ndarray          # platen force sums (bottom, top), double
    FL: np.ndarray           # per-64-block platen partials
    Fabs: np.ndarray = None  # per component: sum of |force contributions|
    Mabs: np.ndarray = None  # per component: sum of |moment contributions|
    Fsens: np.ndarray = None  # per particle: sum over pairs of normal stiffness * ulp(distance)
    overflow: int = 0

    def f_tol(self, F_ref: np.ndarray, rtol: float = 1e-5) -> np.ndarray:
        """Per-component force tolerance: rtol of the contribution scale plus the
        forward error of DIST_ULPS ulp in each pair distance."""
        return rtol * (self.Fabs + np.abs(F_ref)) + DIST_ULPS * np.tile(self.Fsens, 3)

    def m_tol(self, M_ref: np.ndarray, rtol: float = 1e-5) -> np.ndarray:
        return rtol * (self.Mabs + np.abs(M_ref))


@dataclass
class Scalars:
    """Float kernel arguments of one loading step (reference values)."""

    a: float
    inv_a: float
    nx: int
    ny: int
    nz: int
    IonP: int
    il_aacut: float
    aa_farcut: float
    dt: float
    m_E: float
    m_G: float
    b_r: float
    m_Ec: float
    m_Gc: float
    hm_E: float
    hm_G: float
    p_A: float
    p_mu: float
    p_mur: float
    p_m: float
    p_r: float
    wall_E: float
    wall_G: float
    center: np.ndarray
    wall_RR: float
    wall_top: float
    wall_bot: float
    wall_V: float
    Zcut: float
    dt_d_m: float
    dt_d_I: float
    s_center: np.ndarray
    s_spacesized2: np.ndarray
    hidenpoint: np.ndarray
    brazil: int
    b_dd: float = 0.0

    def to_c(self, stages: int) -> L.StepParams:
        p = L.StepParams()
        for k, _ in L.StepParams._fields_:
            if k == "stages":
                p.stages = stages
            elif k in ("center", "s_center", "s_spacesized2", "hidenpoint"):
                v = getattr(self, k)
                for i in range(3):
                    getattr(p, k)[i] = float(v[i])
            else:
                setattr(p, k, getattr(self, k))
        return p


def scalars_from(pot: prm.Potential, cells: prm.Cells, smp: prm.Sample, cmp: prm.Compress, V: float,
                 IonP: int = 32) -> Scalars:
    F = prm.F
    brazil = cmp.brazil
    wE = F(pot.hm_E) if brazil else F(2.0 * pot.hm_E)
    wG = F(pot.hm_G) if brazil else F(2.0 * pot.hm_G)
    return Scalars(
        a=cells.a, inv_a=cells.inv_a, nx=cells.nx, ny=cells.ny, nz=cells.nz, IonP=IonP,
        il_aacut=prm.il_aacut(pot.a_farcut), aa_farcut=F(pot.aa_farcut), dt=F(pot.dt), m_E=F(pot.m_E),
        m_G=F(pot.m_G), b_r=F(pot.b_r), m_Ec=F(pot.m_Ec), m_Gc=F(pot.m_Gc), hm_E=F(pot.hm_E), hm_G=F(pot.hm_G),
        p_A=F(pot.p_A), p_mu=F(pot.p_mu), p_mur=F(pot.p_mur), p_m=F(pot.p_m), p_r=F(pot.p_r), wall_E=wE,
        wall_G=wG, center=cmp.center.copy(), wall_RR=cmp.RR, wall_top=F(cmp.Top), wall_bot=F(cmp.Bottom),
        wall_V=F(V), Zcut=float(np.float32(smp.center[2] + smp.spacesized2[2])), dt_d_m=F(pot.dt_d_m),
        dt_d_I=F(pot.dt_d_I), s_center=smp.center.copy(), s_spacesized2=smp.spacesized2.copy(),
        hidenpoint=smp.hidenpoint.copy(), brazil=int(brazil), b_dd=F(pot.b_dd))


@dataclass
class RefState:
    N: int
    IonP: int = 32
    dtype: type = np.float32
    R: np.ndarray = None
    V: np.ndarray = None
    W: np.ndarray = None
    F: np.ndarray = None
    M: np.ndarray = None
    Oiwt: np.ndarray = None
    IL: np.ndarray = None
    ILtype: np.ndarray = None
    invL0: np.ndarray = None
    Rij: np.ndarray = None
    Oijt: np.ndarray = None
    Mijn: np.ndarray = None
    Mijt: np.ndarray = None
    extra: dict = field(default_factory=dict)

    @classmethod
    def empty(cls, N: int, IonP: int = 32, dtype=np.float32) -> "RefState":
        S = N * IonP
        z3 = lambda: np.zeros(3 * N, dtype)
        return cls(N=N, IonP=IonP, dtype=dtype, R=z3(), V=z3(), W=z3(), F=z3(), M=z3(), Oiwt=z3(),
                   IL=np.full(S, L.EMPTY, np.uint32), ILtype=np.zeros(S, np.uint32), invL0=np.zeros(S, dtype),
                   Rij=np.zeros(3 * S, dtype), Oijt=np.zeros(3 * S, dtype), Mijn=np.zeros(3 * S, dtype),
                   Mijt=np.zeros(3 * S, dtype))

    ARRAYS = ("R", "V", "W", "F", "M", "Oiwt", "IL", "ILtype", "invL0", "Rij", "Oijt", "Mijn", "Mijt")

    def copy(self) -> "RefState":
        s = RefState(N=self.N, IonP=self.IonP, dtype=self.dtype)
        for k in self.ARRAYS:
            setattr(s, k, getattr(self, k).copy())
        return s

    def to_dict(self, prefix: str = "") -> dict:
        return {prefix + k: getattr(self, k) for k in self.ARRAYS}

    @classmethod
    def from_dict(cls, d: dict, prefix: str = "") -> "RefState":
        R = d[prefix + "R"]
        N = R.size // 3
        IonP = d[prefix + "IL"].size // N
        s = cls(N=N, IonP=IonP, dtype=R.dtype.type)
        for k in cls.ARRAYS:
            # a copy: the steps work in place and must not change the caller's arrays
            setattr(s, k, np.array(d[prefix + k], order="C", copy=True))
        return s


# ----------------------------------------------------------------------------- oracle driver

def oracle_cells(R: np.ndarray, N: int, sc: Scalars):
    CI = np.zeros(N, np.uint32)
    CIs = np.zeros(2 * N, np.uint32)
    CN = sc.nx * sc.ny * sc.nz
    pnC = np.zeros(2 * CN, np.uint32)
    L.fn("orc_cell_distribution", R)(L.P(R), N, sc.inv_a, sc.nx, sc.ny, sc.nz, L.P(CI), L.P(CIs), L.P(pnC))
    return CI, CIs, pnC


def oracle_setup_bonds(st: RefState, sc: Scalars, rad=None, gap: float = 0.0) -> int:
    """CellDistribution + InteractionListConstruct + d_ConstructBoundInteractions + d_DeleteFarLinks."""
    CI, CIs, pnC = oracle_cells(st.R, st.N, sc)
    st.IL[:] = L.EMPTY
    ov = L.fn("orc_il_construct", st.R)(L.P(st.R), st.N, L.P(CIs), L.P(pnC), L.P(st.IL), st.IonP, sc.a, sc.inv_a,
                                        sc.il_aacut, sc.nx, sc.ny, sc.nz)
    L.fn("orc_construct_bonds", st.R)(L.P(st.R), st.N, L.P(st.IL), L.P(st.ILtype), L.P(st.invL0), L.P(st.Rij),
                                      L.P(st.Oijt), L.P(st.Mijn), L.P(st.Mijt), st.IonP, sc.b_dd, L.P(rad), gap)
    L.fn("orc_delete_far_links", st.R)(L.P(st.R), st.N, L.P(st.IL), L.P(st.ILtype), L.P(st.Rij), L.P(st.Oijt),
                                       L.P(st.Mijn), L.P(st.Mijt), st.IonP, sc.aa_farcut)
    return int(ov)


def oracle_step(st: RefState, sc: Scalars, stages: int = STAGE_ALL, *, rad=None, mass=None, slot_br=None,
                slot_sn=None, slot_st=None, dtm_i=None, dtI_i=None, want_abs: bool = False, nobreak: int = 0,
                fixsum: bool = False):
    """One pass of the loop body; returns a StepOut (tolerance scales with want_abs).

    fixsum=True sums the pair forces and moments of every particle, and the
    platen forces, in 64-bit fixed point (orc_forces_*_q, orc_platen_q) -
    the exact, order-independent sums of the engine's deterministic mode -
    instead of the reference's running float sum over a particle's slots;
    every per-pair value is the same."""
    N, R = st.N, st.R
    ov = 0
    if stages & STAGE_IL:
        CI, CIs, pnC = oracle_cells(R, N, sc)
        ov = L.fn("orc_il_reconstruct_bpm", R)(L.P(R), N, L.P(CIs), L.P(pnC), L.P(st.IL), L.P(st.ILtype),
                                               st.IonP, sc.a, sc.inv_a, sc.il_aacut, sc.nx, sc.ny, sc.nz)
    Fabs = Mabs = Fsens = None
    if stages & STAGE_FORCES and fixsum:
        Fq = np.zeros(3 * N, np.int64)
        Mq = np.zeros(3 * N, np.int64)
        L.fn("orc_forces_bpm_q", R)(L.P(R), L.P(st.V), L.P(st.W), N, L.P(st.IL), L.P(st.ILtype), L.P(st.invL0),
                                    L.P(st.Rij), L.P(st.Oijt), L.P(st.Mijn), L.P(st.Mijt), st.IonP, sc.dt, sc.m_E,
                                    sc.m_G, sc.b_r, sc.m_Ec, sc.m_Gc, L.P(slot_br), L.P(slot_sn), L.P(slot_st),
                                    nobreak, L.P(Fq), L.P(Mq))
        L.fn("orc_forces_hm_q", R)(L.P(R), L.P(st.V), L.P(st.W), N, L.P(st.IL), L.P(st.ILtype), L.P(st.Oijt),
                                   st.IonP, sc.dt, sc.hm_E, sc.hm_G, sc.p_A, sc.p_mu, sc.p_mur, sc.p_m, sc.p_r,
                                   L.P(rad), L.P(mass), L.P(Fq), L.P(Mq))
        L.fn("orc_fix_to_real", R)(L.P(Fq), L.P(st.F), 3 * N)
        L.fn("orc_fix_to_real", R)(L.P(Mq), L.P(st.M), 3 * N)
    elif stages & STAGE_FORCES:
        st.F[:] = 0
        st.M[:] = 0
        if want_abs:
            Fabs = np.zeros_like(st.F)
            Mabs = np.zeros_like(st.M)
            Fsens = np.zeros(N, st.dtype)
        L.fn("orc_forces_bpm", R)(L.P(R), L.P(st.V), L.P(st.W), N, L.P(st.IL), L.P(st.ILtype), L.P(st.invL0),
                                  L.P(st.Rij), L.P(st.Oijt), L.P(st.Mijn), L.P(st.Mijt), L.P(st.F), L.P(st.M),
                                  st.IonP, sc.dt, sc.m_E, sc.m_G, sc.b_r, sc.m_Ec, sc.m_Gc, L.P(slot_br),
                                  L.P(slot_sn), L.P(slot_st), L.P(Fabs), L.P(Mabs), L.P(Fsens), nobreak)
        L.fn("orc_forces_hm", R)(L.P(R), L.P(st.V), L.P(st.W), N, L.P(st.IL), L.P(st.ILtype), L.P(st.Oijt),
                                 L.P(st.F), L.P(st.M), st.IonP, sc.dt, sc.hm_E, sc.hm_G, sc.p_A, sc.p_mu, sc.p_mur,
                                 sc.p_m, sc.p_r, L.P(rad), L.P(mass), L.P(Fabs), L.P(Mabs), L.P(Fsens))
    sFL = np.zeros(2, np.float64)
    FL = np.zeros(2 * (N // 64 + 1), st.dtype)
    if stages & STAGE_PLATEN and fixsum:
        c = np.asarray(sc.center, st.dtype)
        L.fn("orc_platen_q", R)(1 if sc.brazil else 2, L.P(R), L.P(st.V), L.P(st.W), L.P(st.Oiwt), L.P(st.F),
                                L.P(st.M), N, sc.dt, sc.wall_E, sc.wall_G, sc.p_A, sc.p_mu, sc.p_mur, sc.p_m, sc.p_r,
                                L.P(rad), L.P(mass), L.P(c), sc.wall_RR, sc.wall_top, sc.wall_bot, sc.wall_V,
                                sc.Zcut, L.P(sFL))
    elif stages & STAGE_PLATEN:
        c = np.asarray(sc.center, st.dtype)
        L.fn("orc_platen", R)(1 if sc.brazil else 2, L.P(R), L.P(st.V), L.P(st.W), L.P(st.Oiwt), L.P(st.F),
                              L.P(st.M), N, sc.dt, sc.wall_E, sc.wall_G, sc.p_A, sc.p_mu, sc.p_mur, sc.p_m, sc.p_r,
                              L.P(rad), L.P(mass), L.P(c), sc.wall_RR, sc.wall_top, sc.wall_bot, sc.wall_V, sc.Zcut,
                              L.P(FL), L.P(sFL))
    if stages & STAGE_INCR:
        L.fn("orc_increments", R)(L.P(st.F), L.P(st.V), L.P(R), L.P(st.M), L.P(st.W), N, sc.dt_d_m, sc.dt,
                                  sc.dt_d_I, L.P(dtm_i), L.P(dtI_i))
    if stages & STAGE_CUT:
        c = np.asarray(sc.s_center, st.dtype)
        s2 = np.asarray(sc.s_spacesized2, st.dtype)
        hp = np.asarray(sc.hidenpoint, st.dtype)
        L.fn("orc_cut_restriction", R)(L.P(R), L.P(st.V), L.P(st.F), N, L.P(c), L.P(s2), L.P(hp))
    if stages & STAGE_DELETE:
        L.fn("orc_delete_far_links", R)(L.P(R), N, L.P(st.IL), L.P(st.ILtype), L.P(st.Rij), L.P(st.Oijt),
                                        L.P(st.Mijn), L.P(st.Mijt), st.IonP, sc.aa_farcut)
    return StepOut(sFL=sFL, FL=FL, Fabs=Fabs, Mabs=Mabs, Fsens=Fsens, overflow=int(ov))


# ----------------------------------------------------------------------------- reference harness driver

def ref_cells(R: np.ndarray, N: int, sc: Scalars):
    CI = np.zeros(N, np.uint32)
    CIs = np.zeros(2 * N, np.uint32)
    pnC = np.zeros(2 * sc.nx * sc.ny * sc.nz, np.uint32)
    rc = L.ref().refh_cell_distribution(L.P(R), N, sc.a, sc.nx, sc.ny, sc.nz, L.P(CI), L.P(CIs), L.P(pnC))
    assert rc == 0, rc
    return CI, CIs, pnC


def ref_setup_bonds(st: RefState, sc: Scalars) -> None:
    rc = L.ref().refh_setup_bonds(L.P(st.R), st.N, sc.a, sc.nx, sc.ny, sc.nz, st.IonP, sc.il_aacut, sc.aa_farcut,
                                  sc.b_dd, sc.b_r, L.P(st.IL), L.P(st.ILtype), L.P(st.invL0))
    assert rc == 0, rc
    st.Rij[:] = 0
    st.Oijt[:] = 0
    st.Mijn[:] = 0
    st.Mijt[:] = 0


def ref_time_steps(st: RefState, sc: Scalars, nsteps: int, stages: int = STAGE_ALL, sync_fl: bool = True) -> float:
    """Device milliseconds of nsteps passes of the reference's loop body on the state."""
    p = sc.to_c(stages)
    ms = C.c_double()
    rc = L.ref().refh_time_steps(C.byref(p), st.N, L.P(st.R), L.P(st.V), L.P(st.W), L.P(st.IL), L.P(st.ILtype),
                                 L.P(st.invL0), nsteps, 1 if sync_fl else 0, C.byref(ms))
    assert rc == 0, rc
    return ms.value


def ref_step(st: RefState, sc: Scalars, stages: int = STAGE_ALL):
    FL = np.zeros(2 * (st.N // 64 + 1), np.float32)
    p = sc.to_c(stages)
    rc = L.ref().refh_step(C.byref(p), st.N, *(L.P(getattr(st, k)) for k in RefState.ARRAYS), L.P(FL))
    assert rc == 0, rc
    nb = st.N // 64 + 1
    sFL = np.array([FL[:nb].astype(np.float64).sum(), FL[nb:].astype(np.float64).sum()])
    # the reference sums the partials one by one in double (md_results.cu:60-69)
    s0 = 0.0
    for v in FL[:nb]:
        s0 += float(v)
    s1 = 0.0
    for v in FL[nb:]:
        s1 += float(v)
    sFL[:] = (s0, s1)
    return sFL, FL
