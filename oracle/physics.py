"""Oracle inputs for the configurations' own physics (test infrastructure only).

The configurations extend the reference's monodisperse step (the reference
uses one radius p_r, one modulus m_E for particles and bonds, scalar
strengths m_Ec/m_Gc and an absolute bond radius b_r;
md_calculateforcesdem3.cu:238,365, mp_determineconjgradient.cu:15-47) with
per-sphere radii, a bond modulus and kn/ks ratio of their own, a bond radius
factor * min(r_i, r_j), per-bond normal and shear strengths drawn from a
normal distribution, and a time step from a Rayleigh factor.  The oracle
(dem_oracle.h) takes these as optional per-particle and per-slot arrays and
reduces to the reference's formulas when they are uniform.  This module
derives those arrays and the kernel scalars for a specimen given in the
engine's units and parameter structs, with the engine's formulas restated:

* time step: factor * min(Rayleigh time, bond time 2 sqrt(m/k)) of the
  smallest sphere, k = max(E_b, G_b) pi b^2 / (2 r) (the reference's
  potential_data::CalculateParameters rule, md_data_types.h:168-178, with the
  configuration's factor);
* per-sphere mass, dt/m and dt/I: the reference's p_m, dt_d_m, dt_d_I
  formulas (md_data_types.h:158-181) per radius;
* per-bond strengths: mean + sd * a counter-based normal deviate keyed by
  the pair's original indices (splitmix64 mixing, Box-Muller), clipped at 0.

Values are rounded to the kernel's scalar type (float for FP32 builds,
double for FP64 builds) where the engine rounds them.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import lib as L
from . import params as prm
from . import sim

PI = 3.1415926535897932384626433832795
M64 = (1 << 64) - 1


def rayleigh_time(r, rho, E, nu):
    return PI * r * np.sqrt(2.0 * rho * (1.0 + nu)) / (np.sqrt(E) * (0.163 * nu + 0.8766))


def bond_moduli(mat):
    E_b = mat.E_bond if mat.E_bond > 0 else mat.E
    G_b = E_b / mat.kn_ks if mat.kn_ks > 0 else 0.5 * E_b / (1.0 + mat.nu)
    return E_b, G_b


def time_step(mat, radii) -> float:
    """The engine's time step of a specimen (double)."""
    if mat.dt > 0:
        return float(mat.dt)
    r = float(np.min(np.asarray(radii, np.float64)))
    if not mat.dt_rayleigh_factor > 0:
        raise ValueError("reference-rule time steps are derived by oracle.params")
    E_b, G_b = bond_moduli(mat)
    b = mat.b_r if mat.b_r > 0 else mat.bond_radius_factor * r
    k = max(E_b, G_b) * PI * b * b / (2.0 * r)
    mass = mat.rho * 4.0 * (1.0 / 3.0) * PI * r * r * r
    T = float(rayleigh_time(r, mat.rho, mat.E, mat.nu))
    if k > 0:
        T = min(T, 2.0 * np.sqrt(mass / k))
    return mat.dt_rayleigh_factor * T


def particle_constants(radii, rho, dt):
    """mass, dt/m, dt/I per sphere in double (the reference's formulas per radius)."""
    r = np.asarray(radii, np.float64)
    V = 4.0 * (1.0 / 3.0) * PI * r * r * r
    m = rho * V
    inv_m = 1.0 / m
    I = 0.4 * m * r * r
    return m, inv_m * dt, dt / I


def _splitmix64(z):
    z = (z + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(M64)
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(M64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(M64)
    return z ^ (z >> np.uint64(31))


def _u01(h):
    return ((h >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def normal_deviates(seed: int, a, b, stream: int) -> np.ndarray:
    """Counter-based standard normal deviates keyed by (seed, a, b, stream)."""
    with np.errstate(over="ignore"):
        a = np.asarray(a, np.uint64)
        b = np.asarray(b, np.uint64)
        s = np.uint64(seed)
        k = _splitmix64(s ^ _splitmix64(a * np.uint64(0x100000001B3) + b) ^
                        (np.uint64(stream) * np.uint64(0xD6E8FEB86659FD93)))
        u1 = _u01(_splitmix64(k))
        u2 = _u01(_splitmix64(k ^ np.uint64(0x5851F42D4C957F2D)))
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586476925286766559 * u2)


def bond_strengths(mat, i, j, dtype=np.float32):
    """Normal and shear strength of bonds (i, j) (original indices)."""
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    sn = np.full(lo.shape, mat.Ec, np.float64)
    st = np.full(lo.shape, mat.Gc, np.float64)
    if mat.Ec_sd > 0:
        sn = float(dtype(mat.Ec)) + float(dtype(mat.Ec_sd)) * normal_deviates(mat.seed, lo, hi, 1)
    if mat.Gc_sd > 0:
        st = float(dtype(mat.Gc)) + float(dtype(mat.Gc_sd)) * normal_deviates(mat.seed, lo, hi, 2)
    return np.maximum(sn.astype(dtype), 0), np.maximum(st.astype(dtype), 0)


@dataclass
class PhysicsCase:
    """Oracle arguments of one specimen in physics mode."""

    sc: sim.Scalars
    rad: np.ndarray
    mass: np.ndarray
    dtm: np.ndarray
    dtI: np.ndarray
    dt: float
    IonP: int
    dtype: type

    def kw(self, slot_br=None, slot_sn=None, slot_st=None) -> dict:
        return dict(rad=self.rad, mass=self.mass, slot_br=slot_br, slot_sn=slot_sn, slot_st=slot_st,
                    dtm_i=self.dtm, dtI_i=self.dtI)


def physics_case(mat, ld, radii, dt=None, dtype=np.float32, IonP: int = 48) -> PhysicsCase:
    """Kernel scalars and per-sphere arrays of a specimen (material `mat`,
    loading `ld`: the engine's dem_material / dem_loading) for the oracle."""
    R = dtype
    cast = (lambda x: float(np.float32(x))) if dtype == np.float32 else float
    f32 = lambda x: float(np.float32(x))
    rad = np.ascontiguousarray(radii, np.float32).astype(dtype)
    dt = time_step(mat, radii) if dt is None else float(dt)
    m, dtm, dtI = particle_constants(np.asarray(radii, np.float32), mat.rho, dt)
    p_r = mat.p_r if mat.p_r > 0 else float(np.mean(np.asarray(radii, np.float64)))
    a_far = mat.farcut * p_r
    C_a = f32(2.0 * a_far)
    B = [ld.space_center[d] + ld.space_half[d] + 1.01 * C_a for d in range(3)]
    cells = prm.cells_for(2.0 * a_far, B)
    E_b, G_b = bond_moduli(mat)
    hmE = 0.5 * mat.E / (1.0 - mat.nu ** 2)
    Gp = 0.5 * mat.E / (1.0 + mat.nu)
    hmG = 0.5 * Gp / (2.0 - mat.nu)
    le = np.log(mat.p_e)
    pA = le / np.sqrt(PI * PI + le * le)
    brazil = ld.test == 2
    # platen frame: compression_data::Calculate{U,B}Parameters with float members
    sx2, sz2 = f32(0.5 * ld.size_real[0]), f32(0.5 * ld.size_real[2])
    Rw = (sx2 if sx2 > sz2 else f32(1.05 * sz2)) if brazil else f32(1.5 * sx2)
    sc = sim.Scalars(
        a=cells.a, inv_a=cells.inv_a, nx=cells.nx, ny=cells.ny, nz=cells.nz, IonP=IonP,
        il_aacut=prm.il_aacut(a_far), aa_farcut=cast(a_far * a_far), dt=cast(dt), m_E=cast(E_b), m_G=cast(G_b),
        b_r=0.0, m_Ec=cast(mat.Ec), m_Gc=cast(mat.Gc), hm_E=cast(hmE), hm_G=cast(hmG), p_A=cast(pA),
        p_mu=cast(mat.mu), p_mur=cast(mat.mur), p_m=0.0, p_r=p_r,
        wall_E=cast(hmE) if brazil else cast(2.0 * hmE), wall_G=cast(hmG) if brazil else cast(2.0 * hmG),
        center=np.array([f32(v) for v in ld.center_real], R), wall_RR=f32(np.float32(Rw) * np.float32(Rw)),
        wall_top=f32(ld.center_real[1 if brazil else 2] + 0.5 * ld.size_real[1 if brazil else 2]),
        wall_bot=f32(ld.center_real[1 if brazil else 2] - 0.5 * ld.size_real[1 if brazil else 2]),
        wall_V=f32(ld.velocity), Zcut=f32(ld.zcut), dt_d_m=0.0, dt_d_I=0.0,
        s_center=np.array([f32(v) for v in ld.space_center], R),
        s_spacesized2=np.array([f32(v) for v in ld.space_half], R),
        hidenpoint=np.array([f32(v) for v in ld.hidden_point], R), brazil=int(brazil))
    return PhysicsCase(sc=sc, rad=rad, mass=m.astype(dtype), dtm=dtm.astype(dtype), dtI=dtI.astype(dtype), dt=dt,
                       IonP=IonP, dtype=dtype)


def ref_state_from_pairs(R, V, W, Oiwt, pairs: dict, pc: PhysicsCase):
    """A reference-layout state (oracle slots) holding the given particle state
    and pair table (original indices i < j, kind 1 intact bond / 2 broken bond
    / 3 contact, 16 values: 1/L0, previous direction, tangential, twisting and
    bending histories, normal and shear strength, bond radius).  The slots
    come from the oracle's own interaction-list construction at these
    positions; the j -> i slot of a pair holds the mirrored (negated) vectors.
    Returns the state and the per-slot bond radius and strengths."""
    n = R.size // 3
    st = sim.RefState.empty(n, IonP=pc.IonP, dtype=pc.dtype)
    st.R[:] = R
    st.V[:] = V
    st.W[:] = W
    st.Oiwt[:] = Oiwt
    sc = pc.sc
    CI, CIs, pnC = sim.oracle_cells(st.R, n, sc)
    ov = L.fn("orc_il_construct", st.R)(L.P(st.R), n, L.P(CIs), L.P(pnC), L.P(st.IL), st.IonP, sc.a, sc.inv_a,
                                        sc.il_aacut, sc.nx, sc.ny, sc.nz)
    if ov:
        raise RuntimeError(f"oracle interaction list overflow ({ov} slots)")
    P = pc.IonP
    IL = st.IL.reshape(n, P)
    slot_br = np.zeros(n * P, pc.dtype)
    slot_sn = np.zeros(n * P, pc.dtype)
    slot_st = np.zeros(n * P, pc.dtype)
    # slot of (a, b): position of b in a's row
    rows, cols = np.nonzero(IL != L.EMPTY)
    key = rows.astype(np.int64) * n + IL[rows, cols].astype(np.int64)
    order = np.argsort(key)
    skey = key[order]
    slot_of = (rows * P + cols)[order]

    def find(a, b):
        k = a.astype(np.int64) * n + b.astype(np.int64)
        pos = np.searchsorted(skey, k)
        ok = (pos < skey.size) & (skey[np.minimum(pos, skey.size - 1)] == k)
        if not np.all(ok):
            raise RuntimeError(f"{int((~ok).sum())} pairs beyond the oracle's interaction list")
        return slot_of[pos]

    i, j, kind, s = pairs["i"], pairs["j"], pairs["kind"], pairs["state"].astype(pc.dtype)
    si, sj = find(i, j), find(j, i)
    for slots, sign in ((si, 1), (sj, -1)):
        bond = kind == 1
        st.ILtype[slots] = bond.astype(np.uint32)
        st.invL0[slots] = np.where(kind != 3, s[:, 0], 0)
        for arr, a0 in ((st.Rij, 1), (st.Oijt, 4), (st.Mijn, 7), (st.Mijt, 10)):
            v = arr.reshape(-1, 3)
            vals = sign * s[:, a0:a0 + 3]
            if arr is not st.Oijt:
                vals = np.where(bond[:, None], vals, 0)
            v[slots] = vals
        slot_sn[slots] = s[:, 13]
        slot_st[slots] = s[:, 14]
        slot_br[slots] = s[:, 15]
    return st, slot_br, slot_sn, slot_st
