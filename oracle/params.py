"""Reference parameter derivation (test infrastructure only).

Restates, in double precision with the reference's float conversions, how the
reference turns physical inputs into the scalars its kernels receive:

* potential_data::CalculateParameters      md_data_types.h:155-187
* SetInitialParameters                     mp_determineconjgradient.cu:15-47
* cell_data::CalculateParameters           md_data_types.h:42-55
* interaction_list_data::CalculateParameters md_data_types.h:139-145
* sample_data::SetSpaceSizeSi/SetLSi/CalculateParameters  md_data_types.h:87-123
* h_LoadCylinderSample bounding box        md_createcylindersample.cu:441-466
* compression_data::Calculate{U,B}Parameters md_data_types.h:212-242, 380-409

Units are the reference's: mm, mg, us (stress in GPa, force in kN).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MC_PI = 3.1415926535897932384626433832795
MC_1D3 = 1.0 / 3.0
LENGTH = 1e-3
MASS = 1e-6
TIME = 1e-6
DENSITY = MASS / (LENGTH ** 3)
STRESS = (MASS * LENGTH / TIME ** 2) / LENGTH ** 2
VELOCITY = LENGTH / TIME

f32 = np.float32


def F(x) -> float:
    """C++ double -> float conversion."""
    return float(f32(x))


@dataclass
class Potential:
    """potential_data after CalculateParameters (all doubles)."""

    m_E: float
    m_Ec: float
    m_Gc: float
    b_r: float
    b_d: float
    p_r: float
    m_ro: float
    m_nu: float = 0.247
    p_e: float = 0.6
    p_mu: float = 0.45
    p_mur: float = 0.05
    a_farcut: float = 0.0
    d: dict = field(default_factory=dict)

    def calculate(self) -> "Potential":
        d = self.d
        m_E, m_nu, p_r, m_ro = self.m_E, self.m_nu, self.p_r, self.m_ro
        d["m_G"] = 0.5 * m_E / (1.0 + m_nu)
        d["b_S"] = MC_PI * self.b_r * self.b_r
        d["p_V"] = 4.0 * MC_1D3 * MC_PI * p_r * p_r * p_r
        d["p_m"] = m_ro * d["p_V"]
        d["b_dd"] = self.b_d * self.b_d
        d["p_1d_m"] = 1.0 / d["p_m"]
        d["p_I"] = 0.4 * d["p_m"] * p_r * p_r
        d["hm_E"] = 0.5 * m_E / (1.0 - m_nu * m_nu)
        d["hm_G"] = 0.5 * d["m_G"] / (2.0 - m_nu)
        le = math.log(self.p_e)
        d["p_A"] = le / math.sqrt(MC_PI * MC_PI + le * le)
        d["aa_farcut"] = self.a_farcut * self.a_farcut
        d["Trayleigh"] = MC_PI * p_r * math.sqrt(2.0 * m_ro * (1.0 + m_nu)) / (
            math.sqrt(m_E) * (0.163 * m_nu + 0.8766))
        t0 = m_E * d["b_S"] / (2.0 * p_r)
        t1 = d["m_G"] * d["b_S"] / (2.0 * p_r)
        d["Tsim"] = 2.0 * math.sqrt(d["p_m"] / t0) if t0 > t1 else 2.0 * math.sqrt(d["p_m"] / t1)
        d["dt"] = 0.05 * d["Trayleigh"] if d["Trayleigh"] < d["Tsim"] else 0.05 * d["Tsim"]
        d["D"] = 1e-15 * m_E * d["b_S"] / (2.0 * p_r)
        d["dt_d_m"] = d["p_1d_m"] * d["dt"]
        d["dt_d_I"] = d["dt"] / d["p_I"]
        return self

    def __getattr__(self, k):
        d = self.__dict__.get("d")
        if d is not None and k in d:
            return d[k]
        raise AttributeError(k)


def initial_potential(E_si, Ec_si, Gc_si, br_si, gap_si, p_r_si=0.5e-3, rho_si=2610.0, nu=0.247,
                      p_e=0.6, p_mu=0.45, p_mur=0.05, farcut=3.2) -> Potential:
    """SetInitialParameters, mp_determineconjgradient.cu:15-47."""
    p_r = p_r_si / LENGTH
    pot = Potential(m_E=E_si / STRESS, m_Ec=Ec_si / STRESS, m_Gc=Gc_si / STRESS, b_r=br_si / LENGTH,
                    b_d=2.0 * p_r + gap_si / LENGTH, p_r=p_r, m_ro=rho_si / DENSITY, m_nu=nu, p_e=p_e,
                    p_mu=p_mu, p_mur=p_mur, a_farcut=farcut * p_r)
    return pot.calculate()


@dataclass
class Cells:
    """cell_data after CalculateParameters (md_data_types.h:42-55)."""

    a: float        # float
    inv_a: float    # float
    nx: int
    ny: int
    nz: int

    @property
    def CN(self) -> int:
        return self.nx * self.ny * self.nz


def cells_for(a_double: float, B) -> Cells:
    a = F(a_double)                  # C.a is a float
    inv_a = F(1.0 / a)               # _1d_a = 1.0 / double(a)
    n = []
    for k, extra in ((0, 1), (1, 1), (2, 4)):
        prod = float(B[k]) * inv_a   # double * float -> double
        n.append(int(F(math.floor(F(prod))) + extra))  # floorf(float(prod)) + extra
    return Cells(a=a, inv_a=inv_a, nx=n[0], ny=n[1], nz=n[2])


@dataclass
class Sample:
    """sample_data (md_data_types.h:79-124); float3 members kept as float."""

    spacesize: np.ndarray
    spacesized2: np.ndarray
    L: np.ndarray
    A: np.ndarray
    B: np.ndarray
    center: np.ndarray
    sized2: np.ndarray
    hidenpoint: np.ndarray
    Vext: float
    size_real: np.ndarray = None
    center_real: np.ndarray = None


def sample_for(space_si, lsi, C_a_float: float, p_r: float) -> Sample:
    spacesize = np.array([F(x / LENGTH) for x in space_si], dtype=np.float32)
    spacesized2 = np.array([F(0.5 * float(s)) for s in spacesize], dtype=np.float32)
    L = np.array([F(x / LENGTH - 2.0 * p_r) for x in lsi], dtype=np.float32)
    C_a = float(C_a_float)
    A = np.array([F(1.01 * C_a)] * 3, dtype=np.float32)
    B = (A + spacesize).astype(np.float32)
    center = np.array([F(0.5 * float(f32(A[k] + B[k]))) for k in range(3)], dtype=np.float32)
    sized2 = np.array([F(0.5 * float(L[k])) for k in range(3)], dtype=np.float32)
    Vext = MC_PI * (0.5 * float(L[0]) + p_r) * (0.5 * float(L[0]) + p_r) * (float(L[2]) + 2.0 * p_r)
    hp = np.array([F(float(A[0]) + 0.5 * float(spacesize[0])), F(float(A[1]) + 0.5 * float(spacesize[1])),
                   F((float(f32(math.floor(F(float(B[2]) / C_a)))) + 3 - 0.5) * C_a)], dtype=np.float32)
    return Sample(spacesize, spacesized2, L, A, B, center, sized2, hp, Vext)


def bounding_box(R_soa: np.ndarray, n: int, p_r: float):
    """h_LoadCylinderSample, md_createcylindersample.cu:448-465."""
    x, y, z = R_soa[:n].astype(np.float64), R_soa[n:2 * n].astype(np.float64), R_soa[2 * n:].astype(np.float64)
    mn = np.array([x.min(), y.min(), z.min()])
    mx = np.array([x.max(), y.max(), z.max()])
    size_real = mx - mn + 2.0 * p_r
    center_real = 0.5 * (mx + mn)
    return size_real, center_real


@dataclass
class Compress:
    """The float kernel arguments of the platen kernels plus the double state."""

    brazil: bool
    center: np.ndarray      # float3
    RR: float               # float
    Top: float
    Bottom: float
    Area: float
    inv_Area: float
    size_d: np.ndarray
    Size0: float
    MinStress: float
    ZeroStress: float
    MaxStrain: float
    ConditionFracture: float


def compress_for(brazil: bool, size_real, center_real, p_r: float, minstress, maxstrain, condfract) -> Compress:
    size_d = np.array(size_real, dtype=np.float64)
    sized2 = np.array([F(0.5 * s) for s in size_d], dtype=np.float32)
    center = np.array([F(c) for c in center_real], dtype=np.float32)
    ax = 1 if brazil else 2
    Bottom = float(center_real[ax]) - 0.5 * size_d[ax]
    Top = float(center_real[ax]) + 0.5 * size_d[ax]
    if not brazil:
        R = F(1.5 * float(sized2[0]))
        area = F(MC_PI * (float(sized2[0]) + p_r) * (float(sized2[0]) + p_r))
        zero = 0.33 * minstress
    else:
        R = float(sized2[0]) if sized2[0] > sized2[2] else F(1.05 * float(sized2[2]))
        area = F(0.5 * 2 * MC_PI * float(sized2[0]) * float(f32(size_d[2])))
        zero = 0.5 * minstress
    RR = float(f32(R) * f32(R))
    return Compress(brazil=brazil, center=center, RR=RR, Top=Top, Bottom=Bottom, Area=area,
                    inv_Area=F(1.0 / area), size_d=size_d, Size0=float(size_d[ax]), MinStress=minstress,
                    ZeroStress=zero, MaxStrain=maxstrain, ConditionFracture=condfract)


def il_aacut(a_farcut_double: float) -> float:
    """interaction_list_data::CalculateParameters: acut, aacut are floats."""
    acut = f32(a_farcut_double)
    return float(acut * acut)
