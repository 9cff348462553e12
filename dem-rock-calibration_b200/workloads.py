"""Named specimens of the rock-calibration tests (synthetic, seeded).

* uniaxial_cylinder: 8 mm x 16 mm cylinder, radii U[0.20, 0.30] mm, packing 0.58
* brazilian_disc:    40 mm x 20 mm disc, radii U[0.18, 0.30] mm, packing ~0.6
  (about 245k spheres), diametral platens along y at 0.02 m/s

Micro-parameters: particle E = 50 GPa, nu = 0.25, rho = 2650 kg/m^3, friction
0.5; bond E = 30 GPa, kn/ks = 2.5, bond radius 0.8 min(r_i, r_j), bonds for
gaps < 0.1 r_min, normal and shear strengths N(40, 8) MPa per bond; dt = 0.2
of the smaller of the Rayleigh time and the bond time of the smallest particle.  Every value in reference
units (mm, mg, us, GPa).  Packings come from create_cylinder_sample (the
reference draws its fill from time(NULL); here the seed is explicit).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import (TEST_BRAZIL, TEST_UNIAXIAL, VELOCITY, Loading, Material, bounding_box, create_cylinder_sample,
               loading, material, reference_space)


@dataclass
class Specimen:
    name: str
    material: Material
    loading: Loading
    xyz: np.ndarray
    radii: np.ndarray
    pack: dict

    @property
    def n(self) -> int:
        return self.radii.size


def mean_r3(r_min: float, r_max: float) -> float:
    if r_max == r_min:
        return r_min ** 3
    return (r_max ** 4 - r_min ** 4) / (4.0 * (r_max - r_min))


def rock_material(r_min: float, r_mean: float, **over) -> Material:
    kw = dict(E=50.0, nu=0.25, Ec=0.040, Gc=0.040, b_r=0.0, gap=0.1 * r_min, rho=2.65, p_r=r_mean, p_e=0.6,
              mu=0.5, mur=0.05, farcut=3.2, E_bond=30.0, kn_ks=2.5, Ec_sd=0.008, Gc_sd=0.008,
              bond_radius_factor=0.8, dt_rayleigh_factor=0.2, seed=7)
    kw.update(over)
    return material(**kw)


def _specimen(name, test, diameter, height, r_min, r_max, packing, seed, velocity_m_s, min_stress_gpa, max_strain,
              dNsave, max_steps, space_factor=(1.3, 1.3, 1.5), pack_kw=None, packer=None, **mat_over):
    radius, half_h = 0.5 * diameter, 0.5 * height
    r_mean = 0.5 * (r_min + r_max)
    n = int(round(packing * math.pi * radius * radius * height / (4.0 / 3.0 * math.pi * mean_r3(r_min, r_max))))
    space_si = (2 * radius * space_factor[0] * 1e-3, 2 * radius * space_factor[1] * 1e-3,
                2 * half_h * space_factor[2] * 1e-3)
    lsi = (diameter * 1e-3, diameter * 1e-3, height * 1e-3)
    box = reference_space(space_si, lsi, r_max, 3.2)
    pk = dict(growth_stages=30, steps_per_stage=150, max_fire_steps=6000, overlap_tol=2e-3)
    pk.update(pack_kw or {})
    # `packer`: a function with create_cylinder_sample's signature and result
    # (the default, on the GPU); the same seeded packing can come from another
    # implementation of the same algorithm
    xyz, rad, rep = (packer or create_cylinder_sample)(box.center.astype(np.float64), radius, half_h, n, r_min, r_max,
                                                       E=50.0, nu=0.25, rho=2.65, seed=seed, **pk)
    size_real, center_real = bounding_box(xyz, n, r_max, radii=rad)
    ld = loading(test, box, size_real, center_real, velocity=-velocity_m_s / VELOCITY, min_stress=min_stress_gpa,
                 max_strain=max_strain, cond_fracture=0.1, dNsave=dNsave, max_steps=max_steps, p_r_platen=r_mean)
    mat = rock_material(r_min, r_mean, **mat_over)
    return Specimen(name=name, material=mat, loading=ld, xyz=xyz, radii=rad, pack=rep)


def uniaxial_cylinder(seed: int = 1, velocity_m_s: float = 0.1, max_steps: int = 0, diameter: float = 8.0,
                      height: float = 16.0, **kw) -> Specimen:
    # 0.58 rather than 0.60: the 8 mm column is only 16 diameters wide, and its
    # wall layers keep a relaxed (overlap-free) packing below the disc's 0.60
    return _specimen("uniaxial_cylinder_d8x16", TEST_UNIAXIAL, diameter, height, 0.20, 0.30, 0.58, seed,
                     velocity_m_s, 0.010, 0.01, 100, max_steps, **kw)


def brazilian_disc(seed: int = 1, velocity_m_s: float = 0.02, max_steps: int = 0, diameter: float = 40.0,
                   thickness: float = 20.0, **kw) -> Specimen:
    return _specimen("brazilian_disc_d40x20", TEST_BRAZIL, diameter, thickness, 0.18, 0.30, 0.6, seed,
                     velocity_m_s, 0.0021, 0.03, 1000, max_steps, **kw)
