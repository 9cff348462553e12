"""Shared helpers for the tests and the golden-vector generator.

Seeded specimens in the reference's geometry and units (mm, mg, us):
an FCC lattice of equal spheres with a uniform jitter, cut to a cylinder,
and the reference parameter set built the way the reference builds it.
"""
from __future__ import annotations

import math
import sys
from dataclasses import dataclass
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle import params as prm  # noqa: E402
from oracle import sim  # noqa: E402


@dataclass
class RefCase:
    pot: prm.Potential
    cells: prm.Cells
    smp: prm.Sample
    cmp: prm.Compress
    sc: sim.Scalars
    R: np.ndarray          # float32 SoA positions (mm)
    N: int
    lsi: tuple
    space: tuple
    kw: dict = None


def fcc_cylinder(center, radius: float, half_h: float, d: float, jitter: float, rng) -> np.ndarray:
    """FCC points with nearest-neighbour distance d inside a z-axis cylinder."""
    a = d * math.sqrt(2.0)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) * a
    nxy = int(math.ceil(radius / a)) + 1
    nz = int(math.ceil(half_h / a)) + 1
    g = np.arange(-nxy, nxy + 1)
    gz = np.arange(-nz, nz + 1)
    cell = np.stack(np.meshgrid(g, g, gz, indexing="ij"), -1).reshape(-1, 3) * a
    pts = (cell[:, None, :] + basis[None]).reshape(-1, 3)
    pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    rr = pts[:, 0] ** 2 + pts[:, 1] ** 2
    keep = (rr <= radius ** 2) & (np.abs(pts[:, 2]) <= half_h)
    pts = pts[keep] + np.asarray(center, dtype=np.float64)[None]
    return pts


def ref_case(seed: int = 1, lsi=(0.0045, 0.0045, 0.006), space=(0.009, 0.009, 0.012), p_r_si=0.25e-3,
             E=30e9, Ec=40e6, Gc=40e6, br_si=0.2e-3, gap_si=0.025e-3, jitter_frac=0.03, brazil=False,
             velocity_si=-0.1, minstress_si=10e6, maxstrain=0.01, condfract=0.1, farcut=3.2,
             lattice_gap=0.0) -> RefCase:
    """A reference-mode specimen (equal radii, scalar micro-parameters).

    lattice_gap > 0: nearest-neighbour spacing 2 p_r + lattice_gap * gap and the
    jitter given in units of gap (jitter_frac * gap), so that no two spheres
    overlap and every nearest pair is inside the bond distance."""
    pot = prm.initial_potential(E, Ec, Gc, br_si, gap_si, p_r_si=p_r_si, farcut=farcut)
    C_a = prm.F(2.0 * pot.a_farcut)
    smp = prm.sample_for(space, lsi, C_a, pot.p_r)
    cells = prm.cells_for(2.0 * pot.a_farcut, smp.B)
    rng = np.random.default_rng(seed)
    if lattice_gap > 0:
        gap_mm = gap_si / prm.LENGTH
        d = 2.0 * pot.p_r + lattice_gap * gap_mm
        jitter = jitter_frac * gap_mm
    else:
        d = 2.0 * pot.p_r
        jitter = jitter_frac * d
    pts = fcc_cylinder(smp.center.astype(np.float64), 0.5 * float(smp.L[0]), 0.5 * float(smp.L[2]), d, jitter, rng)
    N = pts.shape[0]
    R = np.ascontiguousarray(pts.T.reshape(-1).astype(np.float32))
    size_real, center_real = prm.bounding_box(R, N, pot.p_r)
    smp.size_real, smp.center_real = size_real, center_real
    cmp = prm.compress_for(brazil, size_real, center_real, pot.p_r, minstress_si / prm.STRESS, maxstrain,
                           condfract)
    sc = sim.scalars_from(pot, cells, smp, cmp, velocity_si / prm.VELOCITY)
    kw = dict(seed=seed, p_r_si=p_r_si, E=E, Ec=Ec, Gc=Gc, br_si=br_si, gap_si=gap_si, brazil=brazil,
              velocity_si=velocity_si, minstress_si=minstress_si, maxstrain=maxstrain, condfract=condfract,
              farcut=farcut, lattice_gap=lattice_gap)
    return RefCase(pot=pot, cells=cells, smp=smp, cmp=cmp, sc=sc, R=R, N=N, lsi=lsi, space=space, kw=kw)


def perturb(st: sim.RefState, rng, dx=0.004, v=2e-4, w=2e-3) -> None:
    """Random displacement, velocity and spin (same draws for any backend)."""
    N = st.N
    st.R += rng.normal(0.0, dx, 3 * N).astype(st.dtype)
    st.V[:] = rng.normal(0.0, v, 3 * N).astype(st.dtype)
    st.W[:] = rng.normal(0.0, w, 3 * N).astype(st.dtype)


def canonical_sets(IL: np.ndarray, N: int, IonP: int, perm=None):
    """Per-particle neighbour sets (sorted), optionally mapped by a permutation."""
    out = []
    M = IL.reshape(N, IonP)
    for i in range(N):
        s = M[i][M[i] != 0xFFFFFFFF]
        out.append(np.sort(s))
    return out
