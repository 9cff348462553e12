"""Whole loading tests run by the CPU oracle (test infrastructure only).

loading_run() repeats the loop body of the reference's drivers
(md_calculationuniaxialcompression.cu:265-314, md_calculationbraziltest.cu:185-231)
with the oracle's kernels - cells and interaction-list rebuild, bond and
Hertz-Mindlin forces, platen contacts, integration, escape parking, far-link
deletion - and the reference's host controller restated in oracle/dem_oracle.c
(SumForces{U,B}Loading, md_results.cu:56-145; Compress{U,B}_S3,
md_data_types.h:347-494): the platen positions, the loading record (strain,
bottom and top platen stress every dNsave steps while the platens move) and
the stop condition (strain limit or fracture).  Optionally it also records
the mean radial distance of a set of lateral-surface spheres on the record
steps, from which a Poisson ratio follows.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as L
from . import sim


def loading_run(st: sim.RefState, sc: sim.Scalars, *, brazil: bool, size_real, center_real, p_r: float,
                min_stress: float, max_strain: float, cond_fracture: float, velocity: float, dt: float,
                dNsave: int, max_steps: int, nobreak: int = 0, lateral=None, axis_center=None,
                fixsum: bool = False, on_step=None, **kw) -> dict:
    """Runs until the strain limit, fracture or max_steps.  `lateral`: indices
    of spheres whose mean distance from the vertical axis through
    axis_center (x, y) is recorded on every record step.
    fixsum=True: pair, platen and lateral sums in 64-bit fixed point, as the
    engine's deterministic mode sums them (sim.oracle_step), so that a whole
    run of the engine in that mode can be compared with this one exactly.
    on_step(step, st, comp), if given, is called after every step (the
    controller updated); a true return value ends the run.
    Returns the record (strain, sigma_bottom, sigma_top per entry), the
    lateral record, the controller's results and the step count."""
    lib = L.lib()
    comp = L.Compress()
    sr = np.ascontiguousarray(size_real, np.float64)
    cr = np.ascontiguousarray(center_real, np.float64)
    lib.orc_compress_init(C.byref(comp), 1 if brazil else 0, L.P(sr), L.P(cr), p_r, min_stress, max_strain,
                          cond_fracture, velocity)
    nsave = max_steps // max(dNsave, 1) + 4
    rec = np.zeros(3 * (nsave + 2), np.float64)
    comp.h_sFL = rec.ctypes.data_as(C.POINTER(C.c_double))
    comp.Nsave = nsave
    comp.dNsave = dNsave
    lat = []
    n = st.N
    steps = 0
    while steps < max_steps:
        sc.wall_top = float(np.float32(comp.Top))
        sc.wall_bot = float(np.float32(comp.Bottom))
        sc.wall_V = float(np.float32(comp.V))
        out = sim.oracle_step(st, sc, sim.STAGE_ALL, nobreak=nobreak, fixsum=fixsum, **kw)
        comp.sFL[0], comp.sFL[1] = float(out.sFL[0]), float(out.sFL[1])
        before = comp.stepsave
        if lateral is not None and dNsave and steps % dNsave == 0:
            x = st.R[lateral].astype(np.float64)
            y = st.R[n + lateral].astype(np.float64)
            d = np.sqrt((x - axis_center[0]) * (x - axis_center[0]) + (y - axis_center[1]) * (y - axis_center[1]))
            if fixsum:
                lat_val = float(np.rint(d * 2.0 ** 40).astype(np.int64).sum()) * 2.0 ** -40 / lateral.size
            else:
                lat_val = float(np.sum(d)) / lateral.size
        lib.orc_sum_forces(C.byref(comp), steps)
        if lateral is not None and comp.stepsave > before:
            lat.append(lat_val)
        lib.orc_compress_s3(C.byref(comp), dt, p_r)
        steps += 1
        if on_step is not None and on_step(steps, st, comp):
            break
        if not (abs(comp.Strain) < comp.MaxStrain) or comp.Fracture:
            break
    m = comp.stepsave
    return dict(rec=rec[:3 * m].reshape(-1, 3).copy(), lat=np.array(lat), steps=steps,
                FractureStress=comp.FractureStress, FractureStrain=comp.FractureStrain, Strain=comp.Strain,
                fracture=comp.Fracture)


def chord_moduli(rec: np.ndarray, lat: np.ndarray | None):
    """Chord Young modulus between 10% and 50% of the peak stress on the
    rising branch of a record, and the Poisson ratio over the same interval
    from the lateral record (the definitions the engine reports; the
    reference computes neither)."""
    sig = 0.5 * (np.abs(rec[:, 1]) + np.abs(rec[:, 2]))
    eps = -rec[:, 0]
    kp = int(np.argmax(sig))
    pts = []
    for level in (0.1, 0.5):
        t = level * sig[kp]
        k = next(k for k in range(1, kp + 1) if sig[k] >= t > sig[k - 1])
        w = (t - sig[k - 1]) / (sig[k] - sig[k - 1])
        e = eps[k - 1] + w * (eps[k] - eps[k - 1])
        l = None if lat is None else lat[k - 1] + w * (lat[k] - lat[k - 1])
        pts.append((e, l))
    (e1, l1), (e5, l5) = pts
    E = 0.4 * sig[kp] / (e5 - e1)
    nu = None if lat is None else ((l5 - l1) / lat[0]) / (e5 - e1)
    return E, nu


def lateral_spheres(xyz: np.ndarray, radii: np.ndarray, center_real, size_real, r_mean: float) -> np.ndarray:
    """The engine's lateral-surface set of a uniaxial specimen: spheres within
    one mean diameter of the outermost surface, |z - z_c| <= H/4."""
    n = radii.size
    x, y, z = (xyz.reshape(3, n).astype(np.float64))
    cx, cy, cz = center_real
    rho = np.hypot(x - cx, y - cy)
    outer = np.max(rho + radii)
    keep = (rho + radii >= outer - 2.0 * r_mean) & (np.abs(z - cz) <= 0.25 * size_real[2])
    return np.nonzero(keep)[0]
