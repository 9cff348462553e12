"""ctypes binding of the CPU restatement of the engine's sample creation
(oracle/dem_pack_oracle.c, in oracle/_build/libdemoracle.so).  Test
infrastructure only: the packer's GPU parity test and the benchmark's
reference leg, which builds its specimens on the host.

create_cylinder_sample() takes the arguments of the product's
create_cylinder_sample (variant-0/1 FIRE, no sphere removal) and returns the
same (xyz SoA, radii, report) - bit for bit the packing the GPU produces.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as L


class PackParams(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("radius", C.c_double), ("half_height", C.c_double),
                ("r_min", C.c_double), ("r_max", C.c_double), ("E", C.c_double), ("nu", C.c_double),
                ("rho", C.c_double), ("overlap_tol", C.c_double), ("n", C.c_uint32), ("growth_stages", C.c_uint32),
                ("steps_per_stage", C.c_uint32), ("max_fire_steps", C.c_uint32), ("seed", C.c_uint64),
                ("device", C.c_int), ("fire_variant", C.c_int), ("max_removed", C.c_uint32),
                ("reserved", C.c_uint32)]


class PackReport(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("max_overlap", C.c_double), ("packing_fraction", C.c_double),
                ("rebuilds", C.c_uint32), ("removed", C.c_uint32)]


def _fn():
    f = L.lib().orc_pack_cylinder
    f.argtypes = [C.POINTER(PackParams), C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32),
                  C.POINTER(PackReport), C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]
    f.restype = C.c_int
    return f


def create_cylinder_sample(center, radius: float, half_height: float, n: int, r_min: float, r_max: float,
                           E: float = 50.0, nu: float = 0.25, rho: float = 2.65, overlap_tol: float = 1e-3,
                           growth_stages: int = 40, steps_per_stage: int = 200, max_fire_steps: int = 20000,
                           seed: int = 1, device: int = 0, fire_variant: int = 0, max_removed: int = 0,
                           trace_cap: int = 0):
    """Returns xyz (SoA float32), radii, report dict; with trace_cap > 0 the
    report also holds 'fire_trace', (dt, alpha, back) after each FIRE step."""
    if max_removed:
        raise ValueError("the CPU packer restates the packer without sphere removal")
    p = PackParams(radius=radius, half_height=half_height, r_min=r_min, r_max=r_max, E=E, nu=nu, rho=rho,
                   overlap_tol=overlap_tol, n=n, growth_stages=growth_stages, steps_per_stage=steps_per_stage,
                   max_fire_steps=max_fire_steps, seed=seed, device=device, fire_variant=fire_variant,
                   max_removed=0)
    for d in range(3):
        p.center[d] = float(center[d])
    xyz = np.zeros(3 * n, np.float32)
    rad = np.zeros(n, np.float32)
    m = C.c_uint32()
    rep = PackReport()
    trace = np.zeros(3 * max(trace_cap, 1), np.float64)
    nt = C.c_uint32()
    rc = _fn()(C.byref(p), L.P(xyz), L.P(rad), n, C.byref(m), C.byref(rep), L.P(trace) if trace_cap else None,
               trace_cap, C.byref(nt))
    if rc != 0:
        raise RuntimeError(f"orc_pack_cylinder returned {rc}")
    out = dict(steps=rep.steps, max_overlap=rep.max_overlap, packing_fraction=rep.packing_fraction,
               rebuilds=rep.rebuilds, removed=rep.removed)
    if trace_cap:
        out["fire_trace"] = trace[:3 * nt.value].reshape(-1, 3)
    return xyz, rad, out
