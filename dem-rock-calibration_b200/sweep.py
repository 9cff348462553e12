"""Batched calibration sweeps: many specimens x micro-parameter sets advanced
together in one engine context (one launch per kernel per step for all of
them), against the same work run one specimen at a time.

The reference runs one specimen per process (kernel.cu:23-123, one
h_Calculation* call per sample, mp_calculateonesample.cu:151-214) and its
calibration drivers call it once per parameter set (mp_determineconjgradient.cu:
84-351: six finite-difference solves per conjugate-gradient step).  Here a
parameter set is a dem_material, a specimen a packed cylinder; a sweep is the
Cartesian pairing given by the caller.

Parameter space of the sweep (seeded Latin hypercube):
    bond E 10-80 GPa, kn/ks 1-4, strength mean 20-80 MPa, strength sd 10-25% of
    the mean, friction 0.2-0.8, bond-radius factor 0.5-1.0.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import (Context, TEST_UNIAXIAL, VELOCITY, Material, bounding_box, create_cylinder_sample, loading,
               reference_space)
from .workloads import mean_r3, rock_material

# name: (low, high)
SWEEP_SPACE = {
    "E_bond": (10.0, 80.0),        # GPa
    "kn_ks": (1.0, 4.0),
    "strength": (0.020, 0.080),    # GPa (mean of N(mean, sd) per bond, normal and shear)
    "strength_sd": (0.10, 0.25),   # fraction of the mean
    "mu": (0.2, 0.8),
    "bond_radius_factor": (0.5, 1.0),
}


def latin_hypercube(n: int, seed: int, space: dict = SWEEP_SPACE) -> list[dict]:
    """n points, one per row of every parameter's n equal strata (seeded)."""
    rng = np.random.default_rng(seed)
    keys = list(space)
    out = np.empty((n, len(keys)))
    for k, name in enumerate(keys):
        lo, hi = space[name]
        u = (rng.permutation(n) + rng.random(n)) / n
        out[:, k] = lo + u * (hi - lo)
    return [dict(zip(keys, row)) for row in out]


def material_for(p: dict, r_min: float, r_mean: float, seed: int) -> Material:
    s = p["strength"]
    return rock_material(r_min, r_mean, E_bond=p["E_bond"], kn_ks=p["kn_ks"], Ec=s, Gc=s,
                         Ec_sd=p["strength_sd"] * s, Gc_sd=p["strength_sd"] * s, mu=p["mu"],
                         bond_radius_factor=p["bond_radius_factor"], seed=seed)


def cylinder(n: int, seed: int, r_min: float = 0.20, r_max: float = 0.30, packing: float = 0.58,
             aspect: float = 2.0, device: int = 0):
    """A packed cylinder of about n spheres (height = aspect x diameter),
    placed at the centre of its reference-style escape box.  Returns
    (xyz, radii, pack report, escape box, size_real, center_real)."""
    # n (4/3) pi <r^3> = packing * pi R^2 * (2 aspect R)
    R = (n * (2.0 / 3.0) * mean_r3(r_min, r_max) / (packing * aspect)) ** (1.0 / 3.0)
    half_h = aspect * R
    space_si = (2 * R * 1.3e-3, 2 * R * 1.3e-3, 2 * half_h * 1.5e-3)
    lsi = (2 * R * 1e-3, 2 * R * 1e-3, 2 * half_h * 1e-3)
    box = reference_space(space_si, lsi, r_max, 3.2)
    xyz, rad, rep = create_cylinder_sample(box.center.astype(np.float64), R, half_h, n, r_min, r_max, seed=seed,
                                           growth_stages=30, steps_per_stage=150, max_fire_steps=6000,
                                           overlap_tol=2e-3, device=device)
    size_real, center_real = bounding_box(xyz, rad.size, float(rad.max()), radii=rad)
    return xyz, rad, rep, box, size_real, center_real


@dataclass
class SweepCase:
    """One specimen under one parameter set, ready for add_sample."""
    specimen: int
    params: dict
    material: Material
    loading: object
    xyz: np.ndarray
    radii: np.ndarray
    index: int = 0          # position in the whole sweep

    @property
    def n(self) -> int:
        return self.radii.size


@dataclass
class Sweep:
    cases: list = field(default_factory=list)

    @property
    def particles(self) -> int:
        return sum(c.n for c in self.cases)


def build_sweep(n_cases: int, sizes: list[int], seed: int = 1, velocity_m_s: float = 0.1, max_steps: int = 0,
                device: int = 0, only=None) -> Sweep:
    """n_cases parameter sets (Latin hypercube) over len(sizes) packed
    cylinders (case k uses specimen k mod len(sizes)): uniaxial loading at
    velocity_m_s until the peak has passed (70% of it) or 1% strain.
    `only`: the case indices to build (a rank's shard); the parameter sets
    and per-case seeds are those of the whole sweep, and only the specimens
    these cases use are packed."""
    keep = range(n_cases) if only is None else sorted(set(int(k) for k in only))
    specs = {}
    for k in keep:
        i = k % len(sizes)
        if i not in specs:
            xyz, rad, rep, box, size_real, center_real = cylinder(sizes[i], seed * 1000 + i, device=device)
            specs[i] = (xyz, rad, box, size_real, center_real)
    params = latin_hypercube(n_cases, seed)
    sw = Sweep()
    for k in keep:
        p = params[k]
        xyz, rad, box, size_real, center_real = specs[k % len(sizes)]
        r_min, r_mean = float(rad.min()), float(rad.mean())
        ld = loading(TEST_UNIAXIAL, box, size_real, center_real, velocity=-velocity_m_s / VELOCITY, min_stress=0.010,
                     max_strain=0.01, cond_fracture=0.7, dNsave=100, max_steps=max_steps, p_r_platen=r_mean)
        sw.cases.append(SweepCase(k % len(sizes), p, material_for(p, r_min, r_mean, seed * 7919 + k), ld, xyz, rad,
                                  index=k))
    return sw


def shard(n_cases: int, rank: int, world: int) -> range:
    """The cases rank `rank` of `world` solves: a contiguous block, sizes
    differing by at most one.  Consecutive cases cycle through the specimens,
    so every block of at least len(sizes) cases holds every specimen size and
    the ranks' particle counts stay balanced."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world size {world}")
    return range(rank * n_cases // world, (rank + 1) * n_cases // world)


# per-case macro properties exchanged between ranks (dem_result fields)
MACRO_FIELDS = ("FractureStress", "FractureStrain", "E_chord", "nu", "Strain", "Stress", "Destruction", "dt", "steps",
                "bonds_initial", "bonds_now", "fracture", "done", "numeric")


def gather_results(local: dict, n_cases: int, group=None, device=None) -> list:
    """All-gather of the per-case macro properties of a sharded sweep: every
    rank passes {case index: result dict} for its own cases and receives the
    whole sweep's results in case order (MACRO_FIELDS of each).  One
    all_gather of a float64 table of ceil(n_cases / world) rows per rank;
    `device` is where the table lives (a CUDA device under the NCCL backend,
    the CPU under gloo).  With no process group (or world size 1) the local
    results are the whole sweep."""
    import torch
    import torch.distributed as td

    F = len(MACRO_FIELDS)
    world = td.get_world_size(group) if td.is_available() and td.is_initialized() else 1
    per = -(-n_cases // max(world, 1))
    if len(local) > per:
        raise ValueError(f"{len(local)} local cases, more than a rank's share {per} of {n_cases}")
    table = np.full((per, 1 + F), np.nan)
    for row, (k, res) in enumerate(sorted(local.items())):
        if not 0 <= k < n_cases:
            raise ValueError(f"case index {k} outside the sweep's {n_cases} cases")
        table[row, 0] = k
        table[row, 1:] = [float(res[f]) for f in MACRO_FIELDS]
    if world > 1:
        t = torch.from_numpy(table).to(device if device is not None else "cpu")
        parts = [torch.empty_like(t) for _ in range(world)]
        td.all_gather(parts, t, group=group)
        table = np.concatenate([p.cpu().numpy() for p in parts])
    out = [None] * n_cases
    for row in table:
        if np.isnan(row[0]):
            continue
        k = int(row[0])
        if out[k] is not None:
            raise RuntimeError(f"case {k} solved by two ranks")
        out[k] = {f: (int(v) if f in _INT_FIELDS else float(v)) for f, v in zip(MACRO_FIELDS, row[1:])}
    missing = [k for k, r in enumerate(out) if r is None]
    if missing:
        raise RuntimeError(f"cases {missing[:8]} solved by no rank")
    return out


_INT_FIELDS = {"steps", "bonds_initial", "bonds_now", "fracture", "done", "numeric"}


def run_sharded(n_cases: int, sizes: list[int], steps: int, rank: int, world: int, seed: int = 1,
                device: int = 0, group=None, gather_device=None, **kw) -> dict:
    """One sweep of n_cases cases split over `world` ranks (shard()): each
    rank packs and solves its block in one batched context, then the ranks
    exchange the per-case macro properties (gather_results()).  No data-path
    collective: the specimens are independent.  Returns this rank's device
    time and the whole sweep's results in case order."""
    sw = build_sweep(n_cases, sizes, seed=seed, device=device, only=shard(n_cases, rank, world), **kw)
    out = run_batched(sw, steps, device=device)
    local = {c.index: r for c, r in zip(sw.cases, out["results"])}
    return dict(device_ms=out["device_ms"], cases=[c.index for c in sw.cases],
                results=gather_results(local, n_cases, group=group, device=gather_device))


def run_batched(sw: Sweep, steps: int, device: int = 0, graph_steps: int = 200) -> dict:
    """All cases in one context; `steps` steps (finished cases stay frozen).
    Returns device time, wall time (set-up included) and per-case results."""
    t0 = time.perf_counter()
    ctx = Context(device=device, graph_steps=graph_steps)
    ids = [ctx.add_sample(c.material, c.loading, c.xyz, c.radii) for c in sw.cases]
    ctx.setup()
    ms = ctx.run_timed(steps)
    res = [ctx.result(i) for i in ids]
    ctx.close()
    return dict(device_ms=ms, wall_s=time.perf_counter() - t0, results=res)


def run_sequential(sw: Sweep, steps: int, device: int = 0, graph_steps: int = 200) -> dict:
    """The same cases one context at a time (the reference's one-specimen-per-run
    pattern on this engine)."""
    t0 = time.perf_counter()
    ms, res = 0.0, []
    for c in sw.cases:
        ctx = Context(device=device, graph_steps=graph_steps)
        ctx.add_sample(c.material, c.loading, c.xyz, c.radii)
        ctx.setup()
        ms += ctx.run_timed(steps)
        res.append(ctx.result(0))
        ctx.close()
    return dict(device_ms=ms, wall_s=time.perf_counter() - t0, results=res)
