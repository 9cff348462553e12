"""Batched sweeps: the Latin hypercube (CPU) and batched == one-at-a-time
(GPU): specimens that share one context advance exactly as they do alone, up
to the summation order of their pair forces."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from dem_api import dem  # noqa: F401  (loads the package)

sweep = importlib.import_module("dem-rock-calibration_b200.sweep")


def test_latin_hypercube_strata_and_bounds():
    n = 64
    pts = sweep.latin_hypercube(n, seed=3)
    assert len(pts) == n
    for name, (lo, hi) in sweep.SWEEP_SPACE.items():
        v = np.array([p[name] for p in pts])
        assert np.all(v >= lo) and np.all(v <= hi)
        strata = np.floor((v - lo) / (hi - lo) * n).astype(int)
        assert sorted(strata.tolist()) == list(range(n))  # one point per stratum
    again = sweep.latin_hypercube(n, seed=3)
    assert all(a == b for a, b in zip(pts, again))
    assert sweep.latin_hypercube(n, seed=4)[0] != pts[0]


def test_material_for_maps_the_parameters():
    p = dict(E_bond=33.0, kn_ks=2.0, strength=0.05, strength_sd=0.2, mu=0.4, bond_radius_factor=0.7)
    m = sweep.material_for(p, 0.2, 0.25, seed=9)
    assert (m.E_bond, m.kn_ks, m.Ec, m.Gc, m.mu, m.bond_radius_factor) == (33.0, 2.0, 0.05, 0.05, 0.4, 0.7)
    assert m.Ec_sd == pytest.approx(0.01) and m.Gc_sd == pytest.approx(0.01) and m.seed == 9


@pytest.mark.gpu
def test_batched_equals_sequential():
    sw = sweep.build_sweep(6, sizes=[3000, 5000, 8000], seed=2)
    steps = 600  # about 0.2% strain: before the first bonds break
    b = sweep.run_batched(sw, steps)
    s = sweep.run_sequential(sw, steps)
    for rb, rs in zip(b["results"], s["results"]):
        assert rb["steps"] == rs["steps"]
        assert rb["platen_top"] == pytest.approx(rs["platen_top"], rel=0, abs=1e-9)
        assert rb["Stress"] == pytest.approx(rs["Stress"], rel=2e-2, abs=1e-6)
        assert rb["bonds_now"] == pytest.approx(rs["bonds_now"], rel=1e-3, abs=2)
