"""The CPU restatement of the engine's packer (oracle/dem_pack_oracle.c) on
its own, without a GPU: a seeded packing repeats exactly, relaxes below its
overlap tolerance at about the requested packing fraction, keeps every
sphere inside the cylinder, and its FIRE time step and mixing follow the
adaptation rule of md_createcylindersample.cu:374-397 (grow by 1.1 and shrink
alpha by 0.99 after more than Ndelay = 20 steps of positive power, halve dt
and reset alpha on non-positive power after the first Ndelay steps, within
[dtmin, dtmax])."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pack

ARGS = ((3.0, 3.0, 5.0), 2.0, 4.0, 850, 0.20, 0.30)


def _run(variant, **over):
    kw = dict(E=50.0, nu=0.25, rho=2.65, overlap_tol=2e-3, growth_stages=12, steps_per_stage=120,
              max_fire_steps=1500, seed=11, fire_variant=variant, trace_cap=4000)
    kw.update(over)
    return pack.create_cylinder_sample(*ARGS, **kw)


def test_cpu_packing_repeats_and_relaxes():
    a = _run(0)
    b = _run(0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    xyz, rad, rep = a
    assert rep["max_overlap"] < 2e-3
    assert 0.5 < rep["packing_fraction"] < 0.62
    assert rad.min() >= 0.20 and rad.max() <= 0.30
    x, y, z = xyz.reshape(3, -1).astype(np.float64)
    c, R, H = ARGS[0], ARGS[1], ARGS[2]
    assert np.all(np.hypot(x - c[0], y - c[1]) <= R + 1e-5) and np.all(np.abs(z - c[2]) <= H + 1e-5)


@pytest.mark.parametrize("variant", [0, 1])
def test_fire_adaptation_rule(variant):
    _, _, rep = _run(variant, max_fire_steps=800, overlap_tol=1e-9)
    tr = rep["fire_trace"]
    assert len(tr) == 800
    dt, alpha, back = tr[:, 0], tr[:, 1], tr[:, 2].astype(bool)
    r, rho, E, nu = 0.20, 2.65, 50.0, 0.25
    dt0 = 0.05 * (np.pi * r * np.sqrt(2.0 * rho * (1.0 + nu)) / (np.sqrt(E) * (0.163 * nu + 0.8766)))
    alpha0, (dtmin, dtmax) = (0.1, (0.001 * dt0, 100.0 * dt0)) if variant == 1 else (0.25, (0.02 * dt0, 4.0 * dt0))
    prev_dt, prev_alpha, npos = dt0, alpha0, 0
    grew = shrank = 0
    for k in range(len(tr)):
        if not back[k]:
            npos += 1
            if npos > 20:
                assert dt[k] == (prev_dt * 1.1 if prev_dt * 1.1 < dtmax else dtmax), k
                assert alpha[k] == prev_alpha * 0.99, k
                grew += 1
            else:
                assert dt[k] == prev_dt and alpha[k] == prev_alpha, k
        else:
            npos = 0
            if k > 20:
                assert dt[k] == (prev_dt * 0.5 if prev_dt * 0.5 > dtmin else dtmin), k
                assert alpha[k] == alpha0, k
                shrank += 1
            else:
                assert dt[k] == prev_dt and alpha[k] == prev_alpha, k
        prev_dt, prev_alpha = dt[k], alpha[k]
    assert grew > 0
