"""The GPU packer (dem_create_cylinder_sample: seeded fill, radius growth with
viscous relaxation, FIRE relaxation; the role of the reference's
h_CreateCylinderSample, md_createcylindersample.cu:184-439) against its CPU
restatement (oracle/dem_pack_oracle.c), on a column and a disc, with FIRE 2.0
and with the reference's FIRE update (md_firerelaxation.cu:18-70 and the
dt / alpha adaptation of md_createcylindersample.cu:368-397).

For the reference's FIRE update the CPU side moves the spheres with the
oracle's restatements of the reference kernels themselves
(orc_fire_half_step_back, orc_fire_increments: d_CalculateDecrementsHalfStepFIRE
and d_CalculateIncrementsFIRE), so this also pins the GPU packer's FIRE
update to the reference's.

Pair forces are summed in fixed point on both sides and every other
operation is rounded the same way, so the packings must agree bit for bit:
positions, radii, step count, list rebuilds and the final largest overlap.
Thousands of FIRE steps of a chaotic relaxation make this a strict check of
every kernel of the packer and of its host schedule.
"""
from __future__ import annotations

import numpy as np
import pytest

from dem_api import dem
from oracle import pack

pytestmark = pytest.mark.gpu

SHAPES = {
    # centre, radius, half height, spheres, r_min, r_max
    "column": ((3.0, 3.0, 5.0), 2.0, 4.0, 850, 0.20, 0.30),
    "disc": ((6.0, 6.0, 3.0), 5.0, 2.5, 3800, 0.18, 0.30),
}


@pytest.mark.parametrize("variant", [0, 1], ids=["fire2", "reference_fire"])
@pytest.mark.parametrize("shape", list(SHAPES))
def test_gpu_packing_equals_cpu_restatement(shape, variant):
    args = SHAPES[shape]
    kw = dict(E=50.0, nu=0.25, rho=2.65, overlap_tol=2e-3, growth_stages=12, steps_per_stage=120,
              max_fire_steps=1500, seed=11, fire_variant=variant)
    gx, gr, grep = dem.create_cylinder_sample(*args, **kw)
    cx, cr, crep = pack.create_cylinder_sample(*args, **kw)
    assert np.array_equal(gr, cr)
    diff = np.abs(gx.astype(np.float64) - cx)
    assert np.array_equal(gx, cx), (int(np.count_nonzero(diff)), float(diff.max()))
    assert grep == crep, (grep, crep)
    print(f"\n{shape}/fire variant {variant}: {args[3]} spheres, {grep['steps']} steps, "
          f"{grep['rebuilds']} list builds, largest overlap {grep['max_overlap']:.2e}: identical")
