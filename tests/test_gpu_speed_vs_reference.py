"""Speed of the engine's step against the reference's own CUDA step on the
same B200, same specimen (the reference-GPU baseline).

Specimen: the Brazilian disc 40 mm x 20 mm in reference mode (equal radii
0.25 mm on a non-overlapping FCC lattice, about 2.9e5 spheres), so the
reference kernels run it unchanged.  The reference's loop body (cell sort and
interaction-list rebuild, DEM_22 + DEM_21 forces, platen contacts with the
per-step host copy of the platen sums, integration, escape restriction,
far-link deletion; md_calculationbraziltest.cu:185-231) is timed with CUDA
events through oracle/_ref; the engine's step through dem_run_timed.  Both
start from the same bonded state at rest.  The engine must be faster; the
numbers are printed (pytest -s) for the record.
"""
from __future__ import annotations

import numpy as np
import pytest

import dem_testlib as T
from dem_api import dem
from oracle import lib as L
from oracle import sim
from test_gpu_parity import _loading, _material

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not L.ref_available(), reason="reference harness not built")
def test_engine_step_faster_than_reference_kernels():
    c = T.ref_case(seed=4, lsi=(0.040, 0.040, 0.020), space=(0.052, 0.052, 0.030), jitter_frac=0.1,
                   lattice_gap=0.5, brazil=True, velocity_si=-0.02, minstress_si=2.1e6, maxstrain=0.03)
    n = c.N
    # reference: its own set-up kernels, then its loop body
    st = sim.RefState.empty(n)
    st.R[:] = c.R
    sim.ref_setup_bonds(st, c.sc)
    ref_steps = 100
    sim.ref_time_steps(st, c.sc, 5)  # warm-up (allocations, module load)
    ref_ms = sim.ref_time_steps(st, c.sc, ref_steps) / ref_steps
    ref_kernels_ms = sim.ref_time_steps(st, c.sc, ref_steps, sync_fl=False) / ref_steps
    # engine: the same positions, reference-mode material and Brazilian loading
    ctx = dem.Context(graph_steps=200)
    ctx.add_sample(_material(c), _loading(c), c.R)
    ctx.setup()
    ctx.run_timed(200)
    steps = 2000
    our_ms = ctx.run_timed(steps) / steps
    prof = ctx.profile(200)
    res = ctx.result(0)
    ctx.close()
    print(f"\nreference-mode disc: {n} spheres, {res['bonds_initial']} bonds")
    print(f"reference kernels (oracle/_ref): {ref_ms * 1e3:.1f} us/step with the per-step platen copy, "
          f"{ref_kernels_ms * 1e3:.1f} us/step kernels only -> {n / (ref_ms * 1e-3):.3e} particle-steps/s")
    print(f"engine: {our_ms * 1e3:.1f} us/step (pair kernel {prof['pair_ms'] * 1e3:.1f} us, particle kernel "
          f"{prof['particle_ms'] * 1e3:.1f} us) -> {n / (our_ms * 1e-3):.3e} particle-steps/s; "
          f"speed-up {ref_ms / our_ms:.1f}x (kernels only {ref_kernels_ms / our_ms:.1f}x)")
    assert res["stale"] == 0
    assert our_ms < ref_kernels_ms
