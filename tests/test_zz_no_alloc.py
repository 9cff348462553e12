"""dem_ref_cells_static, the binning entry point for callers that cannot
allocate GPU memory (cudaMalloc/cudaFree may synchronise the device, fail
under another framework's caching allocator, or be forbidden to a plug-in),
against dem_ref_cells on the same inputs.

Two calls in a row on different specimens (the larger first, so counters left
over from it would show in the second), each compared with dem_ref_cells;
outputs are integers, so the comparison is exact.  A second test runs a
case near the limits (60,000 random points in a 40 x 40 x 40 grid: 64,000
cells, so the cell scan takes its two-level path) and a small specimen after
it.  The size limits are checked before any device work and are tested
without a GPU.
"""
from __future__ import annotations

import numpy as np
import pytest

import dem_testlib as T
from dem_api import dem
from test_oracle_golden import SMALL, load

DEM_ERR_ARG, DEM_ERR_CAPACITY = -1, -4
MAX_PARTICLES, MAX_CELLS = 65536, 65536


def _call(xyz, n, a, nx, ny, nz):
    CI = np.zeros(max(n, 1), np.uint32)
    CIs = np.zeros(2 * max(n, 1), np.uint32)
    pnC = np.zeros(2 * nx * ny * nz, np.uint32) if nx * ny * nz <= 1 << 22 else None
    return dem.lib().dem_ref_cells_static(dem._p(xyz), n, a, nx, ny, nz, dem._p(CI), dem._p(CIs),
                                          None if pnC is None else dem._p(pnC))


def test_static_binning_rejects_sizes_beyond_its_scratch():
    xyz = np.zeros(3 * (MAX_PARTICLES + 1), np.float32)
    assert _call(xyz, MAX_PARTICLES + 1, 1.0, 4, 4, 4) == DEM_ERR_CAPACITY
    assert _call(xyz, 16, 1.0, 64, 64, 17) == DEM_ERR_CAPACITY      # 69632 cells
    assert _call(xyz, 16, 1.0, 1 << 11, 1 << 11, 1 << 11) == DEM_ERR_CAPACITY
    assert _call(xyz, 0, 1.0, 4, 4, 4) == DEM_ERR_ARG
    assert _call(xyz, 16, 0.0, 4, 4, 4) == DEM_ERR_ARG


@pytest.mark.gpu
def test_static_binning_matches_ref_cells_on_two_calls_in_a_row():
    big = T.ref_case(seed=3)                 # default specimen: more particles and cells than SMALL
    small = T.ref_case(seed=1, **SMALL)
    assert big.N > small.N and big.N <= MAX_PARTICLES
    for c in (big, small):
        cells = (c.cells.a, c.cells.nx, c.cells.ny, c.cells.nz)
        assert c.cells.nx * c.cells.ny * c.cells.nz <= MAX_CELLS
        want = dem.ref_cells(c.R, *cells)
        got = dem.ref_cells_static(c.R, *cells)
        for w, g in zip(want, got):
            assert np.array_equal(w, g)
    g = load("cells_il_s1")
    CI, CIs, pnC = got
    assert np.array_equal(CI, g["CI"]) and np.array_equal(CIs, g["CIs"]) and np.array_equal(pnC, g["pnC"])


@pytest.mark.gpu
def test_static_binning_near_its_limits_then_small():
    rng = np.random.default_rng(7)
    n, g, a = 60000, 40, 1.0
    xyz = np.ascontiguousarray(rng.uniform(0.0, g * a, 3 * n).astype(np.float32))
    assert n <= MAX_PARTICLES and g ** 3 <= MAX_CELLS and g ** 3 > 1024   # two scan levels
    small = T.ref_case(seed=1, **SMALL)
    cases = [(xyz, (a, g, g, g)), (small.R, (small.cells.a, small.cells.nx, small.cells.ny, small.cells.nz))]
    for _ in range(2):                     # twice: each call starts from the other's leftovers
        for pts, cells in cases:
            want = dem.ref_cells(pts, *cells)
            got = dem.ref_cells_static(pts, *cells)
            for w, h in zip(want, got):
                assert np.array_equal(w, h)
    CI, CIs, pnC = got
    assert int(pnC[small.cells.nx * small.cells.ny * small.cells.nz:].sum()) == small.N
