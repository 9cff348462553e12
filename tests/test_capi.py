"""C ABI checks that need no GPU: the library builds and loads, exports every
function include/b200dem.h declares, and its host-only entry points (sample
and record files, error strings) behave as the reference's I/O does."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from dem_api import dem, ROOT

HEADER = ROOT / "include" / "b200dem.h"


def declared():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(dem_[a-z_0-9]+)\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    lib = dem.lib()
    names = declared()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", str(dem.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dem_[a-z_0-9]+)$", out, re.M))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert getattr(lib, n) is not None


def test_strerror_and_no_device_error():
    lib = dem.lib()
    assert lib.dem_strerror(0) == b"ok"
    assert b"skin" in lib.dem_strerror(-5)
    if dem.device_count() == 0:
        with pytest.raises(dem.DemError) as e:
            dem.Context()
        assert e.value.code == -2  # DEM_ERR_CUDA, no silent CPU path


def test_sample_file_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    n = 500
    xyz = rng.uniform(1.0, 9.0, 3 * n).astype(np.float32)
    hp = np.array([5.0, 5.0, 40.0])
    xyz_h = xyz.copy()
    xyz_h[7], xyz_h[n + 7], xyz_h[2 * n + 7] = hp  # a parked particle is skipped on save
    p = str(tmp_path / "Sample_0_0.txt")
    dem.save_cylinder_sample(p, xyz_h, hp)
    got, size, cen = dem.load_cylinder_sample(p, 0.25)
    keep = np.ones(n, bool)
    keep[7] = False
    ref = xyz.reshape(3, n)[:, keep]
    assert got.size == 3 * (n - 1)
    assert np.allclose(got.reshape(3, n - 1), ref, rtol=1e-6, atol=1e-6)
    # bounding box of h_LoadCylinderSample: extent + 2 p_r, centre of extent
    g = got.reshape(3, -1).astype(np.float64)
    assert np.allclose(size, g.max(1) - g.min(1) + 0.5)
    assert np.allclose(cen, 0.5 * (g.max(1) + g.min(1)))


def test_sample_file_errors(tmp_path):
    with pytest.raises(dem.DemError) as e:
        dem.load_cylinder_sample(str(tmp_path / "missing.txt"), 0.25)
    assert e.value.code == -6
    bad = tmp_path / "bad.txt"
    bad.write_text("10\n0.1 0.2 0.3\n0.4 nan 0.6\n")
    with pytest.raises(dem.DemError):
        dem.load_cylinder_sample(str(bad), 0.25)
    trunc = tmp_path / "trunc.txt"
    trunc.write_text("3\n0.1 0.2 0.3\n")
    with pytest.raises(dem.DemError):
        dem.load_cylinder_sample(str(trunc), 0.25)


def test_save_sum_forces_loading(tmp_path):
    rec = np.array([[0.0, -0.001, 0.002], [-1e-4, -0.01, 0.011]])
    p = tmp_path / "Uniaxial_0.txt"
    dem.save_sum_forces_loading(str(p), rec)
    lines = p.read_text().splitlines()
    assert lines[0] == "EpsZ StressZ_bottom StressZ_top"
    vals = np.array([[float(v) for v in l.split()] for l in lines[1:]])
    assert np.allclose(vals[:, 0], rec[:, 0])
    assert np.allclose(vals[:, 1:], rec[:, 1:] * 1e9)
