"""rockfit-dem, the reference's command line (kernel.cu:23-123,
mp_calculateonesample.cu:17-250) over the library: argument parsing and the
stdout lines NN_MP.py reads (CPU), and one create + uniaxial run (GPU)."""
from __future__ import annotations

import re
import subprocess

import numpy as np
import pytest

from dem_api import dem

RESULT = re.compile(r"ResultCalculateOneSample\[([^\]]*)\]")


def _cli():
    dem.lib()  # builds the library and the command line when stale
    import importlib
    return str(importlib.import_module("dem-rock-calibration_b200.build").CLI)


def test_reference_space_matches_python():
    import ctypes as C
    for space, lsi, p_r in (((0.04, 0.04, 0.06), (0.025, 0.025, 0.05), 0.5),
                            ((0.009, 0.009, 0.013), (0.0045, 0.0045, 0.007), 0.25)):
        ld = dem.Loading()
        dem.lib().dem_reference_space((C.c_double * 3)(*space), (C.c_double * 3)(*lsi), p_r, 3.2, C.byref(ld))
        box = dem.reference_space(space, lsi, p_r, 3.2)
        assert np.array_equal(np.array(ld.space_center[:]), box.center.astype(np.float64))
        assert np.array_equal(np.array(ld.space_half[:]), box.half.astype(np.float64))
        assert np.array_equal(np.array(ld.hidden_point[:]), box.hidden_point.astype(np.float64))
        assert ld.zcut == box.zcut


def test_cli_contract_without_tests(tmp_path):
    r = subprocess.run([_cli(), "I7", "M(6e10,4e7,4e7,2e-4,2.5e-5,0.375)"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0
    assert re.search(r"^There are \d+ GPUs$", r.stdout, re.M) and "INDEX 7" in r.stdout
    vals = [float(v) for v in RESULT.search(r.stdout).group(1).split(",")]
    # no test requested: the defaults CalculateOneSample reports for skipped tests
    assert vals == [6e10, 4e7, 4e7, 2e-4, 2.5e-5, 0.375, 1e-2, 1e6, 1.0, 1.0, 1e-2, 1e6, 0.0, 1.0]
    bad = subprocess.run([_cli(), "M(6e10,4e7)"], cwd=tmp_path, capture_output=True, text=True)
    assert bad.returncode == 1


@pytest.mark.gpu
def test_cli_creates_and_tests_a_uniaxial_sample(tmp_path):
    r = subprocess.run([_cli(), "G0", "M(3e10,4e7,4e7,2e-4,2.5e-5,0.45)", "CSU", "I1"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Correct GPU request! Requested: 0" in r.stdout and "INDEX 1" in r.stdout
    vals = [float(v) for v in RESULT.search(r.stdout).group(1).split(",")]
    assert len(vals) == 14 and all(np.isfinite(vals))
    assert vals[5] >= 0.45 and vals[7] > 1e6 and 0 < vals[6] <= 0.01
    assert (tmp_path / "result" / "Sample_0_1.txt").exists() and (tmp_path / "result" / "Uniaxial_1.txt").exists()
