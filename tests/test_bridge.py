"""The reference-side binding (dem-rock-calibration_b200/bridge/md_b200_bridge.cpp)
compiles against the reference's own headers (md_data_types.h, mp.h) and links
against libb200dem with no undefined symbol, and it defines the two driver
entry points with the signatures mp.h declares (mp.h:21-22), so the
reference's kernel.cu and mp_*.cu link against it unchanged.  Needs the
reference checkout (DEM_REFERENCE_DIR, or a directory named `reference`
beside this repository) and a host C++ compiler; no GPU."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

from dem_api import ROOT, dem


def _reference_dir():
    for c in (os.environ.get("DEM_REFERENCE_DIR"), str(ROOT.parent / "reference")):
        if c and (Path(c) / "md_data_types.h").exists() and (Path(c) / "mp.h").exists():
            return Path(c)
    return None


def _cuda_include():
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and (Path(c) / "include" / "cuda.h").exists():
            return Path(c) / "include"
    return None


@pytest.mark.skipif(_reference_dir() is None or _cuda_include() is None or shutil.which("g++") is None,
                    reason="reference checkout, CUDA headers or g++ not available")
def test_bridge_compiles_and_links_against_the_library(tmp_path):
    dem.lib()                                   # builds the library if needed
    src = ROOT / "dem-rock-calibration_b200" / "bridge" / "md_b200_bridge.cpp"
    obj, so = tmp_path / "bridge.o", tmp_path / "libbridge.so"
    subprocess.run(["g++", "-std=c++17", "-fPIC", "-c", "-I", str(ROOT / "include"), "-I", str(_reference_dir()),
                    "-I", str(_cuda_include()), str(src), "-o", str(obj)], check=True, capture_output=True)
    subprocess.run(["g++", "-shared", str(obj), "-L", str(ROOT / "dem-rock-calibration_b200"), "-lb200dem",
                    "-Wl,--no-undefined", "-o", str(so)], check=True, capture_output=True)
    syms = subprocess.run(["nm", "-D", "--defined-only", str(so)], check=True, capture_output=True,
                          text=True).stdout
    # void h_CalculationUniaxialCompression(md_task_data&, float*) and the Brazilian twin
    assert "_Z32h_CalculationUniaxialCompressionR12md_task_dataPf" in syms
    assert "_Z23h_CalculationBrazilTestR12md_task_dataPf" in syms
