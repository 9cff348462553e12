"""The Python mirrors of the C ABI's structs have the layout that
include/b200dem.h gives them: the ctypes Structures of the host API
(dem-rock-calibration_b200/__init__.py) and the numpy record of the
surrogate's Adam descriptor list (dem_mlp_tensor) put every field at the
offset the C compiler does and have the same size.  A small C program
compiled against the header with the host compiler prints the C side.  No
GPU is needed."""
from __future__ import annotations

import ctypes as C
import importlib
import shutil
import subprocess

import pytest

from dem_api import ROOT, dem

S = importlib.import_module("dem-rock-calibration_b200.surrogate")

MIRRORS = [("dem_options", dem.Options), ("dem_material", dem.Material), ("dem_loading", dem.Loading),
           ("dem_result", dem.Result), ("dem_sensitivity", dem.Sensitivity), ("dem_tune_report", dem.TuneReport),
           ("dem_pack_params", dem.PackParams), ("dem_pack_report", dem.PackReport)]


def _c_layout(tmp_path, items):
    """items: (C type, [field names]) -> {C type: (sizeof, {field: offsetof})}."""
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "b200dem.h"', "int main(void) {"]
    for t, fields in items:
        lines.append(f'  printf("{t} . %zu\\n", sizeof({t}));')
        for f in fields:
            lines.append(f'  printf("{t} {f} %zu\\n", offsetof({t}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    subprocess.run([cc, "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        t, f, v = line.split()
        entry = out.setdefault(t, [0, {}])
        if f == ".":
            entry[0] = int(v)
        else:
            entry[1][f] = int(v)
    return out


def test_ctypes_structs_match_the_header(tmp_path):
    items = [(t, [f[0] for f in cls._fields_]) for t, cls in MIRRORS]
    c = _c_layout(tmp_path, items)
    for t, cls in MIRRORS:
        size, offs = c[t]
        assert C.sizeof(cls) == size, t
        for f, *_ in cls._fields_:
            assert getattr(cls, f).offset == offs[f], (t, f)


def test_adam_descriptor_record_matches_dem_mlp_tensor(tmp_path):
    d = S.ADAM_TENSOR_DTYPE
    c = _c_layout(tmp_path, [("dem_mlp_tensor", list(d.names))])
    size, offs = c["dem_mlp_tensor"]
    assert d.itemsize == size
    for f in d.names:
        assert d.fields[f][1] == offs[f], f
