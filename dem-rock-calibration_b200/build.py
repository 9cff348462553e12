"""Build of the product library libb200dem.so (sm_100a) in place.

    python dem-rock-calibration_b200/build.py

nvcc compiles the CUDA kernels and host engine for sm_100a only.  -fmad=false
keeps every a*b+c as two rounded operations (the arithmetic contract of the
kernels); host code is built with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SRC = PKG / "csrc"
OUT = PKG / "libb200dem.so"
CLI = PKG / "rockfit-dem"  # the reference's command line over the library (csrc/rockfit_cli.cpp)

SOURCES = ["dem_engine.cu", "dem_pack.cu", "dem_noalloc.cu", "dem_mlp.cu", "dem_capi.cpp"]
HEADERS = ["dem_common.cuh", "dem_dual.cuh", "dem_types.h", "dem_step.cuh", "dem_build.cuh", "dem_pack.cuh", "dem_params.h",
           "dem_engine.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-O3",
    "-shared",
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def stale() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [SRC / s for s in SOURCES + HEADERS + ["rockfit_cli.cpp"]] + [ROOT / "include" / "b200dem.h"]
    return not CLI.exists() or any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra=()) -> Path:
    """Compiles every source to an object in parallel (one nvcc per file; no
    device code crosses files), then links the shared library."""
    if not force and not stale():
        return OUT
    # nvcc's host compiler: the system g++ (a wrapper in CXX may lack parts of the toolchain)
    ccbin = ["-ccbin", "/usr/bin/g++"] if Path("/usr/bin/g++").exists() else []
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs = []
    for src in SOURCES:
        obj = objdir / (src + ".o")
        cmd = [nvcc(), *ccbin, *flags, *extra, "-I", str(ROOT / "include"), "-I", str(SRC), "-c", str(SRC / src),
               "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for src, obj, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode != 0:
            sys.stderr.write(out)
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("libb200dem build failed")
    cmd = [nvcc(), *ccbin, "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
           *[str(objdir / (s + ".o")) for s in SOURCES], "-o", str(OUT) + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("libb200dem link failed")
    os.replace(str(OUT) + ".tmp", OUT)
    build_cli()
    return OUT


def build_cli() -> Path:
    """rockfit-dem, linked against the in-tree library (rpath $ORIGIN)."""
    gxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    cmd = [gxx, "-O2", "-std=c++17", "-I", str(ROOT / "include"), str(SRC / "rockfit_cli.cpp"), "-o", str(CLI) + ".tmp",
           "-L", str(PKG), "-lb200dem", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("rockfit-dem build failed")
    os.replace(str(CLI) + ".tmp", CLI)
    return CLI


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose=True,
              extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
    print(p)
