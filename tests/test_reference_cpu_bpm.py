"""The reference's CPU BPM routine (h_CalculateForceElastic,
md_calculateforcesbpm_cpu.cu:20-262) as timed by bench.py: the harness in
oracle/_ref calls it once per directed bond slot with stdout and stderr sent
to /dev/null, and restores both afterwards.  Timing only (the routine's
maths differs from the GPU path the reference runs); no GPU needed."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import lib as L


def _ref():
    try:
        return L.ref()
    except OSError as e:
        pytest.skip(f"oracle/_ref not built: {e}")


def test_reference_cpu_bpm_timing_runs_silently(capfd):
    R = _ref()
    rng = np.random.default_rng(0)
    n = 500
    pos = rng.uniform(0, 10, (n, 3)).astype(np.float32)
    Rs = np.ascontiguousarray(pos.T.reshape(-1))
    V = np.zeros(3 * n, np.float32)
    W = np.zeros(3 * n, np.float32)
    bi = np.arange(0, n - 1, dtype=np.uint32)
    bj = bi + 1
    br = np.full(bi.size, 0.2, np.float32)
    ev, sec = C.c_double(), C.c_double()
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = R.refh_time_bpm_cpu(P(Rs), P(V), P(W), n, P(bi), P(bj), P(br), bi.size, 1e-3, 30.0, 12.0, 0.04, 0.04,
                             0.2, C.byref(ev), C.byref(sec))
    assert rc == 0 and sec.value >= 0.2 and ev.value > 0
    out, err = capfd.readouterr()
    assert out == "" and err == ""
    print("after")
    out, _ = capfd.readouterr()
    assert out == "after\n"
