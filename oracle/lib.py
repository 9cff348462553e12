"""ctypes bindings of the CPU oracle (oracle/_build/libdemoracle.so) and of the
reference harness (oracle/_ref/libdemref.so).  Test infrastructure only.

All arrays are numpy arrays in the reference layout (see dem_oracle.h);
float32 arrays select the *_f functions and float64 the *_d functions.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libdemoracle.so"
REF_SO = HERE / "_ref" / "libdemref.so"
EMPTY = 0xFFFFFFFF

_lib = None
_ref = None


def build(ref: bool = False) -> None:
    """Compile the oracle (and, where the reference tree exists, the reference harness)."""
    subprocess.run(["make", "-s", "oracle"], cwd=HERE, check=True)
    if ref:
        subprocess.run(["make", "-s", "-j8", "ref"], cwd=HERE, check=True)


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build()
        _lib = C.CDLL(str(ORACLE_SO))
        _declare(_lib)
    return _lib


def ref_available() -> bool:
    return REF_SO.exists()


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(str(REF_SO), mode=os.RTLD_NOW)
        _declare_ref(_ref)
    return _ref


def P(a):
    """Data pointer of a numpy array (or NULL), as an integer: every function
    it is passed to declares the argument c_void_p, and the caller keeps the
    array alive for the call."""
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data


_vp = C.c_void_p
_u32 = C.c_uint32


class Compress(C.Structure):
    _fields_ = [
        ("brazil", C.c_int),
        ("size_d", C.c_double * 3), ("center_d", C.c_double * 3),
        ("Top", C.c_double), ("Bottom", C.c_double), ("TopR", C.c_double), ("BottomR", C.c_double),
        ("Size0", C.c_double),
        ("V", C.c_double), ("VLoad", C.c_double), ("Area", C.c_double), ("inv_Area", C.c_double),
        ("MinStress", C.c_double), ("ZeroStress", C.c_double), ("MaxStrain", C.c_double),
        ("ConditionFracture", C.c_double),
        ("Stress", C.c_double), ("Strain", C.c_double), ("FractureStress", C.c_double),
        ("FractureStrain", C.c_double), ("LinearityDeviation", C.c_double),
        ("StepsStop", C.c_uint32), ("Loading", C.c_int), ("Fracture", C.c_int),
        ("sFL", C.c_double * 2), ("sz0", C.c_double),
        ("dNsave", C.c_uint32), ("Nsave", C.c_uint32), ("stepsave", C.c_uint32),
        ("h_sFL", C.POINTER(C.c_double)), ("h_sSI", C.POINTER(C.c_uint32)),
    ]


def _declare(L):
    for sfx, R in (("f", C.c_float), ("d", C.c_double)):
        g = lambda n: getattr(L, f"{n}_{sfx}")
        g("orc_cell_distribution").argtypes = [_vp, _u32, R, _u32, _u32, _u32, _vp, _vp, _vp]
        g("orc_il_construct").argtypes = [_vp, _u32, _vp, _vp, _vp, _u32, R, R, R, _u32, _u32, _u32]
        g("orc_il_construct").restype = C.c_int64
        g("orc_il_reconstruct_bpm").argtypes = [_vp, _u32, _vp, _vp, _vp, _vp, _u32, R, R, R, _u32, _u32, _u32]
        g("orc_il_reconstruct_bpm").restype = C.c_int64
        g("orc_delete_far_links").argtypes = [_vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _u32, R]
        g("orc_construct_bonds").argtypes = [_vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u32, R, _vp,
                                             C.c_double]
        g("orc_forces_bpm").argtypes = [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u32,
                                        R, R, R, R, R, R, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int]
        g("orc_forces_hm").argtypes = [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _u32, R, R, R, R, R, R, R,
                                       R, _vp, _vp, _vp, _vp, _vp]
        g("orc_platen").argtypes = [C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _u32, R, R, R, R, R, R, R, R, _vp, _vp,
                                    _vp, R, R, R, R, R, _vp, _vp]
        g("orc_forces_bpm_q").argtypes = [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u32, R, R, R,
                                          R, R, R, _vp, _vp, _vp, C.c_int, _vp, _vp]
        g("orc_forces_hm_q").argtypes = [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _u32, R, R, R, R, R, R, R, R, _vp,
                                         _vp, _vp, _vp]
        g("orc_fix_to_real").argtypes = [_vp, _vp, C.c_uint64]
        g("orc_platen_q").argtypes = [C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _u32, R, R, R, R, R, R, R, R, _vp,
                                      _vp, _vp, R, R, R, R, R, _vp]
        g("orc_increments").argtypes = [_vp, _vp, _vp, _vp, _vp, _u32, R, R, R, _vp, _vp]
        g("orc_cut_restriction").argtypes = [_vp, _vp, _vp, _u32, _vp, _vp, _vp]
        g("orc_soft_forces").argtypes = [_vp, _vp, _u32, _vp, _vp, _u32, R, R, _vp]
        g("orc_fire_increments").argtypes = [_vp, _vp, _vp, _u32, R, R, R, _vp]
        g("orc_fire_half_step_back").argtypes = [_vp, _vp, _u32, R]
        g("orc_fdotv").argtypes = [_vp, _vp, _u32]
        g("orc_fdotv").restype = C.c_double
        g("orc_increments_viscous").argtypes = [_vp, _vp, _vp, _u32, R, R, R, _vp]
        g("orc_cylinder_restriction_z").argtypes = [_vp, _vp, _u32, _vp, R, R, R]
    L.orc_rsqrt_rn_f.argtypes = [C.c_float]
    L.orc_rsqrt_rn_f.restype = C.c_float
    L.orc_count_bonds.argtypes = [_vp, _vp, C.c_uint64]
    L.orc_count_bonds.restype = C.c_uint64
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_get_threads.restype = C.c_int
    L.orc_compress_init.argtypes = [C.POINTER(Compress), C.c_int, _vp, _vp, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double]
    L.orc_sum_forces.argtypes = [C.POINTER(Compress), _u32]
    L.orc_sum_interactions.argtypes = [C.POINTER(Compress), C.c_uint64, _u32]
    L.orc_compress_s3.argtypes = [C.POINTER(Compress), C.c_double, C.c_double]
    L.orc_linearity_deviation.argtypes = [C.POINTER(Compress)]
    L.orc_linearity_deviation.restype = C.c_double
    L.orc_destruction.argtypes = [C.POINTER(Compress)]
    L.orc_destruction.restype = C.c_double


class StepParams(C.Structure):
    _fields_ = [
        ("a", C.c_float), ("nx", _u32), ("ny", _u32), ("nz", _u32), ("IonP", _u32),
        ("il_aacut", C.c_float), ("aa_farcut", C.c_float),
        ("dt", C.c_float), ("m_E", C.c_float), ("m_G", C.c_float), ("b_r", C.c_float), ("m_Ec", C.c_float),
        ("m_Gc", C.c_float),
        ("hm_E", C.c_float), ("hm_G", C.c_float), ("p_A", C.c_float), ("p_mu", C.c_float), ("p_mur", C.c_float),
        ("p_m", C.c_float), ("p_r", C.c_float),
        ("wall_E", C.c_float), ("wall_G", C.c_float),
        ("center", C.c_float * 3),
        ("wall_RR", C.c_float), ("wall_top", C.c_float), ("wall_bot", C.c_float), ("wall_V", C.c_float),
        ("Zcut", C.c_float),
        ("dt_d_m", C.c_float), ("dt_d_I", C.c_float),
        ("s_center", C.c_float * 3), ("s_spacesized2", C.c_float * 3), ("hidenpoint", C.c_float * 3),
        ("brazil", C.c_int), ("stages", C.c_int),
    ]


class TestParams(C.Structure):
    _fields_ = [
        ("E", C.c_double), ("Ec", C.c_double), ("Gc", C.c_double), ("b_r", C.c_double), ("gap", C.c_double),
        ("p_r_m", C.c_double), ("rho", C.c_double), ("nu", C.c_double), ("p_e", C.c_double), ("p_mu", C.c_double),
        ("p_mur", C.c_double), ("farcut_factor", C.c_double),
        ("space_si", C.c_double * 3), ("lsi", C.c_double * 3),
        ("velocity_si", C.c_double), ("minstress_si", C.c_double), ("maxstrain", C.c_double),
        ("condfract", C.c_double),
        ("dNsave", _u32), ("fileN", _u32), ("isample", _u32),
    ]


class TestResult(C.Structure):
    _fields_ = [
        ("FractureStress", C.c_double), ("FractureStrain", C.c_double), ("LinearityDeviation", C.c_double),
        ("Destruction", C.c_double), ("Strain", C.c_double), ("dt", C.c_double), ("seconds", C.c_double),
        ("steps_hint", C.c_uint64), ("N", _u32), ("stepsave", _u32),
    ]


def _declare_ref(L):
    L.refh_cell_distribution.argtypes = [_vp, _u32, C.c_float, _u32, _u32, _u32, _vp, _vp, _vp]
    L.refh_setup_bonds.argtypes = [_vp, _u32, C.c_float, _u32, _u32, _u32, _u32, C.c_float, C.c_float, C.c_float,
                                   C.c_float, _vp, _vp, _vp]
    L.refh_step.argtypes = [C.POINTER(StepParams), _u32] + [_vp] * 14
    L.refh_time_steps.argtypes = [C.POINTER(StepParams), _u32] + [_vp] * 6 + [_u32, C.c_int, C.POINTER(C.c_double)]
    L.refh_cg_start_parameters.argtypes = [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_double, _vp, _vp]
    L.refh_cg_new_parameters2.argtypes = [_vp] * 7 + [C.c_int, C.c_double, _vp, _vp]
    L.refh_run_test.argtypes = [C.c_int, C.c_char_p, C.c_char_p, C.POINTER(TestParams), C.POINTER(TestResult)]
    L.refh_time_bpm_cpu.argtypes = [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _u32] + [C.c_float] * 5 + [
        C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]


def sfx(a) -> str:
    return "d" if a.dtype == np.float64 else "f"


def fn(name: str, like):
    return getattr(lib(), f"{name}_{sfx(like)}")
