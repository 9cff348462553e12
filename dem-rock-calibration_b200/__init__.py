"""Python host API of the B200 DEM library (ctypes over include/b200dem.h).

The product is libb200dem.so (CUDA for sm_100a + C++ host engine).  This
module loads it, mirrors the C structs, and offers a small object API:

    ctx = Context()
    sid = ctx.add_sample(material, loading, xyz, radii)
    ctx.setup(); ctx.run(max_steps); ctx.result(sid)

It fails loudly when the library is missing or no CUDA device is present;
there is no CPU fallback.  Units are the reference's (mm, mg, us; GPa).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libb200dem.so"
EMPTY = 0xFFFFFFFF

TEST_NONE, TEST_UNIAXIAL, TEST_BRAZIL = 0, 1, 2
STAGE_PAIRS, STAGE_PARTICLES, STAGE_KEEP_FORCES = 1, 2, 4

LENGTH = 1e-3          # m per mm
STRESS = 1e9           # Pa per GPa
DENSITY = 1e3          # (kg/m^3) per (mg/mm^3)
VELOCITY = 1e3         # (m/s) per (mm/us)


class DemError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        msg = _lib().dem_strerror(code).decode() if _LIB else str(code)
        if code == -2 and _LIB:
            msg += ": " + _lib().dem_last_error_detail().decode()
        super().__init__(f"{where}: {msg} ({code})" if where else f"{msg} ({code})")


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("pair_block", C.c_uint32),
                ("pair_grid", C.c_uint32), ("particle_block", C.c_uint32), ("graph_steps", C.c_uint32),
                ("skin_factor", C.c_double), ("pair_min_blocks", C.c_uint32), ("deterministic", C.c_uint32)]


class Material(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("Ec", C.c_double), ("Gc", C.c_double),
                ("b_r", C.c_double), ("gap", C.c_double), ("rho", C.c_double), ("p_r", C.c_double),
                ("p_e", C.c_double), ("mu", C.c_double), ("mur", C.c_double), ("farcut", C.c_double),
                ("E_bond", C.c_double), ("kn_ks", C.c_double), ("Ec_sd", C.c_double), ("Gc_sd", C.c_double),
                ("bond_radius_factor", C.c_double), ("dt", C.c_double), ("dt_rayleigh_factor", C.c_double),
                ("seed", C.c_uint64), ("nobreak", C.c_int), ("reserved", C.c_int)]


class Loading(C.Structure):
    _fields_ = [("test", C.c_int), ("reserved", C.c_int),
                ("space_center", C.c_double * 3), ("space_half", C.c_double * 3),
                ("hidden_point", C.c_double * 3), ("zcut", C.c_double),
                ("size_real", C.c_double * 3), ("center_real", C.c_double * 3),
                ("velocity", C.c_double), ("min_stress", C.c_double), ("max_strain", C.c_double),
                ("cond_fracture", C.c_double), ("p_r_platen", C.c_double),
                ("dNsave", C.c_uint32), ("reserved2", C.c_uint32), ("max_steps", C.c_uint64)]


SENS_NAMES = ("E_bond", "kn_ks", "bond_radius", "E", "mu")


class Sensitivity(C.Structure):
    _fields_ = [("strain", C.c_double), ("stress", C.c_double), ("E_secant", C.c_double), ("nu_secant", C.c_double),
                ("dstress", C.c_double * 5), ("dE", C.c_double * 5), ("dnu", C.c_double * 5)]


class PackParams(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("radius", C.c_double), ("half_height", C.c_double),
                ("r_min", C.c_double), ("r_max", C.c_double), ("E", C.c_double), ("nu", C.c_double),
                ("rho", C.c_double), ("overlap_tol", C.c_double), ("n", C.c_uint32), ("growth_stages", C.c_uint32),
                ("steps_per_stage", C.c_uint32), ("max_fire_steps", C.c_uint32), ("seed", C.c_uint64),
                ("device", C.c_int), ("fire_variant", C.c_int), ("max_removed", C.c_uint32),
                ("reserved", C.c_uint32)]


class PackReport(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("max_overlap", C.c_double), ("packing_fraction", C.c_double),
                ("rebuilds", C.c_uint32), ("removed", C.c_uint32)]


class Result(C.Structure):
    _fields_ = [("FractureStress", C.c_double), ("FractureStrain", C.c_double),
                ("LinearityDeviation", C.c_double), ("Destruction", C.c_double), ("Strain", C.c_double),
                ("Stress", C.c_double), ("dt", C.c_double), ("platen_top", C.c_double),
                ("platen_bottom", C.c_double), ("platen_velocity", C.c_double), ("steps", C.c_uint64),
                ("stepsave", C.c_uint32), ("bonds_initial", C.c_uint32), ("bonds_now", C.c_uint32),
                ("fracture", C.c_int), ("done", C.c_int), ("stale", C.c_int), ("rebuilds", C.c_int),
                ("E_chord", C.c_double), ("nu", C.c_double), ("numeric", C.c_int), ("reserved_r", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneReport(C.Structure):
    _fields_ = [("candidates", C.c_int), ("pair_min_blocks", C.c_uint32 * 16), ("particle_block", C.c_uint32 * 16),
                ("ms_per_step", C.c_double * 16), ("chosen_pair_min_blocks", C.c_uint32),
                ("chosen_particle_block", C.c_uint32), ("chosen_ms_per_step", C.c_double),
                ("skin_candidates", C.c_int), ("skin_factor", C.c_double * 8), ("skin_ms_per_step", C.c_double * 8),
                ("skin_rebuild_ms", C.c_double * 8), ("chosen_skin_factor", C.c_double)]


_LIB = None
_vp, _u32, _i32, _u64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64


def _declare(L):
    P = C.POINTER
    L.dem_strerror.restype = C.c_char_p
    L.dem_strerror.argtypes = [C.c_int]
    L.dem_device_count.argtypes = [P(C.c_int)]
    L.dem_create.argtypes = [P(Options), P(_vp)]
    L.dem_destroy.argtypes = [_vp]
    L.dem_destroy.restype = None
    L.dem_release_cached_memory.argtypes = []
    L.dem_release_cached_memory.restype = C.c_int
    L.dem_add_sample.argtypes = [_vp, P(Material), P(Loading), _vp, _vp, _u32, P(_i32)]
    L.dem_setup.argtypes = [_vp]
    L.dem_run.argtypes = [_vp, _u64, P(_u64)]
    L.dem_step.argtypes = [_vp, _u32]
    L.dem_step_stages.argtypes = [_vp, C.c_int]
    L.dem_sync.argtypes = [_vp]
    L.dem_counts.argtypes = [_vp, P(_u32), P(_u32), P(_u32), P(_u32)]
    L.dem_sample_result.argtypes = [_vp, _i32, P(Result)]
    L.dem_get_record.argtypes = [_vp, _i32, _vp, _vp, _u32, P(_u32)]
    L.dem_get_particles.argtypes = [_vp, _i32] + [_vp] * 6
    L.dem_get_particles_d.argtypes = [_vp, _i32] + [_vp] * 6
    L.dem_set_particles.argtypes = [_vp, _i32] + [_vp] * 4
    L.dem_get_pairs.argtypes = [_vp, _i32, _u32, _vp, _vp, _vp, _vp, P(_u32)]
    L.dem_get_pairs_d.argtypes = [_vp, _i32, _u32, _vp, _vp, _vp, _vp, P(_u32)]
    L.dem_set_pairs.argtypes = [_vp, _i32, _u32, _vp, _vp, _vp, _vp]
    L.dem_set_platens.argtypes = [_vp, _i32, C.c_double, C.c_double, C.c_double]
    L.dem_rebuild_contacts.argtypes = [_vp]
    L.dem_run_timed.argtypes = [_vp, _u64, P(C.c_double)]
    L.dem_profile.argtypes = [_vp, _u32, P(C.c_double), P(C.c_double), P(C.c_double)]
    L.dem_autotune.argtypes = [_vp, _u32, P(TuneReport)]
    L.dem_create_cylinder_sample.argtypes = [P(PackParams), _vp, _vp, _u32, P(_u32), P(PackReport)]
    L.dem_last_error_detail.restype = C.c_char_p
    L.dem_last_error_detail.argtypes = []
    L.dem_save_lammps_data.argtypes = [_vp, C.c_int32, C.c_char_p, C.c_int]
    L.dem_sensitivities.argtypes = [_vp, C.c_int32, P(Sensitivity)]
    L.dem_get_lateral_record.argtypes = [_vp, C.c_int32, _vp, _u32, P(_u32)]
    L.dem_reference_space.argtypes = [_vp, _vp, C.c_double, C.c_double, P(Loading)]
    L.dem_ref_cells.argtypes = [_vp, _u32, C.c_float, _u32, _u32, _u32, _vp, _vp, _vp]
    L.dem_ref_cells_static.argtypes = [_vp, _u32, C.c_float, _u32, _u32, _u32, _vp, _vp, _vp]
    L.dem_ref_neighbor_sets.argtypes = [_vp, _u32, C.c_float, _u32, _u32, _u32, C.c_float, C.c_float, _u32, _vp,
                                        P(_u32)]
    L.dem_calculation_test.argtypes = [P(Options), P(Material), P(Loading), _vp, _vp, _u32, P(Result), _vp, _vp,
                                       _u32, P(_u32)]
    L.dem_load_cylinder_sample.argtypes = [C.c_char_p, C.c_double, _vp, _u32, P(_u32), _vp, _vp]
    L.dem_save_cylinder_sample.argtypes = [C.c_char_p, _vp, _u32, _vp]
    L.dem_save_sum_forces_loading.argtypes = [C.c_char_p, _vp, _u32]
    _sz, _f = C.c_size_t, C.c_float
    L.dem_mlp_gemm_tn.argtypes = [_vp, _vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, _vp]
    L.dem_mlp_status.argtypes = [P(C.c_int)]
    L.dem_mlp_pack_bf16.argtypes = [_vp, _vp, C.c_int, C.c_int, C.c_int, _vp, _vp]
    L.dem_mlp_gather.argtypes = [_vp, _vp, C.c_int, C.c_int, _vp, _vp]
    L.dem_mlp_transpose_bf16.argtypes = [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp]
    L.dem_mlp_act_backward.argtypes = [_vp, _vp, _sz, C.c_int, _vp, _vp, _vp]
    L.dem_mlp_colsum.argtypes = [_vp, C.c_int, C.c_int, _vp, _vp, _vp]
    L.dem_mlp_mse_grad.argtypes = [_vp, _vp, _sz, _vp, _vp, _vp, _vp]
    L.dem_mlp_adam.argtypes = [_vp, _vp, _vp, _vp, _sz, _f, _f, _f, _f, _f, _vp, _vp, _vp]
    L.dem_mlp_tick.argtypes = [_vp, _vp]
    L.dem_mlp_adam_multi.argtypes = [_vp, C.c_int, _sz, _f, _f, _f, _f, _vp, _vp]


def _lib():
    """Load libb200dem.so (building it first if it is missing or stale)."""
    global _LIB
    if _LIB is None:
        from . import build as _build  # noqa: F401  (package-relative import)
        _build.build()
        _LIB = C.CDLL(str(LIB_PATH))
        _declare(_LIB)
    return _LIB


def lib():
    return _lib()


def _ck(rc: int, where: str = "") -> None:
    if rc != 0:
        raise DemError(rc, where)


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def device_count() -> int:
    n = C.c_int(0)
    _lib().dem_device_count(C.byref(n))
    return n.value


# --------------------------------------------------------------------------- parameter helpers

def material(E=30.0, nu=0.247, Ec=0.04, Gc=0.04, b_r=0.2, gap=0.025, rho=2.61, p_r=0.25, p_e=0.6, mu=0.45,
             mur=0.05, farcut=3.2, **ext) -> Material:
    """Micro-parameters in reference units (GPa, mm, mg/mm^3); extensions by keyword."""
    m = Material(E=E, nu=nu, Ec=Ec, Gc=Gc, b_r=b_r, gap=gap, rho=rho, p_r=p_r, p_e=p_e, mu=mu, mur=mur,
                 farcut=farcut)
    for k, v in ext.items():
        setattr(m, k, v)
    return m


def material_si(E, Ec, Gc, b_r, gap, p_r=0.5e-3, rho=2610.0, nu=0.247, **kw) -> Material:
    """SetInitialParameters (mp_determineconjgradient.cu:15-47) from SI values."""
    return material(E=E / STRESS, nu=nu, Ec=Ec / STRESS, Gc=Gc / STRESS, b_r=b_r / LENGTH, gap=gap / LENGTH,
                    rho=rho / DENSITY, p_r=p_r / LENGTH, **kw)


def f32(x) -> float:
    return float(np.float32(x))


@dataclass
class SpaceBox:
    center: np.ndarray
    half: np.ndarray
    hidden_point: np.ndarray
    zcut: float
    A: np.ndarray
    B: np.ndarray
    cell_a: float
    L: np.ndarray
    Vext: float


def reference_space(space_si, lsi_si, p_r: float, farcut: float = 3.2) -> SpaceBox:
    """Escape box, hidden point and cell grid of the reference's sample set-up
    (sample_data::SetSpaceSizeSi / SetLSi / CalculateParameters,
    md_data_types.h:87-123, with C.a = 2*a_farcut, mp_determineconjgradient.cu:31-32).
    Float members are rounded as the reference stores them."""
    C_a = f32(2.0 * farcut * p_r)
    spacesize = np.array([f32(x / LENGTH) for x in space_si], np.float32)
    spacesized2 = np.array([f32(0.5 * float(s)) for s in spacesize], np.float32)
    L = np.array([f32(x / LENGTH - 2.0 * p_r) for x in lsi_si], np.float32)
    A = np.array([f32(1.01 * C_a)] * 3, np.float32)
    B = (A + spacesize).astype(np.float32)
    center = np.array([f32(0.5 * float(np.float32(A[k] + B[k]))) for k in range(3)], np.float32)
    hp = np.array([f32(float(A[0]) + 0.5 * float(spacesize[0])), f32(float(A[1]) + 0.5 * float(spacesize[1])),
                   f32((float(np.float32(math.floor(f32(float(B[2]) / C_a)))) + 3 - 0.5) * C_a)], np.float32)
    Vext = math.pi * (0.5 * float(L[0]) + p_r) ** 2 * (float(L[2]) + 2.0 * p_r)
    zcut = float(np.float32(center[2] + spacesized2[2]))
    return SpaceBox(center=center, half=spacesized2, hidden_point=hp, zcut=zcut, A=A, B=B, cell_a=C_a, L=L,
                    Vext=Vext)


def bounding_box(xyz: np.ndarray, n: int, p_r: float, radii=None):
    """h_LoadCylinderSample bounding box (md_createcylindersample.cu:448-465):
    extent of the centres plus 2 p_r and their midpoint.  With per-sphere radii
    the extent of the spheres themselves (equal radii give the same box), so
    polydisperse platens start on the specimen's surface."""
    x = xyz.reshape(3, n).astype(np.float64)
    if radii is None:
        mn, mx = x.min(1), x.max(1)
        return mx - mn + 2.0 * p_r, 0.5 * (mx + mn)
    r = np.asarray(radii, np.float64)[None, :]
    lo, hi = (x - r).min(1), (x + r).max(1)
    return hi - lo, 0.5 * (hi + lo)


def loading(test: int, box: SpaceBox, size_real, center_real, velocity: float, min_stress: float, max_strain: float,
            cond_fracture: float = 0.1, dNsave: int = 100, max_steps: int = 0, p_r_platen: float = 0.0) -> Loading:
    ld = Loading()
    ld.test = test
    for d in range(3):
        ld.space_center[d] = float(box.center[d])
        ld.space_half[d] = float(box.half[d])
        ld.hidden_point[d] = float(box.hidden_point[d])
        ld.size_real[d] = float(size_real[d])
        ld.center_real[d] = float(center_real[d])
    ld.zcut = box.zcut
    ld.velocity = velocity
    ld.min_stress = min_stress
    ld.max_strain = max_strain
    ld.cond_fracture = cond_fracture
    ld.dNsave = dNsave
    ld.max_steps = max_steps
    ld.p_r_platen = p_r_platen
    return ld


# --------------------------------------------------------------------------- context

class Context:
    """One engine context: specimens advance together on one GPU."""

    def __init__(self, precision: int = 0, device: int = 0, pair_block: int = 0, pair_grid: int = 0,
                 particle_block: int = 0, graph_steps: int = 0, skin_factor: float = 0.0, pair_min_blocks: int = 0,
                 deterministic: bool = False):
        L = _lib()
        self._opt = Options(precision=precision, device=device, pair_block=pair_block, pair_grid=pair_grid,
                            particle_block=particle_block, graph_steps=graph_steps, skin_factor=skin_factor,
                            pair_min_blocks=pair_min_blocks, deterministic=1 if deterministic else 0)
        h = C.c_void_p()
        _ck(L.dem_create(C.byref(self._opt), C.byref(h)), "dem_create")
        self._h = h
        self.precision = precision
        self._n = []

    def close(self):
        if getattr(self, "_h", None):
            _lib().dem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_sample(self, mat: Material, load: Loading, xyz: np.ndarray, radii: np.ndarray | None = None) -> int:
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1)
        n = xyz.size // 3
        rad = None if radii is None else np.ascontiguousarray(radii, np.float32)
        sid = C.c_int32()
        _ck(_lib().dem_add_sample(self._h, C.byref(mat), C.byref(load), _p(xyz), _p(rad), n, C.byref(sid)),
            "dem_add_sample")
        self._n.append(n)
        return sid.value

    def setup(self):
        _ck(_lib().dem_setup(self._h), "dem_setup")

    def run(self, max_steps: int) -> int:
        done = C.c_uint64()
        _ck(_lib().dem_run(self._h, max_steps, C.byref(done)), "dem_run")
        return done.value

    def step(self, n: int = 1):
        _ck(_lib().dem_step(self._h, n), "dem_step")

    def step_stages(self, stages: int):
        _ck(_lib().dem_step_stages(self._h, stages), "dem_step_stages")

    def sync(self):
        _ck(_lib().dem_sync(self._h), "dem_sync")

    def counts(self) -> dict:
        v = [C.c_uint32() for _ in range(4)]
        _ck(_lib().dem_counts(self._h, *[C.byref(x) for x in v]), "dem_counts")
        return dict(particles=v[0].value, bonds=v[1].value, contacts=v[2].value, samples=v[3].value)

    def result(self, sample: int = 0) -> dict:
        r = Result()
        _ck(_lib().dem_sample_result(self._h, sample, C.byref(r)), "dem_sample_result")
        return r.as_dict()

    def save_lammps_data(self, path: str, sample: int = 0, with_energy: bool = False) -> None:
        """SaveLammpsDATASimple: LAMMPS data file of one specimen."""
        _ck(_lib().dem_save_lammps_data(self._h, sample, path.encode(), 1 if with_energy else 0), "dem_save_lammps_data")

    def sensitivities(self, sample: int = 0) -> dict:
        """Secant modulus and Poisson ratio at the last step; with precision=2
        also their derivatives (arrays over SENS_NAMES)."""
        s = Sensitivity()
        _ck(_lib().dem_sensitivities(self._h, sample, C.byref(s)), "dem_sensitivities")
        return dict(strain=s.strain, stress=s.stress, E_secant=s.E_secant, nu_secant=s.nu_secant,
                    dstress=np.array(s.dstress[:]), dE=np.array(s.dE[:]), dnu=np.array(s.dnu[:]))

    def lateral_record(self, sample: int = 0) -> np.ndarray:
        """Mean radial distance of the lateral surface particles per record entry."""
        n = C.c_uint32()
        _ck(_lib().dem_get_lateral_record(self._h, sample, None, 0, C.byref(n)), "dem_get_lateral_record")
        out = np.zeros(max(n.value, 1), np.float64)
        _ck(_lib().dem_get_lateral_record(self._h, sample, _p(out), n.value, C.byref(n)), "dem_get_lateral_record")
        return out[:n.value]

    def record(self, sample: int = 0):
        n = C.c_uint32()
        _ck(_lib().dem_get_record(self._h, sample, None, None, 0, C.byref(n)), "dem_get_record")
        rec = np.zeros(3 * max(n.value, 1), np.float64)
        bonds = np.zeros(max(n.value, 1), np.uint32)
        _ck(_lib().dem_get_record(self._h, sample, _p(rec), _p(bonds), n.value, C.byref(n)), "dem_get_record")
        return rec[:3 * n.value].reshape(-1, 3), bonds[:n.value]

    def particles(self, sample: int = 0, double: bool = False) -> dict:
        n = self._n[sample]
        dt = np.float64 if double else np.float32
        arrs = {k: np.zeros(3 * n, dt) for k in ("R", "V", "W", "F", "M", "Oiwt")}
        fn = _lib().dem_get_particles_d if double else _lib().dem_get_particles
        _ck(fn(self._h, sample, *[_p(arrs[k]) for k in ("R", "V", "W", "F", "M", "Oiwt")]), "dem_get_particles")
        return arrs

    def set_particles(self, sample: int = 0, R=None, V=None, W=None, Oiwt=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        R, V, W, Oiwt = c(R), c(V), c(W), c(Oiwt)
        _ck(_lib().dem_set_particles(self._h, sample, _p(R), _p(V), _p(W), _p(Oiwt)), "dem_set_particles")

    def pairs(self, sample: int = 0, double: bool = False) -> dict:
        fn = _lib().dem_get_pairs_d if double else _lib().dem_get_pairs
        n = C.c_uint32()
        _ck(fn(self._h, sample, 0, None, None, None, None, C.byref(n)), "dem_get_pairs")
        m = n.value
        i = np.zeros(max(m, 1), np.uint32)
        j = np.zeros(max(m, 1), np.uint32)
        kind = np.zeros(max(m, 1), np.uint32)
        st = np.zeros(16 * max(m, 1), np.float64 if double else np.float32)
        _ck(fn(self._h, sample, m, _p(i), _p(j), _p(kind), _p(st), C.byref(n)), "dem_get_pairs")
        return dict(i=i[:m], j=j[:m], kind=kind[:m], state=st[:16 * m].reshape(-1, 16))

    def set_pairs(self, sample: int, i, j, kind, state):
        i = np.ascontiguousarray(i, np.uint32)
        j = np.ascontiguousarray(j, np.uint32)
        kind = np.ascontiguousarray(kind, np.uint32)
        state = np.ascontiguousarray(state, np.float32).reshape(-1)
        _ck(_lib().dem_set_pairs(self._h, sample, i.size, _p(i), _p(j), _p(kind), _p(state)), "dem_set_pairs")

    def set_platens(self, sample: int, top: float, bottom: float, velocity: float):
        _ck(_lib().dem_set_platens(self._h, sample, top, bottom, velocity), "dem_set_platens")

    def rebuild_contacts(self):
        _ck(_lib().dem_rebuild_contacts(self._h), "dem_rebuild_contacts")

    def run_timed(self, nsteps: int) -> float:
        """Device milliseconds of nsteps graph-replayed steps (CUDA events)."""
        ms = C.c_double()
        _ck(_lib().dem_run_timed(self._h, nsteps, C.byref(ms)), "dem_run_timed")
        return ms.value

    def autotune(self, steps: int = 200) -> dict:
        """Times the launch-schedule candidates and then the contact-list skins
        on the next steps of this run (steps per candidate; the simulation
        advances) and keeps the fastest."""
        r = TuneReport()
        _ck(_lib().dem_autotune(self._h, steps, C.byref(r)), "dem_autotune")
        n = r.candidates
        return dict(candidates=[(r.pair_min_blocks[k], r.particle_block[k], r.ms_per_step[k]) for k in range(n)],
                    pair_min_blocks=r.chosen_pair_min_blocks, particle_block=r.chosen_particle_block,
                    ms_per_step=r.chosen_ms_per_step,
                    skins=[(r.skin_factor[k], r.skin_ms_per_step[k], r.skin_rebuild_ms[k])
                           for k in range(r.skin_candidates)],
                    skin_factor=r.chosen_skin_factor)

    def profile(self, nsteps: int) -> dict:
        a, b, t = C.c_double(), C.c_double(), C.c_double()
        _ck(_lib().dem_profile(self._h, nsteps, C.byref(a), C.byref(b), C.byref(t)), "dem_profile")
        return dict(pair_ms=a.value, particle_ms=b.value, touching=t.value)


# --------------------------------------------------------------------------- stateless entry points

def release_cached_memory() -> None:
    """Device memory of closed contexts, kept for reuse by later contexts,
    goes back to the driver (dem_release_cached_memory)."""
    _ck(_lib().dem_release_cached_memory(), "dem_release_cached_memory")


def ref_cells(xyz: np.ndarray, a: float, nx: int, ny: int, nz: int):
    xyz = np.ascontiguousarray(xyz, np.float32)
    n = xyz.size // 3
    CI = np.zeros(n, np.uint32)
    CIs = np.zeros(2 * n, np.uint32)
    pnC = np.zeros(2 * nx * ny * nz, np.uint32)
    _ck(_lib().dem_ref_cells(_p(xyz), n, a, nx, ny, nz, _p(CI), _p(CIs), _p(pnC)), "dem_ref_cells")
    return CI, CIs, pnC


def ref_cells_static(xyz: np.ndarray, a: float, nx: int, ny: int, nz: int):
    """ref_cells through dem_ref_cells_static (no allocation; limited sizes)."""
    xyz = np.ascontiguousarray(xyz, np.float32)
    n = xyz.size // 3
    CI = np.zeros(n, np.uint32)
    CIs = np.zeros(2 * n, np.uint32)
    pnC = np.zeros(2 * nx * ny * nz, np.uint32)
    _ck(_lib().dem_ref_cells_static(_p(xyz), n, a, nx, ny, nz, _p(CI), _p(CIs), _p(pnC)), "dem_ref_cells_static")
    return CI, CIs, pnC


def ref_neighbor_sets(xyz: np.ndarray, a: float, nx: int, ny: int, nz: int, add_thr: float, del_thr: float,
                      cap: int = 32):
    xyz = np.ascontiguousarray(xyz, np.float32)
    n = xyz.size // 3
    sets = np.zeros(n * cap, np.uint32)
    ovf = C.c_uint32()
    _ck(_lib().dem_ref_neighbor_sets(_p(xyz), n, a, nx, ny, nz, add_thr, del_thr, cap, _p(sets), C.byref(ovf)),
        "dem_ref_neighbor_sets")
    return sets.reshape(n, cap), ovf.value


def calculation_test(mat: Material, load: Loading, xyz: np.ndarray, radii=None, precision: int = 0,
                     rec_cap: int = 1 << 20):
    """h_Calculation{UniaxialCompression,BrazilTest} through the C ABI: host
    positions in, macro results and the loading record out."""
    opt = Options(precision=precision)
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1)
    rad = None if radii is None else np.ascontiguousarray(radii, np.float32)
    r = Result()
    rec = np.zeros(3 * rec_cap, np.float64)
    rb = np.zeros(rec_cap, np.uint32)
    n = C.c_uint32()
    _ck(_lib().dem_calculation_test(C.byref(opt), C.byref(mat), C.byref(load), _p(xyz), _p(rad), xyz.size // 3,
                                    C.byref(r), _p(rec), _p(rb), rec_cap, C.byref(n)), "dem_calculation_test")
    m = min(n.value, rec_cap)
    return r.as_dict(), rec[:3 * m].reshape(-1, 3), rb[:m]


def create_cylinder_sample(center, radius: float, half_height: float, n: int, r_min: float, r_max: float,
                           E: float = 50.0, nu: float = 0.25, rho: float = 2.65, overlap_tol: float = 1e-3,
                           growth_stages: int = 40, steps_per_stage: int = 200, max_fire_steps: int = 20000,
                           seed: int = 1, device: int = 0, fire_variant: int = 0, max_removed: int = 0):
    """Seeded packed cylinder (h_CreateCylinderSample): returns xyz (SoA), radii, report.
    fire_variant 0 relaxes with inertial FIRE 2.0, 1 with the reference's FIRE update;
    max_removed > 0 lets it remove spheres of the worst overlaps (fewer than n are returned)."""
    p = PackParams(radius=radius, half_height=half_height, r_min=r_min, r_max=r_max, E=E, nu=nu, rho=rho,
                   overlap_tol=overlap_tol, n=n, growth_stages=growth_stages, steps_per_stage=steps_per_stage,
                   max_fire_steps=max_fire_steps, seed=seed, device=device, fire_variant=fire_variant,
                   max_removed=max_removed)
    for d in range(3):
        p.center[d] = float(center[d])
    xyz = np.zeros(3 * n, np.float32)
    rad = np.zeros(n, np.float32)
    m = C.c_uint32()
    rep = PackReport()
    _ck(_lib().dem_create_cylinder_sample(C.byref(p), _p(xyz), _p(rad), n, C.byref(m), C.byref(rep)),
        "dem_create_cylinder_sample")
    k = m.value
    return np.ascontiguousarray(xyz[:3 * k]), rad[:k].copy(), dict(
        steps=rep.steps, max_overlap=rep.max_overlap, packing_fraction=rep.packing_fraction, rebuilds=rep.rebuilds,
        removed=rep.removed)


def load_cylinder_sample(path: str, p_r: float):
    n = C.c_uint32()
    _ck(_lib().dem_load_cylinder_sample(path.encode(), p_r, None, 0, C.byref(n), None, None), "load")
    xyz = np.zeros(3 * n.value, np.float32)
    size = (C.c_double * 3)()
    cen = (C.c_double * 3)()
    _ck(_lib().dem_load_cylinder_sample(path.encode(), p_r, _p(xyz), n.value, C.byref(n), size, cen), "load")
    return xyz, np.array(size[:]), np.array(cen[:])


def save_cylinder_sample(path: str, xyz: np.ndarray, hidden_point=None):
    xyz = np.ascontiguousarray(xyz, np.float32)
    hp = None if hidden_point is None else (C.c_double * 3)(*[float(v) for v in hidden_point])
    _ck(_lib().dem_save_cylinder_sample(path.encode(), _p(xyz), xyz.size // 3, hp), "save")


def save_sum_forces_loading(path: str, rec: np.ndarray):
    rec = np.ascontiguousarray(rec, np.float64)
    _ck(_lib().dem_save_sum_forces_loading(path.encode(), _p(rec), rec.size // 3), "save")
