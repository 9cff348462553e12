"""Conjugate-gradient calibration of the bond micro-parameters, with the
finite-difference solves of each step run as one batched engine context.

The reference's DetermineConjGradient (mp_determineconjgradient.cu:186-352)
runs, per step, one uniaxial (and optionally one Brazilian) test for the
current parameters and one per varied parameter - six sequential
h_Calculation* calls (CalculateStepCG, mp_determineconjgradient.cu:84-145) -
then updates the parameters by a Fletcher-Reeves direction with a
Gauss-Newton step length (mp_task_data::CalculateNewParameters2,
mp_task.h:223-311).  Here the six (or twelve) solves of a step are specimens
of ONE context and advance together on the GPU; the parameter update is the
reference's arithmetic, in the same order, in double.

Parameters (internal units, mm / GPa): E, Ec, Gc, bond radius b_r, bond gap
(b_d - 2 p_r).  Results: uniaxial strain at peak, uniaxial peak stress,
Brazilian peak stress, uniaxial linearity deviation.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import Context, material

NPARAM, NRESULT = 5, 4
# mp_task.h:138 (varflags): which parameters each variation type varies
VARFLAGS = np.array([[1, 1, 1, 0, 0], [0, 0, 0, 1, 1], [1, 1, 1, 1, 1], [0, 1, 1, 1, 1], [0, 0, 1, 1, 1],
                     [1, 0, 0, 1, 1], [1, 0, 0, 0, 0], [0, 1, 1, 1, 0]], dtype=np.float64)
# unit constants as the reference computes them (md_phys_constants.h:5-12)
LENGTH_CONST, MASS_CONST, TIME_CONST = 1e-3, 1e-6, 1e-6
STRESS_CONST = (MASS_CONST * LENGTH_CONST / (TIME_CONST * TIME_CONST)) / (LENGTH_CONST * LENGTH_CONST)
# SetMaterialContractions (mp_task.h:107-128) lower bounds, internal units:
# E, Ec >= 1e5 Pa, Gc >= 1e8 Pa, b_r >= 1e-6 m, gap >= 1e-5 m
FLOORS = (1e5 / STRESS_CONST, 1e5 / STRESS_CONST, 1e8 / STRESS_CONST, 1e-6 / LENGTH_CONST, 1e-5 / LENGTH_CONST)


@dataclass
class CGTask:
    """mp_task_data of the reference (mp_task.h:11-99), for NParam = 5, NResult = 4."""
    params: np.ndarray                      # current parameters (5)
    goal: np.ndarray                        # ResultsGoal (4)
    weight_multiplier: np.ndarray           # FunctionalParametersWeightMultiplier (4)
    variation_type: int = 2                 # ParameterVariationType
    delta_factor: float = 0.1               # MaterialDeltaFactor
    calc_u: bool = True                     # CalculateUTest
    calc_b: bool = False                    # CalculateBTest
    step: int = 0
    weight: np.ndarray = field(default_factory=lambda: np.zeros(NRESULT))
    variation: np.ndarray = field(default_factory=lambda: np.zeros((NPARAM + 1, NPARAM)))
    rfun: np.ndarray = field(default_factory=lambda: np.zeros((NPARAM + 1, NRESULT)))
    dfun: np.ndarray = field(default_factory=lambda: np.zeros(NPARAM + 1))
    ddfun: np.ndarray = field(default_factory=lambda: np.zeros(NPARAM + 1))
    functional: np.ndarray = field(default_factory=lambda: np.zeros(NRESULT))
    history: list = field(default_factory=list)

    def start_parameters(self) -> None:
        """CalculateStartParameters (mp_task.h:129-145)."""
        self.params = np.asarray(self.params, np.float64).copy()
        self.goal = np.asarray(self.goal, np.float64).copy()
        self.variation[:] = 0.0
        for j in range(NRESULT):
            self.weight[j] = self.weight_multiplier[j] / (self.goal[j] * self.goal[j])
        if not self.calc_u:
            self.weight[0] = 1.0
            self.weight[3] = 1.0
            self.goal[0] = self.goal[1] = self.goal[3] = 1.0
        if not self.calc_b:
            self.weight[2] = 100.0
            self.goal[2] = 1.0
        flags = VARFLAGS[self.variation_type]
        for i in range(NPARAM):
            self.variation[i + 1, i] = flags[i] * self.delta_factor * self.params[i]

    def solve_parameters(self, i: int):
        """SetVariationParameters (mp_determineconjgradient.cu:49-80): the
        parameters of solve i, or None when row i varies nothing (i > 0)."""
        if i > 0 and self.variation[i].sum() < 1e-12:
            return None
        return self.params + self.variation[i]

    def new_parameters(self) -> np.ndarray:
        """CalculateNewParameters2 (mp_task.h:223-311) with SetMaterialContractions
        (mp_task.h:107-128); returns the next step's parameters."""
        w, R, V = self.weight, self.rfun, self.variation
        dR = np.zeros((NPARAM + 1, NRESULT))
        for i in range(NPARAM):
            for j in range(NRESULT):
                if V[i + 1, i] > 1e-12:
                    dR[i + 1, j] = 1.0 * (R[i + 1, j] - R[0, j]) / V[i + 1, i]
        D = np.zeros(NRESULT)
        for j in range(NRESULT):
            D[j] = self.goal[j] - R[0, j]
            self.functional[j] = w[j] * D[j] * D[j]
        dF0 = dF1 = 0.0
        for i in range(NPARAM):
            self.ddfun[i + 1] = self.dfun[i + 1]
            dF0 += self.dfun[i + 1] * self.dfun[i + 1]
            g = 0.0
            for j in range(NRESULT):
                g += -2 * w[j] * D[j] * dR[i + 1, j]
            self.dfun[i + 1] = g
            dF1 += g * g
        b = dF1 / dF0 if dF0 > 1e-12 else 0.0
        for i in range(NPARAM):
            self.ddfun[i + 1] = self.dfun[i + 1] + b * self.ddfun[i + 1]
        a0 = a1 = 0.0
        for j in range(NRESULT):
            for i in range(NPARAM):
                a1 += w[j] * D[j] * dR[i + 1, j] * self.ddfun[i + 1]
                for k in range(NPARAM):
                    a0 += w[j] * dR[i + 1, j] * self.ddfun[i + 1] * dR[k + 1, j] * self.ddfun[k + 1]
        t = -a1 / a0
        new = np.empty(NPARAM)
        for i in range(NPARAM):
            new[i] = self.params[i] - t * self.ddfun[i + 1] / 1.0
        # SetMaterialContractions (lower bounds; a NaN passes, as there)
        for k, floor in enumerate(FLOORS):
            if new[k] < floor:
                new[k] = floor
        self.variation[:] = 0.0
        flags = VARFLAGS[self.variation_type]
        for i in range(NPARAM):
            self.variation[i + 1, i] = flags[i] * self.delta_factor * new[i]
        return new


def descent_step(R0: np.ndarray, dR: np.ndarray, goal: np.ndarray, weight: np.ndarray):
    """The first step of CalculateNewParameters2 (mp_task.h:253-300) for a
    functional F = sum_j w_j (goal_j - R_j)^2 over any number of results and
    parameters, given the result Jacobian dR[i, j] = dR_j / dp_i: from the
    reference's one-sided finite differences (its six solves per step) or from
    the sensitivity build.  Returns the direction dfun_i = -2 sum_j w_j D_j
    dR[i, j] (the gradient of F; on a first step the conjugate direction is
    dfun itself, bcoeff = 0) and the Gauss-Newton step length t = -a1 / a0
    along it; the reference's update is then p - t dfun."""
    R0, dR = np.asarray(R0, np.float64), np.asarray(dR, np.float64)
    w, goal = np.asarray(weight, np.float64), np.asarray(goal, np.float64)
    D = goal - R0
    dfun = np.array([sum(-2 * w[j] * D[j] * dR[i, j] for j in range(D.size)) for i in range(dR.shape[0])])
    a0 = a1 = 0.0
    for j in range(D.size):
        for i in range(dR.shape[0]):
            a1 += w[j] * D[j] * dR[i, j] * dfun[i]
            for k in range(dR.shape[0]):
                a0 += w[j] * dR[i, j] * dfun[i] * dR[k, j] * dfun[k]
    return dfun, -a1 / a0


def finite_difference_jacobian(R0: np.ndarray, R_varied: np.ndarray, variation: np.ndarray) -> np.ndarray:
    """dR[i, j] = (R_varied[i, j] - R0[j]) / variation[i]: the reference's
    one-sided differences (mp_task.h:233-246, ParameterVariation = MaterialDeltaFactor
    x parameter)."""
    R0, Rv, v = (np.asarray(a, np.float64) for a in (R0, R_varied, variation))
    return (Rv - R0[None, :]) / v[:, None]


@dataclass
class Specimen:
    """A loaded sample file: positions (SoA) and the loading set-up."""
    xyz: np.ndarray
    loading: object


def material_from(p: np.ndarray, p_r: float = 0.5, farcut: float = 2.9):
    """The material SetVariationParameters builds (mp_determineconjgradient.cu:49-69):
    nu 0.247, rho 2610 kg/m^3, p_r 0.5 mm, restitution 0.6, friction 0.45,
    rolling friction 0.05, far cut-off 2.9 p_r."""
    return material(E=p[0], nu=0.247, Ec=p[1], Gc=p[2], b_r=p[3], gap=p[4], rho=2.61, p_r=p_r, p_e=0.6, mu=0.45,
                    mur=0.05, farcut=farcut)


def evaluate(task: CGTask, uni: Specimen | None, braz: Specimen | None, device: int = 0,
             max_steps: int = 0) -> None:
    """CalculateStepCG (mp_determineconjgradient.cu:84-145): every solve of the
    step (uniaxial and Brazilian) in one context; fills task.rfun."""
    ctx = Context(device=device, graph_steps=200)
    slots = []
    for i in range(NPARAM + 1):
        p = task.solve_parameters(i)
        if uni is not None and task.calc_u and p is not None:
            slots.append((i, "u", ctx.add_sample(material_from(p), _with_max(uni.loading, max_steps), uni.xyz)))
        if braz is not None and task.calc_b and p is not None:
            slots.append((i, "b", ctx.add_sample(material_from(p), _with_max(braz.loading, max_steps), braz.xyz)))
    task.rfun[:] = 0.0
    task.rfun[:, 2] = 1.0  # a skipped Brazilian solve reports 1 (mp_determineconjgradient.cu:118)
    if slots:
        ctx.setup()
        ctx.run(max_steps if max_steps else (1 << 62))
        for i, kind, sid in slots:
            r = ctx.result(sid)
            if kind == "u":
                task.rfun[i, 0] = r["FractureStrain"]
                task.rfun[i, 1] = r["FractureStress"]
                task.rfun[i, 3] = r["LinearityDeviation"]
            else:
                task.rfun[i, 2] = r["FractureStress"]
    ctx.close()


def _with_max(ld, max_steps):
    if not max_steps:
        return ld
    c = type(ld).from_buffer_copy(ld)
    c.max_steps = max_steps
    return c


def calibrate(task: CGTask, uni: Specimen | None, braz: Specimen | None, steps: int, device: int = 0,
              max_steps: int = 0, results_file: str | None = None) -> CGTask:
    """The loop of DetermineConjGradient: start parameters, then per step the
    batched solves, the parameter update and one SaveResults record
    (mp_task.h:312-321 format when results_file is given)."""
    task.start_parameters()
    for step in range(steps):
        task.step = step
        evaluate(task, uni, braz, device=device, max_steps=max_steps)
        new = task.new_parameters()
        task.history.append(dict(step=step, params=task.params.copy(), results=task.rfun[0].copy(),
                                 functional=task.functional.copy()))
        if results_file:
            save_results(results_file, task)
        task.params = new
    return task


def save_results(path: str, task: CGTask) -> None:
    """mp_task_data::SaveResults (mp_task.h:312-321), appended."""
    p, r, f = task.params, task.rfun[0], task.functional
    with open(path, "a") as fh:
        fh.write(f"Step: {task.step}\n")
        fh.write("Parameters (E, Ecrit, Gcrit, boundR, boundDistance): "
                 f"{p[0] * STRESS_CONST:g} {p[1] * STRESS_CONST:g} {p[2] * STRESS_CONST:g} "
                 f"{p[3] * LENGTH_CONST:g} {p[4] * LENGTH_CONST:g} \n")
        fh.write("Results (UniaxialFractureStrain UniaxialFractureStress BrasilFractureStress): "
                 f"{r[0]:g} {r[1] * STRESS_CONST:g} {r[2] * STRESS_CONST:g}\n")
        fh.write("DFunctional" + "".join(f" {v:g}" for v in f) + f" | {f.sum():g}\n")
