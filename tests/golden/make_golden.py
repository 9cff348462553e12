"""Generate the golden vectors of tests/golden/*.npz from the reference's OWN
CUDA kernels (oracle/_ref/libdemref.so, compiled by oracle/Makefile from the
reference sources).  Needs a GPU:

    python tests/golden/make_golden.py --out <directory>

(then copy the .npz files into tests/golden/).

Each fixture holds a seeded input state in the reference layout and the state
the reference kernels produce from it, so that the CPU oracle (and through it
the CUDA product) can be pinned to the reference on the same inputs.

Fixtures
  cells_il_s<k>   CellDistribution, InteractionListConstruct, bond creation
  step_<case>     one full pass of the loading-loop body from a warmed-up state
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
import dem_testlib as T  # noqa: E402
from oracle import lib as L  # noqa: E402
from oracle import sim  # noqa: E402

SMALL = dict(lsi=(0.0035, 0.0035, 0.005), space=(0.008, 0.008, 0.011))

# name: (ref_case kwargs, perturbation kwargs, warm-up steps)
STEP_CASES = {
    "u_plain": (dict(seed=11), dict(dx=2e-4, v=1e-4, w=1e-3), 6),
    "b_plain": (dict(seed=12, brazil=True), dict(dx=2e-4, v=1e-4, w=1e-3), 6),
    "u_break": (dict(seed=13), dict(dx=1.2e-3, v=1e-4, w=1e-3), 2),
    "u_contact": (dict(seed=14, gap_si=-0.01e-3, jitter_frac=0.05), dict(dx=2e-3, v=3e-4, w=3e-3), 4),
}


def cells_fixture(seed: int, out: Path) -> None:
    c = T.ref_case(seed=seed, **SMALL)
    CI, CIs, pnC = sim.ref_cells(c.R, c.N, c.sc)
    st = sim.RefState.empty(c.N)
    st.R[:] = c.R
    sim.ref_setup_bonds(st, c.sc)
    np.savez_compressed(out / f"cells_il_s{seed}.npz", R=c.R, CI=CI, CIs=CIs, pnC=pnC, IL=st.IL, ILtype=st.ILtype,
                        invL0=st.invL0, seed=seed)
    print(f"cells_il_s{seed}: N={c.N} CN={c.cells.CN} bonds={int(((st.IL != L.EMPTY) & (st.ILtype == 1)).sum())}")


def step_fixture(name: str, out: Path) -> None:
    kw, pk, warm = STEP_CASES[name]
    c = T.ref_case(**SMALL, **kw)
    # platens moved 0.01 mm into the specimen so that both carry load
    c.sc.wall_top = float(np.float32(c.sc.wall_top - 0.01))
    c.sc.wall_bot = float(np.float32(c.sc.wall_bot + 0.01))
    st = sim.RefState.empty(c.N)
    st.R[:] = c.R
    sim.ref_setup_bonds(st, c.sc)
    rng = np.random.default_rng(1000 + kw["seed"])
    T.perturb(st, rng, **pk)
    for _ in range(warm):
        sim.ref_step(st, c.sc)
    st_in = st.copy()
    sFL, FL = sim.ref_step(st, c.sc)
    d = {"seed": kw["seed"], "name": name, "FL": FL, "sFL": sFL, "wall_top": c.sc.wall_top,
         "wall_bot": c.sc.wall_bot}
    d.update(st_in.to_dict("in_"))
    d.update(st.to_dict("out_"))
    np.savez_compressed(out / f"step_{name}.npz", **d)
    nb_in = int(((st_in.IL != L.EMPTY) & (st_in.ILtype == 1)).sum())
    nb_out = int(((st.IL != L.EMPTY) & (st.ILtype == 1)).sum())
    print(f"step_{name}: N={c.N} bonded slots {nb_in}->{nb_out} sFL={sFL}")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    for seed in (1, 2):
        cells_fixture(seed, out)
    for name in STEP_CASES:
        step_fixture(name, out)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
