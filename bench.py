"""Benchmark of the bonded-particle DEM step (BPM + Hertz-Mindlin) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload brazilian_disc|brazilian_disc_postpeak|uniaxial_cylinder|
                                calibration_sweep|calibration_solves|surrogate]

A step is one DEM time step of a loading test (pair forces, platens,
integration, loading controller; contact-list rebuilds when needed) over the
whole specimen.  The default workload is the Brazilian disc 40 mm x 20 mm
with radii U[0.18, 0.30] mm (~245k spheres, seeded synthetic packing).
Metric: particle-steps/s (particles x steps / device time, all ranks summed).

Under torchrun every rank runs its own specimen (different seed) on its own
GPU: the specimens are independent, so the work shards with no data-path
collective (weak scaling); the timing barrier and max-over-ranks use
torch.distributed.

--impl reference times the CPU restatement of the reference step (oracle,
all host threads) for the same --warmup and --steps on the same specimens,
which it packs on the host with the CPU restatement of the packer (the same
packings bit for bit); it does not load the product library.

Other workloads (each prints its own line): calibration_sweep (many
cylinders and parameter sets in one context against one context at a time),
calibration_solves (whole uniaxial solves per hour, batched against one
solve per context), surrogate (training of the tensor-core MLP and its
forward GEMM against the tensor peak).
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "BPM particle-steps/s"
UNIT = "particle-steps/s"
# DRAM bytes (read + write) of one k_pairs launch on the default workload (two
# 245,098-sphere Brazilian discs), ncu --set full early in the loading
PAIR_TRAFFIC_DISC_X2 = 195.5e6


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    def __init__(self, ws):
        self.ws = ws
        self.pg = None
        if ws > 1:
            import datetime

            import torch.distributed as td

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            td.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.td = td

    def barrier(self):
        if self.ws > 1:
            self.td.barrier()

    def max(self, v: float) -> float:
        if self.ws == 1:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if self.ws == 1:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.ws > 1:
            self.td.destroy_process_group()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def tensor_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["bf16_tflops"]), "measured (burst)"
    return 1590.0, "fallback"


class Clocks:
    """SM clocks and throttle reasons sampled during the timed region: an NVML
    thread polling every half millisecond (so that a region of a few
    milliseconds still gets samples; it takes its first sample before the
    constructor returns and a last one in stop()), else nvidia-smi at 100 ms."""

    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    _BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int):
        self.p = None
        self.nv = None
        self.rows = []
        try:
            import threading

            import pynvml
            import torch

            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(device)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.nv = pynvml
            self.stop_ev = threading.Event()
            self._sample()
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nv = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={device}", f"--query-gpu={q}", "--format=csv,noheader",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def _sample(self):
        nv = self.nv
        try:
            fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.rows.append((float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)),
                              float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)), int(fn(self.h))))
        except Exception:
            pass

    def _loop(self):
        while not self.stop_ev.wait(0.0005):
            self._sample()

    def stop(self) -> dict:
        if self.nv is not None:
            self._sample()
            self.stop_ev.set()
            self.t.join(5)
            sm = [r[0] for r in self.rows]
            mx = [r[1] for r in self.rows]
            reasons = sorted({k for r in self.rows for k, bit in self._BITS.items() if r[2] & bit})
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                    "reasons": reasons, "samples": len(sm), "source": "nvml"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in Path(self.f.name).read_text().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1].split()[0]))
                mx.append(float(r[2].split()[0]))
                for k, v in zip(names, r[5:9]):
                    if "Active" in v and "Not" not in v:
                        reasons.add(k)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def build_specimen(dem, workload: str, seed: int, device: int, packer=None):
    """A named specimen; `packer` replaces the GPU packer by another
    implementation of the same seeded algorithm (the reference leg builds its
    specimens on the host with the CPU restatement, bit for bit the same)."""
    W = importlib.import_module("dem-rock-calibration_b200.workloads")
    pk = dict(device=device) if packer is None else {}
    return getattr(W, workload)(seed=seed, pack_kw=pk, packer=packer)


def specimen_seeds(args, rank: int) -> list[int]:
    return [1 + rank * args.specimens + k for k in range(args.specimens)]


def workload_config(args, specs, ws: int) -> dict:
    """The benchmark configuration (identical for both legs): what is run, not
    what was measured."""
    n = sum(sp.n for sp in specs)
    spec = specs[0]
    if args.workload == "brazilian_disc":
        what = (f"{args.specimens} x brazilian_disc ({spec.n} spheres each, radii U[0.18,0.30] mm, "
                f"Brazilian platens at 0.02 m/s) advanced together")
    else:
        what = f"{args.specimens} x {args.workload} ({spec.n} spheres each)"
    return {"workload": what, "particles_per_gpu": n, "specimens": args.specimens,
            "seeds": specimen_seeds(args, 0), "precision": "f64" if args.precision == 1 else "f32",
            "parallelism": f"{ws} GPU(s), independent specimens",
            "l2": "inputs larger than L2 (state above 126 MB), no flush" if n > 300000 else "state inside the L2"}


class CpuStep:
    """The oracle's full loop body (cells, interaction-list rebuild, BPM, HM,
    platens, integration, escape parking, far-link deletion) of one specimen
    in the configuration's physics (oracle/physics.py: per-sphere radii and
    masses, per-slot bond radius and strengths), on host cores."""

    def __init__(self, spec, IonP: int = 48):
        from oracle import physics as PH
        from oracle import sim

        self.sim = sim
        mat, ld = spec.material, spec.loading
        self.pc = PH.physics_case(mat, ld, spec.radii, IonP=IonP)
        st = sim.RefState.empty(spec.n, IonP=IonP)
        st.R[:] = spec.xyz
        sim.oracle_setup_bonds(st, self.pc.sc, rad=self.pc.rad, gap=mat.gap)
        n = spec.n
        IL = st.IL.reshape(n, IonP)
        jj = np.where(IL == 0xFFFFFFFF, 0, IL)
        lo, hi = np.minimum(np.arange(n)[:, None], jj), np.maximum(np.arange(n)[:, None], jj)
        slot_br = (np.float32(mat.bond_radius_factor) * np.minimum(self.pc.rad[:, None], self.pc.rad[jj]))
        sn, stn = PH.bond_strengths(mat, lo.reshape(-1), hi.reshape(-1))
        self.kw = self.pc.kw(slot_br.astype(np.float32).reshape(-1), sn, stn)
        self.st = st
        self.n = n

    def step(self):
        self.sim.oracle_step(self.st, self.pc.sc, **self.kw)

    def bonds(self):
        """Intact undirected bonds (i < j) and their radii."""
        n, P = self.n, self.pc.IonP
        IL = self.st.IL.reshape(n, P)
        ty = self.st.ILtype.reshape(n, P)
        r, c = np.nonzero((IL != 0xFFFFFFFF) & (ty == 1))
        j = IL[r, c]
        keep = r < j
        br = self.kw["slot_br"].reshape(n, P)[r, c]
        return r[keep].astype(np.uint32), j[keep].astype(np.uint32), br[keep].astype(np.float32)


def algorithmic_bytes(n, bonds, touching, fp64=False):
    """Per step: 60 N + 104 B + 28 C bytes (FP32), 120 N + 204 B + 52 C (FP64):
    particle R,V,W read + F,M written; per undirected bond j, L0 and four
    3-vector histories read and written; per touching contact j and the
    tangential history read and written."""
    if fp64:
        return 120.0 * n + 204.0 * bonds + 52.0 * touching
    return 60.0 * n + 104.0 * bonds + 28.0 * touching


def particle_bytes(n, fp64=False):
    """Per step, the particle kernel: position, velocity, spin, list reference,
    force and moment read (6 x 16 B), sample id and platen flag (5 B);
    position, velocity and spin written and the force and moment
    accumulators reset (5 x 16 B): 181 B per particle (FP64: 357 B)."""
    return (357.0 if fp64 else 181.0) * n


def cpu_baseline(specs, nsteps: int, warmup: int, threads: int):
    """Times nsteps loop bodies of every specimen (after `warmup` untimed
    ones) on `threads` host threads: particle-steps/s, seconds, threads."""
    from oracle import lib as L

    L.lib().orc_set_threads(threads)
    steps = [CpuStep(sp) for sp in specs]
    for _ in range(warmup):
        for c in steps:
            c.step()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        for c in steps:
            c.step()
    el = time.perf_counter() - t0
    n = sum(c.n for c in steps)
    return n * nsteps / el, el, L.lib().orc_get_threads(), steps


def reference_bpm_cpu(spec, bonds, seconds: float = 3.0, max_bonds: int = 20000):
    """The reference's own CPU BPM routine, h_CalculateForceElastic
    (md_calculateforcesbpm_cpu.cu:20-262), compiled from the reference sources
    into oracle/_ref/libdemref.so: one call per directed bond slot of the
    specimen's first max_bonds intact bonds (fresh bond state; bonds and radii
    from the oracle's set-up), on one host thread (the routine prints on every
    call and is not re-entrant; its output goes to /dev/null), for `seconds`.
    Reported as directed-bond evaluations per second and as the
    particle-steps/s of a BPM-only step (2 B evaluations per step over the
    whole specimen)."""
    try:
        from oracle import lib as L
        R = L.ref()
    except Exception as e:                      # library not built / not shipped
        return {"value": None, "unavailable": f"oracle/_ref/libdemref.so: {type(e).__name__}: {e}"[:200]}
    bi_all, bj_all, br_all = bonds
    bi = np.ascontiguousarray(bi_all[:max_bonds])
    bj = np.ascontiguousarray(bj_all[:max_bonds])
    br = np.ascontiguousarray(br_all[:max_bonds])
    n = spec.n
    Rs = np.ascontiguousarray(spec.xyz, np.float32)
    V = np.zeros(3 * n, np.float32)
    W = np.zeros(3 * n, np.float32)
    m = spec.material
    ev, sec = C.c_double(), C.c_double()
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = R.refh_time_bpm_cpu(P(Rs), P(V), P(W), n, P(bi), P(bj), P(br), bi.size, 1e-3, m.E_bond,
                             m.E_bond / m.kn_ks, m.Ec, m.Gc, seconds, C.byref(ev), C.byref(sec))
    if rc != 0:
        return {"value": None, "unavailable": f"refh_time_bpm_cpu returned {rc}"}
    B = int(bi_all.size)
    return {"value": n * ev.value / (2.0 * B), "unit": UNIT, "cores": 1, "kind": "reference",
            "bond_evaluations_per_s": ev.value, "seconds": sec.value,
            "sample": f"h_CalculateForceElastic over {bi.size} of the {B} bonds of the {n}-sphere specimen, "
                      f"both directions, repeated for {sec.value:.1f} s; value = particle-steps/s of a BPM-only "
                      f"step (2 x {B} evaluations)"}


def run_reference(args, ws, rank, local):
    """--impl reference: the reference's loop body restated by the oracle (the
    reference has no CPU implementation of the step; its kernels are CUDA) on
    all host threads, over the same specimens as the engine's leg - built on
    the host by the CPU restatement of the packer, bit for bit the GPU's
    packing - for exactly --warmup untimed and --steps timed steps.  Rank 0
    alone runs; the product library is not loaded."""
    if rank != 0:
        return 0
    from oracle import pack

    dem = importlib.import_module("dem-rock-calibration_b200")   # Python helpers only (no library load)
    t0 = time.perf_counter()
    specs = [build_specimen(dem, args.workload, sd, local, packer=pack.create_cylinder_sample)
             for sd in specimen_seeds(args, 0)]
    t_pack = time.perf_counter() - t0
    threads = os.cpu_count() or 1
    v, el, th, steps = cpu_baseline(specs, args.steps, args.warmup, threads)
    n = sum(sp.n for sp in specs)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded packings, FIRE-relaxed)",
            "config": workload_config(args, specs, ws),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": th, "kind": "port",
                             "sample": f"{args.steps} full loading steps (cells, list rebuild, BPM, HM, platens, "
                                       f"integration) of each of the {len(specs)} specimens ({n} spheres)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "details": {"packing_seconds_untimed": t_pack,
                        "packing": [sp.pack for sp in specs],
                        "note": "specimens packed on the host by oracle/dem_pack_oracle.c (the engine's packer "
                                "restated; identical packings); the reference's own step is CUDA only, so the "
                                "oracle's restatement of it stands in on the CPU"}}
    line["cpu_baseline_reference_bpm"] = reference_bpm_cpu(specs[0], steps[0].bonds())
    print(json.dumps(line), flush=True)
    return 0


def sweep_sizes(k: int, seed: int = 11) -> list[int]:
    """k cylinder sizes, particle counts spread over [5k, 60k] (seeded, shuffled)."""
    rng = np.random.default_rng(seed)
    return [int(v) for v in rng.permutation(np.linspace(5000, 60000, k).round())]


def run_sweep(args, ws, rank, local):
    """Batched calibration sweep: `cases` Latin-hypercube parameter sets per
    rank over 16 packed cylinders (5k-60k spheres) in one context, against the
    same cases one context at a time.  Under torchrun one sweep of
    cases x ranks parameter sets is split into contiguous blocks (weak
    scaling); after the timed steps the ranks exchange the per-case macro
    properties, so every rank holds the whole sweep's results."""
    sweep = importlib.import_module("dem-rock-calibration_b200.sweep")
    D = Dist(ws)
    n_total = args.cases * ws
    sw = sweep.build_sweep(n_total, sweep_sizes(16, 11), seed=1, device=local, only=sweep.shard(n_total, rank, ws))
    n = sw.particles
    dem = importlib.import_module("dem-rock-calibration_b200")
    # launch schedule and contact-list skin chosen by the engine's autotuner on
    # a scratch context of the same cases (its tuning steps advance that run),
    # then applied to a fresh context, so the timed steps start from set-up
    tune = None
    if args.pair_min_blocks == 0:
        scratch = dem.Context(device=local, graph_steps=200, skin_factor=args.skin)
        for c in sw.cases:
            scratch.add_sample(c.material, c.loading, c.xyz, c.radii)
        scratch.setup()
        tune = scratch.autotune(max(20, min(args.steps, 100)))
        scratch.close()
    ctx = dem.Context(device=local, graph_steps=200,
                      pair_min_blocks=tune["pair_min_blocks"] if tune else args.pair_min_blocks,
                      particle_block=tune["particle_block"] if tune else 0,
                      skin_factor=tune["skin_factor"] if tune else args.skin)
    for c in sw.cases:
        ctx.add_sample(c.material, c.loading, c.xyz, c.radii)
    ctx.setup()
    ctx.run_timed(args.warmup)
    D.barrier()
    clk = Clocks(local)
    ms = ctx.run_timed(args.steps)
    clocks = clk.stop()
    D.barrier()
    ms_max = D.max(ms)
    value = D.sum(float(n)) * args.steps / (ms_max * 1e-3)
    prof = ctx.profile(min(args.steps, 200))
    res = [ctx.result(i) for i in range(len(sw.cases))]
    ctx.close()
    whole = sweep.gather_results({c.index: r for c, r in zip(sw.cases, res)}, n_total)
    gathered = {"cases": len(whole), "done": sum(r["done"] for r in whole),
                "bonds_broken": sum(r["bonds_initial"] - r["bonds_now"] for r in whole),
                "max_stress_mean_GPa": float(np.mean([r["FractureStress"] for r in whole]))}
    # the same cases one context at a time, a bounded sample of them
    k_seq = min(len(sw.cases), 32)
    sub = sweep.Sweep(cases=sw.cases[:k_seq])
    seq = sweep.run_sequential(sub, args.steps, device=local)
    n_sub = sub.particles
    seq_rate = n_sub * args.steps / (seq["device_ms"] * 1e-3)
    bonds = sum(r["bonds_now"] for r in res)
    A = algorithmic_bytes(n, bonds, prof["touching"])
    achieved = A / (prof["pair_ms"] * 1e-3) / 1e9
    peak, peak_kind = peaks()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded packings, Latin-hypercube micro-parameters)",
        "config": {"workload": f"calibration sweep: {len(sw.cases)} uniaxial cylinders (16 packings, "
                               f"{min(c.n for c in sw.cases)}-{max(c.n for c in sw.cases)} spheres) in one context",
                   "particles_per_gpu": n, "cases": len(sw.cases), "bonds": bonds,
                   "sweep_results_gathered": gathered,
                   "sequential": {"cases": k_seq, "particles": n_sub, "value": seq_rate,
                                  "device_ms": seq["device_ms"],
                                  "note": "the same cases one context at a time (device time summed)"},
                   "batched_over_sequential": value / D.sum(seq_rate),
                   "autotune": tune,
                   "l2": "inputs larger than L2, no flush"},
        "gpu_launches": 2 * args.steps, "clocks": clocks,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "k_pairs", "pair_ms": prof["pair_ms"],
                     "particle_ms": prof["particle_ms"], "algorithmic_bytes_per_step": A, "peak_kind": peak_kind},
        "e2e": None, "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    D.close()
    return 0


def surrogate_flops(sizes, rows: int) -> float:
    """Algorithmic FLOPs of one training pass over `rows` samples: forward
    GEMMs, weight-gradient GEMMs, and input-gradient GEMMs of every layer but
    the first (unpadded layer sizes)."""
    mm = [a * b for a, b in zip(sizes[:-1], sizes[1:])]
    return 2.0 * rows * (2 * sum(mm) + sum(mm[1:]))


def S_space():
    return importlib.import_module("dem-rock-calibration_b200.sweep").SWEEP_SPACE


def run_surrogate(args, ws, rank, local):
    """Surrogate MLP 6-256-256-256-4 (GELU, BF16 operands, FP32 accumulation in
    tensor memory) trained by mini-batch Adam (batch 256) on 8192 samples, one
    CUDA-graph replay per epoch; every rank trains its own network (weak
    scaling).  Inputs are the six sweep micro-parameters scaled to [-1, 1],
    targets a seeded smooth four-output map standing in for (UCS, E, nu,
    tensile strength) of simulated specimens - or, with --sim-data N, the
    properties of N Latin-hypercube parameter sets simulated first by the
    batched engine (uniaxial and Brazilian tests of 2,000-sphere specimens,
    deterministic mode), reported with the simulation rate and the held-out
    error of the trained network.  Also times the forward GEMM of a
    65,536-candidate proposal batch."""
    import torch
    S = importlib.import_module("dem-rock-calibration_b200.surrogate")
    D = Dist(ws)
    torch.cuda.set_device(local)
    sizes = (6, 256, 256, 256, 4)
    batch = 256
    sim = None
    if args.sim_data > 0:
        Xs, Ys, t_sim = S.simulate_dataset(args.sim_data, seed=1 + rank,
                                           uni=S.UniaxialSolver(n=args.sim_size, device=local),
                                           braz=S.BrazilSolver(n=args.sim_size, device=local), batch=args.sim_batch)
        ok = np.all(np.isfinite(Ys), axis=1) & (Ys[:, 0] > 0) & (Ys[:, 3] > 0)
        Xs, Ys = Xs[ok], Ys[ok]
        lo = np.array([v[0] for v in S_space().values()])
        hi = np.array([v[1] for v in S_space().values()])
        Xn = (2.0 * (Xs - lo) / (hi - lo) - 1.0).astype(np.float32)
        mu_y, sd_y = Ys.mean(0), Ys.std(0) + 1e-30
        Yn = ((Ys - mu_y) / sd_y).astype(np.float32)
        n_test = max(1, len(Xn) // 10)
        X, Y = Xn[n_test:], Yn[n_test:]
        if args.sim_save:
            np.savez(args.sim_save, X=Xs, Y=Ys)
        sim = dict(cases=int(args.sim_data), kept=int(ok.sum()), seconds=t_sim, spheres=args.sim_size,
                   batch=args.sim_batch, train=int(len(X)), held_out=int(n_test),
                   solves_per_hour=2 * args.sim_data / t_sim * 3600.0,
                   test=(Xn[:n_test], Yn[:n_test], sd_y))
    else:
        n = 8192
        rng = np.random.default_rng(17 + rank)
        X = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
        Y = np.stack([np.sin(2 * X[:, 0]) + X[:, 1] ** 2 - X[:, 3], X[:, 2] * X[:, 3] + 0.5 * X[:, 0],
                      np.exp(0.5 * X[:, 4]) - X[:, 5] * X[:, 1], X[:, 0] * X[:, 5] + 0.3 * X[:, 2]], 1)
        Y = ((Y - Y.mean(0)) / Y.std(0)).astype(np.float32)
    net = S.MLP(sizes, seed=rank, device=local)
    ep = S.Epochs(net, X, Y, batch, seed=rank)
    loss0 = ep.run()
    for _ in range(max(args.warmup, 3)):
        ep.run()
    epochs = max(1, args.steps)
    D.barrier()
    clk = Clocks(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ep.stream.synchronize()
    e0.record(ep.stream)
    for _ in range(epochs):
        ep.launch()
    e1.record(ep.stream)
    e1.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    loss1 = float(net.loss_acc.item()) / len(ep.sizes)
    D.barrier()
    ms_max = D.max(ms)
    rows = ep.n
    value = D.sum(float(rows)) * epochs / (ms_max * 1e-3)
    flops = surrogate_flops(sizes, rows) * epochs
    ep.close()
    if sim is not None:
        # held-out error of the trained network, per property, in units of that
        # property's spread over the dataset, and relative to its mean magnitude
        Xt, Yt, sd_y = sim.pop("test")
        pred = net.predict(Xt)
        rmse = np.sqrt(np.mean((pred - Yt) ** 2, axis=0))
        sim["test_rmse_in_sd"] = dict(zip(("UCS", "E", "nu", "sigma_t"), map(float, rmse)))
    # inference GEMM of a 65,536-candidate proposal batch (hidden layer 256 x 256:
    # bias + GELU, BF16 out, no pre-activation kept), alone
    M, N, K = 65536, 256, 256
    A = torch.randn(M, K, device=net.dev).to(torch.bfloat16)
    Bm = torch.randn(N, K, device=net.dev).to(torch.bfloat16)
    bias = torch.zeros(N, device=net.dev)
    zh = torch.empty(M, N, dtype=torch.bfloat16, device=net.dev)
    P = lambda t: C.c_void_p(t.data_ptr())
    st = torch.cuda.current_stream(net.dev)
    call = lambda: net.L.dem_mlp_gemm_tn(P(A), P(Bm), M, N, K, P(bias), S.BIAS_GELU, None, P(zh),
                                         C.c_void_p(st.cuda_stream))
    for _ in range(5):
        call()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 50
    # eager calls (each pays its host work: argument checks, tensor maps, launch)
    g0.record(st)
    for _ in range(reps):
        call()
    g1.record(st)
    g1.synchronize()
    gemm_call_ms = g0.elapsed_time(g1) / reps
    # device time: the same launches captured in one CUDA graph and replayed
    cs = torch.cuda.Stream(net.dev)
    graph = torch.cuda.CUDAGraph()
    callg = lambda: net.L.dem_mlp_gemm_tn(P(A), P(Bm), M, N, K, P(bias), S.BIAS_GELU, None, P(zh),
                                          C.c_void_p(cs.cuda_stream))
    with torch.cuda.graph(graph, stream=cs):
        for _ in range(reps):
            callg()
    graph.replay()
    torch.cuda.synchronize(net.dev)
    g0.record(st)
    graph.replay()
    g1.record(st)
    g1.synchronize()
    gemm_ms = g0.elapsed_time(g1) / reps
    del graph
    net.check()
    gemm_tf = 2.0 * M * N * K / (gemm_ms * 1e-3) / 1e12
    # algorithmic bytes: A and B read once, BF16 output written once; at width
    # 256 the arithmetic intensity (about 130 flop/byte) is below the B200
    # ridge (measured bf16 peak / measured HBM bandwidth, about 250), so HBM
    # bounds this layer
    gemm_bytes = 2.0 * M * K + 2.0 * N * K + 2.0 * M * N
    hbm_peak, _ = peaks()
    # end to end through the public API: host arrays in, a fitted network and host predictions out
    t0 = time.perf_counter()
    net2 = S.MLP(sizes, seed=rank + 100, device=local)
    net2.fit(X, Y, epochs=epochs, batch=batch, seed=rank)
    _ = net2.predict(X[:batch])
    t_e2e = time.perf_counter() - t0
    peak_tf, peak_kind = tensor_peak()
    line = {
        "metric": "surrogate training samples/s", "value": value, "unit": "samples/s", "n_gpus": ws,
        "steps": epochs, "warmup": max(args.warmup, 3), "ms_per_step": ms_max / epochs, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 operands, f32 accumulation",
        "data": ("simulated: batched uniaxial + Brazilian solves of Latin-hypercube parameter sets"
                 if sim is not None else "synthetic (seeded inputs in the sweep box, smooth 4-output targets)"),
        "config": {"workload": f"surrogate MLP {'-'.join(map(str, sizes))} GELU, {rows} samples per epoch, "
                               f"batch {batch}, Adam", "step": "one epoch (one CUDA-graph replay)",
                   "loss_first_epoch": loss0, "loss_last_epoch": loss1, "simulated_dataset": sim,
                   "train_tflops": flops / (ms_max * 1e-3) / 1e12,
                   "l2": "dataset and weights inside the L2 (the whole job is 10 MB)"},
        "gpu_launches": epochs * sum(net.launches_per_step(b) for b in ep.sizes),
        "clocks": clocks,
        "roofline": (lambda ai, ridge, gbs: {
            "bound": "hbm" if ai < ridge else "tensor",
            "achieved": gbs if ai < ridge else gemm_tf, "peak": hbm_peak if ai < ridge else peak_tf,
            "unit": "GB/s" if ai < ridge else "TFLOP/s",
            "frac": gbs / hbm_peak if ai < ridge else gemm_tf / peak_tf, "traffic": None,
            "kernel": f"k_gemm_tn<256> forward layer {M} x {N} x {K} (bias + GELU epilogue, BF16 out)",
            "gemm_us": gemm_ms * 1e3, "gemm_eager_call_us": gemm_call_ms * 1e3, "tflops": gemm_tf, "tensor_frac": gemm_tf / peak_tf,
            "arithmetic_intensity": ai, "ridge": ridge, "algorithmic_bytes": gemm_bytes,
            "peak_kind": peak_kind})(2.0 * M * N * K / gemm_bytes, peak_tf * 1e12 / (hbm_peak * 1e9),
                                     gemm_bytes / (gemm_ms * 1e-3) / 1e9),
        "e2e": {"value": rows * epochs / t_e2e, "unit": "samples/s",
                "h2d_bytes_per_step": (X.nbytes + Y.nbytes) / epochs, "d2h_bytes_per_step": 4.0 * 2,
                "seconds": t_e2e, "note": "MLP.fit from host arrays (upload, eager first epoch, graph capture, "
                                          "replays, loss read per epoch) plus one host prediction"},
        "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    D.close()
    return 0


def run_solves_cfg2(args, ws, rank, local):
    """Calibration solves per hour at the batched configuration's sizes:
    `cases` Latin-hypercube parameter sets over 16 packed cylinders of 5k-60k
    spheres (case k on cylinder k mod 16), uniaxial tests to 70% post-peak
    (or 1% strain), deterministic mode.  Batched: all cases in one context,
    until the last one finishes.  Plain: one context per solve, one after
    another, for one case per cylinder (16 solves covering the size range).
    Wall-clock per whole solve (context, set-up, loading, results)."""
    sweep = importlib.import_module("dem-rock-calibration_b200.sweep")
    dem = importlib.import_module("dem-rock-calibration_b200")
    D = Dist(ws)
    max_steps = 2_000_000
    sw = sweep.build_sweep(args.cases, sweep_sizes(16, 11 + rank), seed=1 + rank, max_steps=max_steps, device=local)

    def solve(cases):
        ctx = dem.Context(device=local, graph_steps=200, deterministic=True)
        ids = [ctx.add_sample(c.material, c.loading, c.xyz, c.radii) for c in cases]
        ctx.setup()
        ctx.run(max_steps)
        res = [ctx.result(i) for i in ids]
        ctx.close()
        return res

    solve(sw.cases[:2])                                   # kernel loading, allocator warm-up
    D.barrier()
    clk = Clocks(local)
    t0 = time.perf_counter()
    res_b = solve(sw.cases)
    t_b = time.perf_counter() - t0
    clocks = clk.stop()
    t_b = D.max(t_b)
    plain_cases = sw.cases[:16]
    t0 = time.perf_counter()
    res_p = [solve([c])[0] for c in plain_cases]
    t_p = time.perf_counter() - t0
    agree = max(abs(a["FractureStress"] - b["FractureStress"]) / max(abs(b["FractureStress"]), 1e-30)
                for a, b in zip(res_b[:16], res_p))
    value = D.sum(float(len(sw.cases))) / t_b * 3600.0
    plain = D.sum(len(plain_cases) / t_p * 3600.0)
    steps = [r["steps"] for r in res_b]
    line = {
        "metric": "calibration solves/hour", "value": value, "unit": "solves/hour", "n_gpus": ws, "steps": 1,
        "warmup": 1, "ms_per_step": t_b * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded packings, Latin-hypercube micro-parameters)",
        "config": {"workload": f"{len(sw.cases)} uniaxial solves over 16 cylinders of 5k-60k spheres "
                               f"({sw.particles} spheres in all) to 70% post-peak or 1% strain, one context",
                   "step": "the whole batch of solves, wall-clock (context, set-up, loading, results)",
                   "plain": {"solves": len(plain_cases), "seconds": t_p, "value": plain,
                             "note": "one context per solve, one after another, one case per cylinder size"},
                   "batched_over_plain": value / plain, "max_rel_difference_batched_vs_plain_ucs": agree,
                   "solve_steps_range": [min(steps), max(steps)], "all_done": all(r["done"] for r in res_b),
                   "l2": "state above the L2 (batch); no flush"},
        "gpu_launches": None, "clocks": clocks, "roofline": None, "e2e": None, "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    D.close()
    return 0


def solves_measure(args, rank, local, cases: int, plain_cases: int, D=None) -> dict:
    """Calibration solves per hour: `cases` uniaxial tests of one packed
    cylinder of about 2,000 spheres (Latin-hypercube micro-parameters over the
    sweep box), each run until its peak has passed (stress down to 70% of the
    peak) or 1% strain, all in one context; against the same solves one
    context at a time (the plain method: one specimen per run, as the
    reference's CalculateOneSample), on the first `plain_cases` cases.  Times
    are wall-clock per whole solve (context, set-up, loading to the end,
    results back), the unit a calibration pays for.  D (optional): the timing
    barrier and max over ranks."""
    import torch
    S = importlib.import_module("dem-rock-calibration_b200.surrogate")
    sweep = importlib.import_module("dem-rock-calibration_b200.sweep")
    torch.cuda.set_device(local)
    J = S.UniaxialSolver(n=2000, seed=5 + rank, device=local)
    lo = np.array([v[0] for v in sweep.SWEEP_SPACE.values()])
    hi = np.array([v[1] for v in sweep.SWEEP_SPACE.values()])
    X = S.latin_box(cases, lo, hi, 1 + rank)
    for _ in range(max(1, min(args.warmup, 3))):
        J(X[:2])                                       # kernel loading, allocator warm-up
    if D is not None:
        D.barrier()
    clk = Clocks(local)
    t0 = time.perf_counter()
    Yb = J(X)
    t_b = time.perf_counter() - t0
    clocks = clk.stop()
    if D is not None:
        t_b = D.max(t_b)
    k = min(cases, plain_cases)
    t0 = time.perf_counter()
    Ys = np.vstack([J(X[i:i + 1]) for i in range(k)])
    t_s = time.perf_counter() - t0
    agree = float(np.max(np.abs(Yb[:k] - Ys) / np.maximum(np.abs(Ys), 1e-30)))
    return dict(n=J.rad.size, cases=cases, t_b=t_b, plain_cases=k, t_s=t_s, agree=agree, clocks=clocks,
                ucs=[float(Yb[:, 0].min()), float(Yb[:, 0].max())])


def run_solves(args, ws, rank, local):
    """Calibration solves per hour, batched against plain (solves_measure);
    every rank solves its own cases (weak scaling)."""
    D = Dist(ws)
    m = solves_measure(args, rank, local, args.cases, 32, D)
    value = D.sum(float(args.cases)) / m["t_b"] * 3600.0
    plain = D.sum(float(m["plain_cases"]) / m["t_s"] * 3600.0)
    line = {
        "metric": "calibration solves/hour", "value": value, "unit": "solves/hour", "n_gpus": ws, "steps": 1,
        "warmup": max(1, min(args.warmup, 3)), "ms_per_step": m["t_b"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded packing, Latin-hypercube micro-parameters)",
        "config": {"workload": f"{args.cases} uniaxial solves of a {m['n']}-sphere cylinder to 70% post-peak "
                               f"(or 1% strain) in one context",
                   "step": "the whole batch of solves, wall-clock (context, set-up, loading, results)",
                   "plain": {"solves": m["plain_cases"], "seconds": m["t_s"], "value": plain,
                             "note": "one context per solve, one after another"},
                   "batched_over_plain": value / plain,
                   "max_rel_difference_batched_vs_plain": m["agree"],
                   "ucs_gpa_range": m["ucs"],
                   "l2": "whole state inside the L2 (small specimens); no flush"},
        "gpu_launches": None, "clocks": m["clocks"], "roofline": None, "e2e": None, "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    D.close()
    return 0


def postpeak_measure(dem, args, specs, local, steps: int, warmup: int, D=None) -> dict:
    """The discs `specs` loaded past the peak first (platens at ten times the
    configuration's speed, no stop condition) until every disc has lost
    `args.damage` of its bonds, then `steps` timed steps in which broken
    bonds and new touching pairs make the Hertz-Mindlin contacts and the
    contact-list rebuilds part of every step.  D (optional): the timing
    barrier and max over ranks."""
    ctx = dem.Context(precision=args.precision, device=local, graph_steps=200, pair_min_blocks=args.pair_min_blocks,
                      deterministic=args.deterministic, skin_factor=args.skin)
    sids = []
    for sp in specs:
        ld = dem.Loading.from_buffer_copy(sp.loading)
        ld.velocity *= 10.0
        ld.min_stress = 1.0                      # 1 GPa: the fracture test never arms
        ld.max_strain = 0.5
        sids.append(ctx.add_sample(sp.material, ld, sp.xyz, sp.radii))
    ctx.setup()
    t0 = time.perf_counter()
    prep = 0
    while prep < 400000:
        ctx.step(5000)
        prep += 5000
        res = [ctx.result(s) for s in sids]
        if all(r["bonds_now"] <= (1.0 - args.damage) * r["bonds_initial"] for r in res):
            break
    t_prep = time.perf_counter() - t0
    n_gpu = ctx.counts()["particles"]
    ctx.run_timed(warmup)
    rb0 = ctx.result(sids[0])["rebuilds"]
    if D is not None:
        D.barrier()
    clk = Clocks(local)
    ms = ctx.run_timed(steps)
    clocks = clk.stop()
    if D is not None:
        D.barrier()
    rb1 = ctx.result(sids[0])["rebuilds"]
    prof = ctx.profile(min(steps, 300))
    res = [ctx.result(s) for s in sids]
    cnt = ctx.counts()
    ctx.close()
    bonds = sum(r["bonds_now"] for r in res)
    A = algorithmic_bytes(n_gpu, bonds, prof["touching"], fp64=args.precision == 1)
    achieved = A / (prof["pair_ms"] * 1e-3) / 1e9
    peak, peak_kind = peaks()
    return dict(n_gpu=n_gpu, ms=ms, clocks=clocks, prep=prep, t_prep=t_prep, rebuilds_timed=rb1 - rb0, prof=prof,
                bonds=bonds, bonds_initial=sum(r["bonds_initial"] for r in res), contacts=cnt["contacts"],
                stale=sum(r["stale"] for r in res), done=[r["done"] for r in res], A=A, achieved=achieved, peak=peak,
                peak_kind=peak_kind)


def run_postpeak(args, ws, rank, local):
    """The default workload's discs loaded past the peak, then timed
    (postpeak_measure).  Every rank loads its own discs (weak scaling)."""
    dem = importlib.import_module("dem-rock-calibration_b200")
    D = Dist(ws)
    specs = [build_specimen(dem, "brazilian_disc", sd, local) for sd in specimen_seeds(args, rank)]
    m = postpeak_measure(dem, args, specs, local, args.steps, args.warmup, D)
    ms_max = D.max(m["ms"])
    value = D.sum(float(m["n_gpu"])) * args.steps / (ms_max * 1e-3)
    prof = m["prof"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == 1 else "f32", "data": "synthetic (seeded packings, FIRE-relaxed)",
        "config": {"workload": f"{args.specimens} x brazilian_disc loaded past the peak ({args.damage:.0%} of the "
                               f"bonds broken)", "particles_per_gpu": m["n_gpu"], "specimens": args.specimens,
                   "seeds": specimen_seeds(args, 0), "parallelism": f"{ws} GPU(s), independent specimens",
                   "l2": "inputs larger than L2, no flush"},
        "details": {"bonds_intact": m["bonds"], "bonds_initial": m["bonds_initial"],
                    "contacts_listed": m["contacts"], "touching_contacts": prof["touching"],
                    "contact_list_builds_timed": m["rebuilds_timed"], "preparation_steps": m["prep"],
                    "preparation_seconds_untimed": m["t_prep"], "stale_lists": m["stale"], "done": m["done"]},
        "gpu_launches": None, "clocks": m["clocks"],
        "roofline": {"bound": "hbm", "achieved": m["achieved"], "peak": m["peak"], "unit": "GB/s",
                     "frac": m["achieved"] / m["peak"], "traffic": None,
                     "kernel": "k_pairs (BPM bonds + Hertz-Mindlin contacts)",
                     "pair_ms": prof["pair_ms"], "particle_ms": prof["particle_ms"],
                     "algorithmic_bytes_per_step": m["A"], "peak_kind": m["peak_kind"]},
        "e2e": None, "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    D.close()
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="brazilian_disc",
                    choices=["brazilian_disc", "brazilian_disc_postpeak", "uniaxial_cylinder", "calibration_sweep",
                             "calibration_solves", "surrogate"])
    ap.add_argument("--solve-sizes", default="2000", choices=["2000", "cfg2"],
                    help="calibration_solves: one 2,000-sphere cylinder, or 16 cylinders of 5k-60k spheres")
    ap.add_argument("--damage", type=float, default=0.03,
                    help="brazilian_disc_postpeak: fraction of the bonds broken before the timed steps")
    ap.add_argument("--cases", type=int, default=256, help="calibration_sweep: parameter sets")
    ap.add_argument("--pair-min-blocks", type=int, default=0, help="pair kernel register budget (blocks per SM)")
    ap.add_argument("--cpu-steps", type=int, default=6)
    ap.add_argument("--solves-cases", type=int, default=256,
                    help="brazilian_disc: also time this many batched calibration solves (0: skip)")
    ap.add_argument("--post-peak-steps", type=int, default=200,
                    help="brazilian_disc: also time this many steps of the discs after the peak (0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--sim-size", type=int, default=2000, help="surrogate --sim-data: spheres per specimen")
    ap.add_argument("--sim-batch", type=int, default=256, help="surrogate --sim-data: parameter sets per context")
    ap.add_argument("--sim-save", default="", help="surrogate --sim-data: write the dataset (X, Y) to this .npz")
    ap.add_argument("--sim-data", type=int, default=0,
                    help="surrogate: train on this many simulated parameter sets instead of synthetic targets")
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1],
                    help="0: FP32 (default), 1: FP64 build (the Brazilian configuration's FP64 case)")
    ap.add_argument("--skin", type=float, default=0.0,
                    help="contact-list skin as a multiple of the smallest radius (0: the engine default, 0.1)")
    ap.add_argument("--deterministic", action="store_true",
                    help="exact fixed-point force sums (bit-reproducible runs) instead of float atomics")
    ap.add_argument("--specimens", type=int, default=2,
                    help="specimens of the workload advanced together per GPU (2 discs: state above the L2)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_env()
    if args.impl == "reference":
        if args.workload not in ("brazilian_disc", "uniaxial_cylinder"):
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": f"the reference leg times the loop body on the "
                                  f"specimen workloads only, not {args.workload}"}), flush=True)
            return 0
        return run_reference(args, ws, rank, local)
    if args.workload == "calibration_sweep":
        return run_sweep(args, ws, rank, local)
    if args.workload == "surrogate":
        return run_surrogate(args, ws, rank, local)
    if args.workload == "calibration_solves":
        return run_solves_cfg2(args, ws, rank, local) if args.solve_sizes == "cfg2" else run_solves(args, ws, rank,
                                                                                                    local)
    if args.workload == "brazilian_disc_postpeak":
        return run_postpeak(args, ws, rank, local)
    dem = importlib.import_module("dem-rock-calibration_b200")
    D = Dist(ws)
    specs = [build_specimen(dem, args.workload, sd, local) for sd in specimen_seeds(args, rank)]
    spec = specs[0]
    ctx = dem.Context(precision=args.precision, device=local, graph_steps=200, pair_min_blocks=args.pair_min_blocks,
                      deterministic=args.deterministic, skin_factor=args.skin)
    sids = [ctx.add_sample(sp.material, sp.loading, sp.xyz, sp.radii) for sp in specs]
    ctx.setup()
    cnt = ctx.counts()
    n_gpu = cnt["particles"]
    ctx.run_timed(args.warmup)
    rb0 = ctx.result(sids[0])["rebuilds"]
    D.barrier()
    clk = Clocks(local)
    ms = ctx.run_timed(args.steps)
    clocks = clk.stop()
    D.barrier()
    rb1 = ctx.result(sids[0])["rebuilds"]
    ms_max = D.max(ms)
    n_total = D.sum(float(n_gpu))
    value = n_total * args.steps / (ms_max * 1e-3)
    # per-kernel timing of the same pipeline (events around each launch)
    prof = ctx.profile(min(args.steps, 300))
    res = [ctx.result(s) for s in sids]
    bonds = sum(r["bonds_now"] for r in res)
    A = algorithmic_bytes(n_gpu, bonds, prof["touching"], fp64=args.precision == 1)
    achieved = A / (prof["pair_ms"] * 1e-3) / 1e9
    peak, peak_kind = peaks()
    w = 2 if args.precision == 1 else 1
    state_mb = (n_gpu * (7 * 16 * w + 8) + cnt["bonds"] * (8 + 4 * 16 * w) + cnt["contacts"] * 24 * w) / 1e6
    stale = sum(r["stale"] for r in res)
    ctx.close()
    # the same pipeline on one specimen alone (state inside the L2), for reference
    one = dem.Context(precision=args.precision, device=local, graph_steps=200, skin_factor=args.skin,
                      deterministic=args.deterministic)
    one.add_sample(spec.material, spec.loading, spec.xyz, spec.radii)
    one.setup()
    one.run_timed(args.warmup)
    ms1 = one.run_timed(args.steps)
    prof1 = one.profile(min(args.steps, 300))
    one.close()
    # end to end through the public API with host buffers: positions uploaded,
    # set-up (Morton sort, bonds, contact list), K steps, results and records read back
    t0 = time.perf_counter()
    e2 = dem.Context(precision=args.precision, device=local, graph_steps=200, skin_factor=args.skin,
                     deterministic=args.deterministic)
    for sp in specs:
        ld = dem.Loading.from_buffer_copy(sp.loading)
        ld.max_steps = args.steps
        e2.add_sample(sp.material, ld, sp.xyz, sp.radii)
    e2.setup()
    t_setup = time.perf_counter() - t0
    e2.run(args.steps)
    t_run = time.perf_counter() - t0 - t_setup
    recs = [e2.record(k) for k in range(len(specs))]
    res2 = [e2.result(k) for k in range(len(specs))]
    t_e2e = time.perf_counter() - t0
    t1 = time.perf_counter()
    e2.close()
    t_close = time.perf_counter() - t1
    e2e_val = D.sum(n_gpu * args.steps / t_e2e)
    h2d = sum(sp.xyz.nbytes + sp.radii.nbytes for sp in specs)
    d2h = sum(r.nbytes + b.nbytes for r, b in recs) + len(specs) * 160
    # the same discs after the peak (Hertz-Mindlin contacts and list rebuilds in
    # every step), this rank's GPU
    post = None
    if args.post_peak_steps > 0 and args.workload == "brazilian_disc":
        m = postpeak_measure(dem, args, specs, local, args.post_peak_steps, 20)
        post = {"value": m["n_gpu"] * args.post_peak_steps / (m["ms"] * 1e-3), "unit": UNIT,
                "ms_per_step": m["ms"] / args.post_peak_steps, "steps": args.post_peak_steps,
                "bonds_broken": 1.0 - m["bonds"] / m["bonds_initial"],
                "touching_contacts": m["prof"]["touching"], "contact_list_builds_timed": m["rebuilds_timed"],
                "stale_lists": m["stale"], "pair_ms": m["prof"]["pair_ms"], "particle_ms": m["prof"]["particle_ms"],
                "roofline_frac": m["achieved"] / m["peak"], "clocks": m["clocks"],
                "note": "rank 0's discs loaded past the peak at ten times the platen speed until "
                        f"{args.damage:.0%} of the bonds broke (untimed), then timed"}
    # calibration solves per hour, batched against one context per solve (this
    # rank's GPU): the batching half of the configurations' second metric
    solves = None
    if args.solves_cases > 0 and args.workload == "brazilian_disc":
        m = solves_measure(args, rank, local, args.solves_cases, 16)
        b, pl = m["cases"] / m["t_b"] * 3600.0, m["plain_cases"] / m["t_s"] * 3600.0
        solves = {"batched": b, "plain": pl, "unit": "solves/hour", "batched_over_plain": b / pl,
                  "cases": m["cases"], "plain_solves": m["plain_cases"], "spheres": m["n"],
                  "max_rel_difference_batched_vs_plain": m["agree"], "clocks": m["clocks"],
                  "note": f"{m['cases']} uniaxial solves of a {m['n']}-sphere cylinder to 70% post-peak (or 1% "
                          "strain), deterministic sums, Latin-hypercube micro-parameters, in one context, against "
                          f"the first {m['plain_cases']} solved one context at a time; wall-clock per whole solve"}
    cpu = cpu_bpm = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        v, el, th, steps = cpu_baseline([spec], args.cpu_steps, 1, os.cpu_count() or 1)
        cpu = {"value": v, "unit": UNIT, "cores": th, "kind": "port",
               "sample": f"{args.cpu_steps} full loading steps (cells, list rebuild, BPM, HM, platens, "
                         f"integration) of the {spec.n}-sphere specimen"}
        cpu_bpm = reference_bpm_cpu(spec, steps[0].bonds())
    default_disc = (args.workload == "brazilian_disc" and args.specimens == 2 and args.precision == 0
                    and not args.deterministic and args.skin in (0.0, 0.1))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == 1 else "f32", "data": "synthetic (seeded packings, FIRE-relaxed)",
        "config": workload_config(args, specs, ws),
        "details": {"bonds": bonds, "contacts_listed": cnt["contacts"], "touching_contacts": prof["touching"],
                    "packing": spec.pack, "stale_lists": stale,
                    "force_sums": "fixed point (deterministic)" if args.deterministic else "float atomics",
                    "contact_list_builds_timed": rb1 - rb0, "state_mb": state_mb,
                    "single_specimen": {"particles": spec.n, "value": spec.n * args.steps / (ms1 * 1e-3),
                                        "ms_per_step": ms1 / args.steps, "pair_ms": prof1["pair_ms"],
                                        "note": "state inside the L2"},
                    "post_peak": post,
                    "calibration_solves": solves},
        "gpu_launches": 2 * args.steps,
        "clocks": clocks,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     # DRAM read + write bytes of one pair-kernel launch on this workload, from the ncu
                     # capture summarised in profiles/k_pairs_brazilian_disc_x2.md (not re-measured here)
                     "traffic": PAIR_TRAFFIC_DISC_X2 if default_disc else None,
                     "kernel": "k_pairs (BPM bonds + Hertz-Mindlin contacts)",
                     "pair_ms": prof["pair_ms"], "particle_ms": prof["particle_ms"],
                     "algorithmic_bytes_per_step": A, "peak_kind": peak_kind,
                     # the whole step (both kernels, launch gaps, rebuilds): bytes of the pair
                     # and particle kernels over the measured time per step
                     "step": {"bytes": A + particle_bytes(n_gpu, args.precision == 1),
                              "achieved": (A + particle_bytes(n_gpu, args.precision == 1))
                              / (ms_max / args.steps * 1e-3) / 1e9,
                              "frac": (A + particle_bytes(n_gpu, args.precision == 1))
                              / (ms_max / args.steps * 1e-3) / 1e9 / peak}},
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps, "seconds": t_e2e, "setup_seconds": t_setup,
                "run_seconds": t_run, "close_seconds_untimed": t_close,
                "contact_list_builds": res2[0]["rebuilds"],
                "note": "public API from host positions: upload, set-up, steps, results and records read back"},
        "cpu_baseline": cpu,
        "cpu_baseline_reference_bpm": cpu_bpm,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    D.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
