"""Surrogate MLP on the tensor cores: micro-parameters -> macro properties.

The reference's surrogate workflow (NN_MP.py:766-930) fits sklearn's
MLPRegressor (NN_MP.py:374-378; hidden layers 300-500-900-500-300, ReLU, Adam,
L2 alpha 1e-4, mini-batches of min(200, n)) on the CPU to the simulations run
so far (NN_MP.py:895), searches it with scipy's dual_annealing
(Material_Surface, NN_MP.py:384-395; NN_MP.py:896), runs new simulations around
the optimum it proposes (SetNTasksVariation, NN_MP.py:327-358) and repeats.

Here the network trains and predicts on the B200 through the library's own
kernels (dem_mlp_*: tcgen05 BF16 GEMMs with FP32 accumulation in tensor memory
and fused bias + activation epilogues, activation backward, column sums, MSE
gradient, Adam on FP32 master weights).  torch only holds the device buffers,
provides the stream and captures the CUDA graph of a training epoch; every
arithmetic step is a dem_mlp_* launch.

MLP            the network: forward, backward, Adam, fit, predict, input gradient
Surrogate      normalisation of parameters and properties around an MLP
propose        batched multi-start inversion: the parameter sets whose predicted
               properties are closest to a target
calibrate      the loop of the reference workflow with the batched simulator as
               the judge: fit, propose, simulate the proposals, accept a
               proposal only when the simulator confirms it, else add the new
               simulations to the data and refit
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import DemError, lib

PLAIN, BIAS, BIAS_GELU, BIAS_RELU = 0, 1, 2, 3
COLSUM_SPLIT = 32


def _r32(n: int) -> int:
    return (n + 31) // 32 * 32


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise DemError(-3, "the surrogate MLP needs a CUDA device (no CPU path)")
    return torch


def _ck(rc: int, what: str) -> None:
    if rc != 0:
        raise DemError(rc, what)


class MLP:
    """Dense network sizes[0] -> ... -> sizes[-1], hidden activation GELU (exact
    erf form) or ReLU, identity output, loss mean((y - t)^2).

    Device layout: layer l holds FP32 master weights W_l (out_p x in_p), a BF16
    copy, bias b_l (out_p) and Adam moments; in_p and the hidden out_p are the
    sizes rounded up to 32 (the GEMM's K step), the padding rows and columns
    are zero and stay zero under training (their gradients are exactly zero).
    Initialisation: sklearn's Glorot-uniform rule (bound sqrt(6 / (fan_in +
    fan_out))), seeded.
    """

    def __init__(self, sizes=(6, 256, 256, 256, 4), activation: str = "gelu", seed: int = 0, device: int = 0,
                 lr: float = 1e-3, l2: float = 0.0, betas=(0.9, 0.999), eps: float = 1e-8):
        torch = _torch()
        if activation not in ("gelu", "relu"):
            raise ValueError("activation is 'gelu' or 'relu'")
        self.torch, self.L = torch, lib()
        self.sizes = tuple(int(s) for s in sizes)
        self.activation = activation
        self.mode = BIAS_GELU if activation == "gelu" else BIAS_RELU
        self.dev = torch.device("cuda", device)
        self.lr, self.l2, self.b1, self.b2, self.eps = lr, l2, betas[0], betas[1], eps
        self.n_in, self.n_out = self.sizes[0], self.sizes[-1]
        self.kp = [_r32(s) for s in self.sizes[:-1]]                 # padded inputs of each layer
        self.np_ = self.kp[1:] + [self.n_out]                          # padded outputs of each layer
        rng = np.random.default_rng(seed)
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.W, self.b, self.Wh = [], [], []
        for l in range(len(self.sizes) - 1):
            fi, fo = self.sizes[l], self.sizes[l + 1]
            bound = np.sqrt(6.0 / (fi + fo))
            w = np.zeros((self.np_[l], self.kp[l]), np.float32)
            w[:fo, :fi] = rng.uniform(-bound, bound, (fo, fi))
            bb = np.zeros(self.np_[l], np.float32)
            bb[:fo] = rng.uniform(-bound, bound, fo)
            self.W.append(torch.from_numpy(w).to(self.dev))
            self.b.append(torch.from_numpy(bb).to(self.dev))
            self.Wh.append(self.W[-1].to(torch.bfloat16))
        self.params = self.W + self.b
        self.grads = [torch.zeros_like(p) for p in self.params]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.loss_acc = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.scratch = torch.zeros(COLSUM_SPLIT * max(self.np_ + self.kp), **f32)
        self._bufs = {}
        self._graph = None

    # ---- buffers -------------------------------------------------------
    def _buffers(self, B: int):
        if B in self._bufs:
            return self._bufs[B]
        t, bf = self.torch, self.torch.bfloat16
        Bp = _r32(B)
        mx = max(self.np_ + self.kp)
        f32 = dict(dtype=t.float32, device=self.dev)
        h16 = dict(dtype=bf, device=self.dev)
        bufs = dict(
            B=B, Bp=Bp,
            h=[t.zeros(B, k, **h16) for k in self.kp],                 # layer inputs (BF16)
            z=[t.zeros(B, n, **f32) for n in self.np_[:-1]],           # hidden pre-activations
            y=t.zeros(B, self.n_out, **f32),
            t=t.zeros(B, self.n_out, **f32),
            dy=t.zeros(B, self.n_out, **f32),
            dy16=t.zeros(B, self.n_out, **h16),
            dyp=t.zeros(B, 32, **h16),
            dh=t.zeros(B, mx, **f32),
            dz=t.zeros(B, mx, **f32),
            dz16=t.zeros(B, mx, **h16),
            aT=t.zeros(mx, Bp, **h16),
            hT=t.zeros(mx, Bp, **h16),
            wT=t.zeros(mx, mx, **h16),
            dx=t.zeros(B, self.kp[0], **f32),
        )
        self._bufs[B] = bufs
        return bufs

    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    @staticmethod
    def _ptr(x):
        return C.c_void_p(x.data_ptr())

    def _gemm(self, A, B_, M, N, K, bias, mode, outf, outh):
        P = self._ptr
        _ck(self.L.dem_mlp_gemm_tn(P(A), P(B_), M, N, K, None if bias is None else P(bias), mode,
                                   None if outf is None else P(outf), None if outh is None else P(outh), self._s()),
            "dem_mlp_gemm_tn")

    # ---- passes --------------------------------------------------------
    def _forward(self, bufs, x, idx=None):
        """x: FP32 (rows, n_in) device tensor, rows selected by idx when given."""
        P, B = self._ptr, bufs["B"]
        _ck(self.L.dem_mlp_pack_bf16(P(x), None if idx is None else P(idx), B, self.n_in, self.kp[0],
                                     P(bufs["h"][0]), self._s()), "dem_mlp_pack_bf16")
        last = len(self.W) - 1
        for l in range(len(self.W)):
            if l < last:
                self._gemm(bufs["h"][l], self.Wh[l], B, self.np_[l], self.kp[l], self.b[l], self.mode,
                           bufs["z"][l], bufs["h"][l + 1])
            else:
                self._gemm(bufs["h"][l], self.Wh[l], B, self.n_out, self.kp[l], self.b[l], BIAS, bufs["y"], None)
        return bufs["y"]

    def _backward(self, bufs, weights: bool = True, input_grad: bool = False):
        """Gradients of mean((y - t)^2) for the batch in bufs (targets in bufs['t'])."""
        P, L, s = self._ptr, self.L, self._s()
        B, Bp = bufs["B"], bufs["Bp"]
        nl = len(self.W)
        _ck(L.dem_mlp_mse_grad(P(bufs["y"]), P(bufs["t"]), B * self.n_out, P(bufs["dy16"]), P(bufs["dy"]),
                               P(self.loss_acc), s), "dem_mlp_mse_grad")
        _ck(L.dem_mlp_pack_bf16(P(bufs["dy"]), None, B, self.n_out, 32, P(bufs["dyp"]), s), "dem_mlp_pack_bf16")
        # current layer's output gradient: FP32 dfp (rows x width), BF16 d16 (rows x kwidth)
        dfp, d16, width, kwidth = bufs["dy"], bufs["dyp"], self.n_out, 32
        for l in range(nl - 1, -1, -1):
            K_in = self.kp[l]
            if weights:
                # dW_l = d^T h_l: both operands transposed so that the batch is the K dimension
                _ck(L.dem_mlp_transpose_bf16(P(d16), B, kwidth, Bp, P(bufs["aT"]), s), "transpose")
                _ck(L.dem_mlp_transpose_bf16(P(bufs["h"][l]), B, K_in, Bp, P(bufs["hT"]), s), "transpose")
                self._gemm(bufs["aT"], bufs["hT"], width, K_in, Bp, None, PLAIN, self.grads[l], None)
                _ck(L.dem_mlp_colsum(P(dfp), B, width, P(self.grads[nl + l]), P(self.scratch), s), "colsum")
            if l == 0 and not input_grad:
                break
            # dh_{l} = d W_l  (B operand: W_l^T, in_p x kwidth, padding columns zero)
            _ck(L.dem_mlp_transpose_bf16(P(self.Wh[l]), width, K_in, kwidth, P(bufs["wT"]), s), "transpose")
            out = bufs["dx"] if l == 0 else bufs["dh"]
            self._gemm(d16, bufs["wT"], B, K_in, kwidth, None, PLAIN, out, None)
            if l == 0:
                break
            n = B * K_in
            _ck(L.dem_mlp_act_backward(P(bufs["dh"]), P(bufs["z"][l - 1]), n, self.mode, P(bufs["dz16"]),
                                       P(bufs["dz"]), s), "dem_mlp_act_backward")
            dfp, d16, width, kwidth = bufs["dz"], bufs["dz16"], K_in, K_in

    def _adam(self):
        P, L, s = self._ptr, self.L, self._s()
        _ck(L.dem_mlp_tick(P(self.step), s), "dem_mlp_tick")
        nl = len(self.W)
        for i, (w, g, m, v) in enumerate(zip(self.params, self.grads, self.m, self.v)):
            wh = P(self.Wh[i]) if i < nl else None
            l2 = self.l2 if i < nl else 0.0      # sklearn penalises the weights, not the biases
            _ck(L.dem_mlp_adam(P(w), P(g), P(m), P(v), w.numel(), self.lr, self.b1, self.b2, self.eps, l2,
                               P(self.step), wh, s), "dem_mlp_adam")

    def train_step(self, x, t, idx):
        """One Adam step on the rows idx (device int32) of x / t (device FP32)."""
        bufs = self._buffers(int(idx.numel()))
        _ck(self.L.dem_mlp_gather(self._ptr(t), self._ptr(idx), bufs["B"], self.n_out, self._ptr(bufs["t"]),
                                  self._s()), "dem_mlp_gather")
        self._forward(bufs, x, idx)
        self._backward(bufs)
        self._adam()

    def check(self):
        flag = C.c_int(0)
        _ck(self.L.dem_mlp_status(C.byref(flag)), "dem_mlp_status")
        if flag.value:
            raise DemError(-3, "tensor-core commit timed out in dem_mlp_gemm_tn")

    # ---- public --------------------------------------------------------
    def fit(self, X: np.ndarray, Y: np.ndarray, epochs: int, batch: int = 256, seed: int = 0,
            graph: bool = True) -> list[float]:
        """Mini-batch Adam over (X, Y) (float arrays, rows = samples) for the
        given number of epochs, rows shuffled every epoch (seeded), the last
        partial batch dropped; after the first (eager) epoch, one CUDA graph
        replay per epoch.  Returns the mean training loss of each epoch."""
        ep = Epochs(self, X, Y, batch, seed)
        losses = [ep.run(graph) for _ in range(epochs)]
        ep.close()
        return losses

    def predict(self, X: np.ndarray, chunk: int = 65536) -> np.ndarray:
        torch = self.torch
        X = np.ascontiguousarray(X, np.float32)
        out = np.empty((X.shape[0], self.n_out), np.float32)
        for a in range(0, X.shape[0], chunk):
            xd = torch.from_numpy(X[a:a + chunk]).to(self.dev)
            bufs = self._buffers(xd.shape[0])
            self._forward(bufs, xd)
            out[a:a + chunk] = bufs["y"].cpu().numpy()
        self.check()
        return out

    def predict_device(self, xd):
        """Forward pass of a device FP32 (rows, n_in) tensor; returns the device output buffer."""
        bufs = self._buffers(int(xd.shape[0]))
        return self._forward(bufs, xd)

    def gradients(self, X: np.ndarray, T: np.ndarray, input_grad: bool = False):
        """(loss, dW, db, dX) of mean((y - t)^2) at the current weights (no update)."""
        torch = self.torch
        xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(self.dev)
        bufs = self._buffers(xd.shape[0])
        bufs["t"].copy_(torch.from_numpy(np.ascontiguousarray(T, np.float32)))
        self.loss_acc.zero_()
        self._forward(bufs, xd)
        self._backward(bufs, weights=True, input_grad=input_grad)
        torch.cuda.synchronize(self.dev)
        self.check()
        nl = len(self.W)
        dW = [self.grads[l].cpu().numpy() for l in range(nl)]
        db = [self.grads[nl + l].cpu().numpy() for l in range(nl)]
        dX = bufs["dx"][:, :self.n_in].cpu().numpy() if input_grad else None
        return float(self.loss_acc.item()), dW, db, dX

    def input_gradient(self, xd, target_rows):
        """dL/dx on the device for a device batch xd against device targets
        (rows x n_out); L = mean((y - t)^2).  Returns (y, dx) device views."""
        bufs = self._buffers(int(xd.shape[0]))
        bufs["t"].copy_(target_rows)
        self._forward(bufs, xd)
        self._backward(bufs, weights=False, input_grad=True)
        return bufs["y"], bufs["dx"][:, :self.n_in]

    def weights(self):
        """FP32 master weights and biases, cut to the unpadded sizes."""
        out_W, out_b = [], []
        for l in range(len(self.W)):
            fo, fi = self.sizes[l + 1], self.sizes[l]
            out_W.append(self.W[l][:fo, :fi].cpu().numpy())
            out_b.append(self.b[l][:fo].cpu().numpy())
        return out_W, out_b


class Epochs:
    """Training epochs of an MLP over a dataset held on the device: a seeded
    permutation per epoch, one Adam step per mini-batch; the first epoch runs
    eagerly (it also loads every kernel before a capture starts), the later ones
    replay one captured CUDA graph on a private stream."""

    def __init__(self, net: MLP, X: np.ndarray, Y: np.ndarray, batch: int = 256, seed: int = 0):
        torch = net.torch
        self.net, self.torch = net, torch
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.float32)
        self.n = X.shape[0]
        self.batch = min(batch, self.n)
        self.nb = self.n // self.batch
        self.stream = torch.cuda.Stream(net.dev)
        self.stream.wait_stream(torch.cuda.current_stream(net.dev))   # weights set up on the caller's stream
        with torch.cuda.stream(self.stream):
            self.x = torch.from_numpy(X).to(net.dev)
            self.y = torch.from_numpy(Y).to(net.dev)
            self.perm = torch.zeros(self.nb * self.batch, dtype=torch.int32, device=net.dev)
        self.rng = np.random.default_rng(seed)
        self.graph = None
        self.count = 0

    def _steps(self):
        for k in range(self.nb):
            self.net.train_step(self.x, self.y, self.perm[k * self.batch:(k + 1) * self.batch])

    def launch(self, graph: bool = True) -> None:
        """Enqueue one epoch on self.stream (no host synchronisation)."""
        torch = self.torch
        with torch.cuda.stream(self.stream):
            self.perm.copy_(torch.from_numpy(self.rng.permutation(self.n)[:self.nb * self.batch].astype(np.int32)))
            self.net.loss_acc.zero_()
            if not graph or self.count == 0:
                self._steps()
            else:
                if self.graph is None:
                    self.stream.synchronize()
                    self.graph = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(self.graph, stream=self.stream):
                        self._steps()
                self.graph.replay()
        self.count += 1

    def run(self, graph: bool = True) -> float:
        """One epoch; returns its mean training loss."""
        self.launch(graph)
        self.stream.synchronize()
        return float(self.net.loss_acc.item()) / self.nb

    def close(self) -> None:
        self.torch.cuda.synchronize(self.net.dev)
        self.graph = None
        self.net.check()


@dataclass
class Surrogate:
    """An MLP on standardised inputs and outputs.  lo / hi bound the parameter
    box (inputs are mapped to [-1, 1]); outputs are standardised by the mean and
    standard deviation of the training targets."""
    lo: np.ndarray
    hi: np.ndarray
    hidden: tuple = (256, 256, 256)
    activation: str = "gelu"
    seed: int = 0
    device: int = 0
    lr: float = 1e-3
    l2: float = 0.0
    net: MLP | None = None
    y_mean: np.ndarray | None = None
    y_std: np.ndarray | None = None
    history: list = field(default_factory=list)

    def _xn(self, X):
        return 2.0 * (np.asarray(X, np.float64) - self.lo) / (self.hi - self.lo) - 1.0

    def fit(self, X, Y, epochs: int = 200, batch: int = 256, refit: bool = False) -> list[float]:
        Y = np.asarray(Y, np.float64)
        if self.net is None or not refit:
            self.y_mean, self.y_std = Y.mean(axis=0), Y.std(axis=0) + 1e-12
            self.net = MLP((len(self.lo),) + tuple(self.hidden) + (Y.shape[1],), self.activation, self.seed,
                           self.device, self.lr, self.l2)
        losses = self.net.fit(self._xn(X), (Y - self.y_mean) / self.y_std, epochs, batch, seed=len(self.history))
        self.history.append(losses[-1])
        return losses

    def predict(self, X) -> np.ndarray:
        return self.net.predict(self._xn(X)) * self.y_std + self.y_mean

    def propose(self, target, k: int = 8, candidates: int = 16384, iters: int = 200, step: float = 0.02,
                weights=None, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """k parameter sets whose predicted properties are closest to target
        (weighted squared error of the standardised properties): the best k of
        a seeded Latin-hypercube set of candidates, each refined by projected
        gradient descent on the input (the network's own input gradient), all
        on the device.  Returns (params (k x d), predicted properties)."""
        torch = self.net.torch
        d = len(self.lo)
        rng = np.random.default_rng(seed)
        cand = (rng.permuted(np.tile(np.arange(candidates), (d, 1)), axis=1).T + rng.random((candidates, d)))
        cand = cand / candidates * 2.0 - 1.0
        tn = (np.asarray(target, np.float64) - self.y_mean) / self.y_std
        w = np.ones_like(tn) if weights is None else np.asarray(weights, np.float64)
        y = self.net.predict(cand)
        err = ((y - tn) ** 2 * w).sum(axis=1)
        best = cand[np.argsort(err)[:k]]
        xd = torch.from_numpy(best.astype(np.float32)).to(self.net.dev)
        tgt = torch.from_numpy(np.tile(tn.astype(np.float32), (k, 1))).to(self.net.dev)
        sw = torch.from_numpy(w.astype(np.float32)).to(self.net.dev)
        for _ in range(iters):
            if weights is None:
                _, dx = self.net.input_gradient(xd, tgt)
            else:
                # weighted error mean(w (y - t)^2): its output gradient is that of
                # mean((y - t')^2) with t' = y - w (y - t) held fixed
                yv = self.net.predict_device(xd).clone()
                _, dx = self.net.input_gradient(xd, yv - sw * (yv - tgt))
            g = dx / (dx.norm(dim=1, keepdim=True) + 1e-12)
            xd = (xd - step * g).clamp_(-1.0, 1.0)
        params = (xd.double().cpu().numpy() + 1.0) / 2.0 * (self.hi - self.lo) + self.lo
        return params, self.predict(params)


def macro_error(props: np.ndarray, target: np.ndarray, weights=None) -> np.ndarray:
    """Largest relative deviation of each row of props from target (weighted
    properties only)."""
    rel = np.abs(np.asarray(props, np.float64) / np.asarray(target, np.float64) - 1.0)
    if weights is not None:
        rel = rel[:, np.asarray(weights) > 0]
    return rel.max(axis=1)


# ---- the plain simulator as the judge, and the calibration loop ----------

PROPS = ("UCS", "E", "nu")


class UniaxialJudge:
    """Uniaxial tests of one packed cylinder (about n spheres) under many
    parameter sets (rows in the order of sweep.SWEEP_SPACE) in one batched
    context.  Every case draws its bond strengths with the same seed, so the
    macro properties are a deterministic function of the parameters.  Returns
    rows (UCS GPa, chord modulus GPa, Poisson ratio)."""

    def __init__(self, n: int = 2000, seed: int = 5, velocity_m_s: float = 0.1, max_steps: int = 400000,
                 device: int = 0):
        from . import sweep
        self.sweep, self.seed, self.device = sweep, seed, device
        self.velocity, self.max_steps = velocity_m_s, max_steps
        self.xyz, self.rad, _, self.box, self.size_real, self.center_real = sweep.cylinder(n, seed, device=device)
        self.keys = list(sweep.SWEEP_SPACE)
        self.calls = 0
        self.cases = 0

    def __call__(self, P: np.ndarray) -> np.ndarray:
        from . import TEST_UNIAXIAL, VELOCITY, Context, loading
        P = np.atleast_2d(np.asarray(P, np.float64))
        r_min, r_mean = float(self.rad.min()), float(self.rad.mean())
        ctx = Context(device=self.device)
        try:
            for row in P:
                p = dict(zip(self.keys, row))
                ld = loading(TEST_UNIAXIAL, self.box, self.size_real, self.center_real,
                             velocity=-self.velocity / VELOCITY, min_stress=0.010, max_strain=0.01,
                             cond_fracture=0.7, dNsave=100, max_steps=self.max_steps, p_r_platen=r_mean)
                ctx.add_sample(self.sweep.material_for(p, r_min, r_mean, self.seed * 7919 + 1), ld, self.xyz,
                               self.rad)
            ctx.setup()
            ctx.run(self.max_steps)
            res = [ctx.result(i) for i in range(len(P))]
        finally:
            ctx.close()
        self.calls += 1
        self.cases += len(P)
        return np.array([[r["FractureStress"], r["E_chord"], r["nu"]] for r in res])


@dataclass
class CalibrationRun:
    target: np.ndarray
    X: np.ndarray
    Y: np.ndarray
    best: np.ndarray          # parameters of the best simulated case
    best_props: np.ndarray    # its simulated properties
    best_error: float         # its largest relative deviation from the target
    accepted: bool            # best_error <= tol, confirmed by the simulator
    rounds: int
    simulations: int
    errors: list              # best error after the initial set and after each round


def latin_box(n: int, lo, hi, seed: int) -> np.ndarray:
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    rng = np.random.default_rng(seed)
    u = (np.stack([rng.permutation(n) for _ in lo], axis=1) + rng.random((n, lo.size))) / n
    return lo + u * (hi - lo)


def calibrate(judge, target, lo, hi, n_init: int = 64, rounds: int = 3, per_round: int = 16, tol: float = 0.01,
              epochs: int = 300, weights=None, seed: int = 0, X0=None, Y0=None, device: int = 0) -> CalibrationRun:
    """The reference's surrogate loop (NN_MP.py:766-930) with the simulator as
    the judge: simulate a Latin-hypercube start set (or take X0, Y0), then per
    round fit the surrogate to everything simulated so far, propose per_round
    parameter sets whose predicted properties are closest to target, simulate
    them, and stop when a simulated case is within tol (largest relative
    deviation over the weighted properties).  Only simulated properties decide
    acceptance; the surrogate only chooses what to simulate."""
    target = np.asarray(target, np.float64)
    if X0 is None:
        X = latin_box(n_init, lo, hi, seed)
        Y = judge(X)
    else:
        X, Y = np.asarray(X0, np.float64), np.asarray(Y0, np.float64)
    sims = len(X)
    err = macro_error(Y, target, weights)
    errors = [float(err.min())]
    sur = Surrogate(np.asarray(lo, np.float64), np.asarray(hi, np.float64), seed=seed, device=device)
    r = 0
    while r < rounds and errors[-1] > tol:
        r += 1
        ok = np.all(np.isfinite(Y), axis=1)
        sur.fit(X[ok], Y[ok], epochs=epochs, batch=min(256, int(ok.sum())))
        P, _ = sur.propose(target, k=per_round, weights=weights, seed=seed + r)
        Yp = judge(P)
        sims += len(P)
        X, Y = np.vstack([X, P]), np.vstack([Y, Yp])
        err = macro_error(Y, target, weights)
        errors.append(float(err.min()))
    i = int(np.argmin(err))
    return CalibrationRun(target, X, Y, X[i], Y[i], float(err[i]), bool(err[i] <= tol), r, sims, errors)


def random_search(judge, target, lo, hi, budget: int, weights=None, seed: int = 0, X0=None, Y0=None,
                  batch: int = 16) -> CalibrationRun:
    """The method without the network at the same simulator budget: further
    Latin-hypercube points after the start set, the best simulated case kept."""
    target = np.asarray(target, np.float64)
    X, Y = np.asarray(X0, np.float64), np.asarray(Y0, np.float64)
    errors = [float(macro_error(Y, target, weights).min())]
    extra = latin_box(budget - len(X), lo, hi, seed + 1000) if budget > len(X) else np.empty((0, len(lo)))
    for a in range(0, len(extra), batch):
        P = extra[a:a + batch]
        X, Y = np.vstack([X, P]), np.vstack([Y, judge(P)])
        errors.append(float(macro_error(Y, target, weights).min()))
    err = macro_error(Y, target, weights)
    i = int(np.argmin(err))
    return CalibrationRun(target, X, Y, X[i], Y[i], float(err[i]), False, len(errors) - 1, len(X), errors)
