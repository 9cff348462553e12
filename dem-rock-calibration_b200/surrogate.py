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
calibrate      the loop of the reference workflow with the batched simulator
               deciding: fit, propose, simulate the proposals, accept a
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
# one entry of the device list that dem_mlp_adam_multi reads (dem_mlp_tensor:
# weights, gradient, moments, BF16 copy, element count, L2 penalty, padding)
ADAM_TENSOR_DTYPE = np.dtype([("w", "<u8"), ("g", "<u8"), ("m", "<u8"), ("v", "<u8"), ("w_bf16", "<u8"),
                              ("n", "<u8"), ("l2", "<f4"), ("pad", "<f4")])


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
    """Dense network sizes[0] -> ... -> sizes[-1], hidden activation GELU (tanh
    form) or ReLU, identity output, loss mean((y - t)^2).

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
        # device descriptor list of every weight and bias array for the one-launch
        # Adam step (dem_mlp_tensor: w, g, m, v, w_bf16, n, l2, pad)
        nl = len(self.W)
        rec = np.zeros(len(self.params), dtype=ADAM_TENSOR_DTYPE)
        for i, (w, g, m, v) in enumerate(zip(self.params, self.grads, self.m, self.v)):
            rec[i] = (w.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(),
                      self.Wh[i].data_ptr() if i < nl else 0, w.numel(),
                      self.l2 if i < nl else 0.0, 0.0)      # sklearn penalises the weights, not the biases
        self.adam_list = torch.from_numpy(rec.view(np.uint8).copy()).to(self.dev)
        self.adam_max_n = int(max(p.numel() for p in self.params))
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
    def _forward(self, bufs, x, idx=None, keep_z: bool = True):
        """x: FP32 (rows, n_in) device tensor, rows selected by idx when given;
        keep_z stores the hidden pre-activations (needed by a backward pass)."""
        P, B = self._ptr, bufs["B"]
        _ck(self.L.dem_mlp_pack_bf16(P(x), None if idx is None else P(idx), B, self.n_in, self.kp[0],
                                     P(bufs["h"][0]), self._s()), "dem_mlp_pack_bf16")
        last = len(self.W) - 1
        for l in range(len(self.W)):
            if l < last:
                self._gemm(bufs["h"][l], self.Wh[l], B, self.np_[l], self.kp[l], self.b[l], self.mode,
                           bufs["z"][l] if keep_z else None, bufs["h"][l + 1])
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
        _ck(L.dem_mlp_adam_multi(P(self.adam_list), len(self.params), self.adam_max_n, self.lr, self.b1, self.b2,
                                 self.eps, P(self.step), s), "dem_mlp_adam_multi")

    def launches_per_step(self, batch: int = 256) -> int:
        """Kernel launches of one train_step: gather + input pack + one GEMM per
        layer; MSE gradient + pack, per layer two transposes, the weight-gradient
        GEMM and the column sums (one pass up to 2048 rows, else two), per layer
        but the first a transpose, the input-gradient GEMM and the activation
        backward; the step tick and one Adam launch for all arrays."""
        nl = len(self.W)
        cs = 1 if batch <= 2048 else 2
        return (2 + nl) + (2 + (4 + cs) * nl + 3 * (nl - 1)) + 2

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
        batch smaller when batch does not divide the rows; after the first
        (eager) epoch, one CUDA graph replay per epoch.  Returns the mean
        training loss of each epoch (the mean of its batch losses)."""
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
            self._forward(bufs, xd, keep_z=False)
            out[a:a + chunk] = bufs["y"].cpu().numpy()
        self.check()
        return out

    def predict_device(self, xd):
        """Forward pass of a device FP32 (rows, n_in) tensor; returns the device output buffer."""
        bufs = self._buffers(int(xd.shape[0]))
        return self._forward(bufs, xd, keep_z=False)

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
    permutation per epoch, one Adam step per mini-batch (the last one smaller
    when batch does not divide the rows); the first epoch runs
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
        # the last, smaller batch is trained too (as sklearn's gen_batches yields it)
        self.sizes = [self.batch] * self.nb + ([self.n - self.nb * self.batch] if self.n % self.batch else [])
        self.stream = torch.cuda.Stream(net.dev)
        self.stream.wait_stream(torch.cuda.current_stream(net.dev))   # weights set up on the caller's stream
        with torch.cuda.stream(self.stream):
            self.x = torch.from_numpy(X).to(net.dev)
            self.y = torch.from_numpy(Y).to(net.dev)
            self.perm = torch.zeros(self.n, dtype=torch.int32, device=net.dev)
        self.rng = np.random.default_rng(seed)
        self.graph = None
        self.count = 0

    def _steps(self):
        a = 0
        for b in self.sizes:
            self.net.train_step(self.x, self.y, self.perm[a:a + b])
            a += b

    def launch(self, graph: bool = True) -> None:
        """Enqueue one epoch on self.stream (no host synchronisation)."""
        torch = self.torch
        with torch.cuda.stream(self.stream):
            self.perm.copy_(torch.from_numpy(self.rng.permutation(self.n).astype(np.int32)))
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
        return float(self.net.loss_acc.item()) / len(self.sizes)

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


# ---- the plain simulator that decides, and the calibration loop ----------

PROPS = ("UCS", "E", "nu")


class UniaxialSolver:
    """Uniaxial tests of one packed cylinder (about n spheres) under many
    parameter sets (rows in the order of sweep.SWEEP_SPACE) in one batched
    context.  Every case draws its bond strengths with the same seed, and the
    context runs in deterministic mode (exact fixed-point force sums), so the
    macro properties are a reproducible function of the parameters alone - the
    same in a batch as in a plain one-sample run.  Returns rows (UCS GPa, chord
    modulus GPa, Poisson ratio)."""

    def __init__(self, n: int = 2000, seed: int = 5, velocity_m_s: float = 0.1, max_steps: int = 400000,
                 device: int = 0, deterministic: bool = True):
        from . import sweep
        self.sweep, self.seed, self.device = sweep, seed, device
        self.deterministic = deterministic
        self.velocity, self.max_steps = velocity_m_s, max_steps
        self.xyz, self.rad, _, self.box, self.size_real, self.center_real = sweep.cylinder(n, seed, device=device)
        self.keys = list(sweep.SWEEP_SPACE)
        self.calls = 0
        self.cases = 0

    def __call__(self, P: np.ndarray) -> np.ndarray:
        from . import TEST_UNIAXIAL, VELOCITY, Context, loading
        P = np.atleast_2d(np.asarray(P, np.float64))
        r_min, r_mean = float(self.rad.min()), float(self.rad.mean())
        ctx = Context(device=self.device, deterministic=self.deterministic)
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


class BrazilSolver:
    """Brazilian tests of one packed disc (about n spheres, thickness half the
    diameter, axis z, platens across the diameter) under many parameter sets,
    in one batched context, deterministic mode; returns the tensile strength
    (GPa) per row (the reference's sigma_B = F / (pi R t), md_data_types.h:395)."""

    def __init__(self, n: int = 2000, seed: int = 6, velocity_m_s: float = 0.1, max_steps: int = 400000,
                 device: int = 0, deterministic: bool = True):
        from . import sweep
        self.sweep, self.seed, self.device = sweep, seed, device
        self.deterministic = deterministic
        self.velocity, self.max_steps = velocity_m_s, max_steps
        self.xyz, self.rad, _, self.box, self.size_real, self.center_real = sweep.cylinder(n, seed, aspect=0.5,
                                                                                           device=device)
        self.keys = list(sweep.SWEEP_SPACE)

    def __call__(self, P: np.ndarray) -> np.ndarray:
        from . import TEST_BRAZIL, VELOCITY, Context, loading
        P = np.atleast_2d(np.asarray(P, np.float64))
        r_min, r_mean = float(self.rad.min()), float(self.rad.mean())
        ctx = Context(device=self.device, deterministic=self.deterministic)
        try:
            for row in P:
                p = dict(zip(self.keys, row))
                ld = loading(TEST_BRAZIL, self.box, self.size_real, self.center_real,
                             velocity=-self.velocity / VELOCITY, min_stress=0.0021, max_strain=0.03,
                             cond_fracture=0.1, dNsave=1000, max_steps=self.max_steps, p_r_platen=r_mean)
                ctx.add_sample(self.sweep.material_for(p, r_min, r_mean, self.seed * 7919 + 1), ld, self.xyz,
                               self.rad)
            ctx.setup()
            ctx.run(self.max_steps)
            out = np.array([ctx.result(i)["FractureStress"] for i in range(len(P))])
        finally:
            ctx.close()
        return out


def simulate_dataset(n: int, seed: int = 0, uni: "UniaxialSolver | None" = None, braz: "BrazilSolver | None" = None,
                     batch: int = 256, space=None):
    """n Latin-hypercube parameter sets of the sweep box and their simulated
    macro properties: columns (UCS, E, nu) from uniaxial tests, plus the
    tensile strength from Brazilian tests when braz is given; batch cases per
    context.  Returns (X (n x 6), Y (n x 3 or 4), seconds)."""
    import time

    from . import sweep
    space = space or sweep.SWEEP_SPACE
    lo = np.array([v[0] for v in space.values()])
    hi = np.array([v[1] for v in space.values()])
    X = latin_box(n, lo, hi, seed)
    uni = uni or UniaxialSolver()
    t0 = time.perf_counter()
    cols = [np.vstack([uni(X[a:a + batch]) for a in range(0, n, batch)])]
    if braz is not None:
        cols.append(np.concatenate([braz(X[a:a + batch]) for a in range(0, n, batch)])[:, None])
    return X, np.hstack(cols), time.perf_counter() - t0


@dataclass
class CalibrationRun:
    target: np.ndarray
    tol: np.ndarray           # per-property relative tolerance
    X: np.ndarray
    Y: np.ndarray
    best: np.ndarray          # parameters of the best simulated case
    best_props: np.ndarray    # its simulated properties
    best_score: float         # its largest deviation in units of the tolerance (<= 1: within tol)
    accepted: bool            # best_score <= 1 in the batched run and in its plain re-run
    confirmed_props: np.ndarray | None   # the plain re-run of the accepted case
    rounds: int
    simulations: int
    scores: list              # best score after the start set and after each round


def latin_box(n: int, lo, hi, seed: int) -> np.ndarray:
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    rng = np.random.default_rng(seed)
    u = (np.stack([rng.permutation(n) for _ in lo], axis=1) + rng.random((n, lo.size))) / n
    return lo + u * (hi - lo)


def score(props, target, tol) -> np.ndarray:
    """Per row: the largest relative deviation from target in units of the
    per-property tolerance (a property with tolerance inf is not compared)."""
    rel = np.abs(np.atleast_2d(np.asarray(props, np.float64)) / np.asarray(target, np.float64) - 1.0)
    out = (rel / np.broadcast_to(np.asarray(tol, np.float64), rel.shape[1:])).max(axis=1)
    return np.where(np.isfinite(out), out, np.inf)


def calibrate(solve, target, lo, hi, n_init: int = 64, rounds: int = 3, per_round: int = 16, tol=0.01,
              epochs: int = 300, seed: int = 0, X0=None, Y0=None, device: int = 0) -> CalibrationRun:
    """The reference's surrogate loop (NN_MP.py:766-930) with the simulator as
    the arbiter: simulate a Latin-hypercube start set (or take X0, Y0), then per
    round fit the surrogate to everything simulated so far, propose per_round
    parameter sets whose predicted properties are closest to target (errors
    weighted by 1 / tol^2), simulate them in one batched context, and stop
    once a simulated case is within tol on every property AND a plain re-run
    of that case (one sample per context: the plain method) is within tol as
    well.  Simulated properties alone decide acceptance; the surrogate only
    chooses what to simulate.  A case whose re-run misses tol stays in the data
    but cannot be accepted."""
    target = np.asarray(target, np.float64)
    tol = np.broadcast_to(np.asarray(tol, np.float64), target.shape).copy()
    if X0 is None:
        X = latin_box(n_init, lo, hi, seed)
        Y = solve(X)
    else:
        X, Y = np.asarray(X0, np.float64), np.asarray(Y0, np.float64)
    sims = len(X)
    rejected = np.zeros(len(X), bool)
    sur = Surrogate(np.asarray(lo, np.float64), np.asarray(hi, np.float64), seed=seed, device=device)
    w = 1.0 / np.where(np.isfinite(tol), tol, np.inf) ** 2
    w = w / w.max()
    accepted, confirmed, r = False, None, 0
    sc = score(Y, target, tol)
    scores = [float(sc.min())]

    def confirm():
        nonlocal sims, confirmed, accepted
        while True:
            cand = np.where(rejected, np.inf, score(Y, target, tol))
            i = int(np.argmin(cand))
            if cand[i] > 1.0:
                return
            again = solve(X[i:i + 1])[0]
            sims += 1
            if score(again, target, tol)[0] <= 1.0:
                accepted, confirmed = True, again
                return
            rejected[i] = True

    confirm()
    while r < rounds and not accepted:
        r += 1
        ok = np.all(np.isfinite(Y), axis=1)
        sur.fit(X[ok], Y[ok], epochs=epochs, batch=min(256, int(ok.sum())))
        P, _ = sur.propose(target, k=per_round, weights=w, seed=seed + r)
        Yp = solve(P)
        sims += len(P)
        X, Y = np.vstack([X, P]), np.vstack([Y, Yp])
        rejected = np.concatenate([rejected, np.zeros(len(P), bool)])
        scores.append(float(score(Y, target, tol).min()))
        confirm()
    sc = np.where(rejected, np.inf, score(Y, target, tol))
    i = int(np.argmin(sc))
    return CalibrationRun(target, tol, X, Y, X[i], Y[i], float(sc[i]), accepted, confirmed, r, sims, scores)


def random_search(solve, target, lo, hi, budget: int, tol=0.01, seed: int = 0, X0=None, Y0=None,
                  batch: int = 16) -> CalibrationRun:
    """The method without the network at the same simulator budget: further
    Latin-hypercube points after the start set, the best simulated case kept
    (scored as in calibrate; not re-run)."""
    target = np.asarray(target, np.float64)
    tol = np.broadcast_to(np.asarray(tol, np.float64), target.shape).copy()
    X, Y = np.asarray(X0, np.float64), np.asarray(Y0, np.float64)
    scores = [float(score(Y, target, tol).min())]
    extra = latin_box(budget - len(X), lo, hi, seed + 1000) if budget > len(X) else np.empty((0, len(lo)))
    for a in range(0, len(extra), batch):
        P = extra[a:a + batch]
        X, Y = np.vstack([X, P]), np.vstack([Y, solve(P)])
        scores.append(float(score(Y, target, tol).min()))
    sc = score(Y, target, tol)
    i = int(np.argmin(sc))
    return CalibrationRun(target, tol, X, Y, X[i], Y[i], float(sc[i]), False, None, len(scores) - 1, len(X),
                          scores)


class MLPRegressorB200:
    """sklearn.neural_network.MLPRegressor's interface (the surrogate of
    NN_MP.py:374-378: fit(X, y) at :895, predict at :395) over the tensor-core
    MLP, so that the workflow swaps one constructor:

        mlp = MLPRegressorB200(hidden_layer_sizes=[300, 500, 900, 500, 300], max_iter=20000, tol=0)

    Same meaning as sklearn for hidden_layer_sizes, activation ('relu' or
    'gelu'; sklearn's default 'relu'), alpha (L2 penalty, weights only, its
    gradient alpha W / batch against the data gradient of sum((y - t)^2) / (2
    batch)), batch_size ('auto' = min(200, n)), learning_rate_init, max_iter
    (epochs), tol and n_iter_no_change (stop when the epoch loss has not
    improved by tol for n_iter_no_change epochs), beta_1, beta_2, epsilon,
    shuffle (always on), random_state.  Inputs are used as given (sklearn
    does not scale them either); a 1-D y gives 1-D predictions.  The numerics
    differ from sklearn's float64 CPU path by BF16 operands (FP32
    accumulation and master weights)."""

    def __init__(self, hidden_layer_sizes=(100,), activation="relu", alpha=1e-4, batch_size="auto",
                 learning_rate_init=1e-3, max_iter=200, tol=1e-4, n_iter_no_change=10, beta_1=0.9, beta_2=0.999,
                 epsilon=1e-8, random_state=None, device=0):
        self.hidden_layer_sizes = tuple(hidden_layer_sizes)
        self.activation, self.alpha, self.batch_size = activation, alpha, batch_size
        self.learning_rate_init, self.max_iter, self.tol = learning_rate_init, max_iter, tol
        self.n_iter_no_change, self.beta_1, self.beta_2, self.epsilon = n_iter_no_change, beta_1, beta_2, epsilon
        self.random_state, self.device = random_state, device
        self.net = None
        self.loss_curve_ = []
        self.n_iter_ = 0

    def fit(self, X, y):
        X = np.asarray(X, np.float32)
        y = np.asarray(y, np.float32)
        self._1d = y.ndim == 1
        Y = y.reshape(len(y), -1)
        n = len(X)
        batch = min(200, n) if self.batch_size == "auto" else min(int(self.batch_size), n)
        seed = 0 if self.random_state is None else int(self.random_state)
        n_out = Y.shape[1]
        # device loss mean((y - t)^2) has gradient (2 / n_out) x sklearn's data term
        l2 = self.alpha / batch * 2.0 / n_out
        self.net = MLP((X.shape[1],) + self.hidden_layer_sizes + (n_out,), self.activation, seed, self.device,
                       self.learning_rate_init, l2, (self.beta_1, self.beta_2), self.epsilon)
        ep = Epochs(self.net, X, Y, batch, seed)
        best, stall = np.inf, 0
        self.loss_curve_ = []
        for it in range(self.max_iter):
            loss = 0.5 * n_out * ep.run()          # sklearn's loss scale, sum((y - t)^2) / (2 n)
            self.loss_curve_.append(loss)
            self.n_iter_ = it + 1
            if loss > best - self.tol:
                stall += 1
            else:
                stall = 0
            best = min(best, loss)
            if stall > self.n_iter_no_change:
                break
        ep.close()
        return self

    def predict(self, X):
        out = self.net.predict(np.asarray(X, np.float32))
        return out[:, 0] if self._1d else out
