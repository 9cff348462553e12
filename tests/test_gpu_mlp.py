"""Surrogate MLP kernels on the GPU (dem_mlp_*), against torch FP32 on the same
BF16 operands and against the CPU oracle (oracle/mlp.py).

Tolerances:
  GEMM (FP32 accumulation of BF16 products, summation order free):
      |C - C_ref| <= 1e-5 * (|A| |B|^T) + 1e-6 elementwise
  BF16 activations: within one BF16 rounding of the FP32 reference
      (relative 2^-8 of the value) plus the hardware tanh's error in GELU
      (relative 1e-3 of the value, plus 1e-6)
  network gradients against the oracle's BF16 path: relative Frobenius error
      <= 2e-2 per layer (hidden activations rounded to BF16 on both sides may
      differ by one BF16 unit where the FP32 sums differ in their last bits)
  training: eager and graph-replayed epochs give bit-identical weights (every
      kernel on the weight path sums in a fixed order)
"""
from __future__ import annotations

import ctypes as C
import importlib

import numpy as np
import pytest

from dem_api import dem
from oracle import mlp as O

S = importlib.import_module("dem-rock-calibration_b200.surrogate")
pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _p(t):
    return C.c_void_p(t.data_ptr())


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _status_ok():
    f = C.c_int(0)
    assert dem.lib().dem_mlp_status(C.byref(f)) == 0
    assert f.value == 0


# the last four shapes take the persistent kernel (at least two 128-row tiles
# per SM, N <= 256, K <= 256): ragged rows, narrow and ragged columns, K = 32
@pytest.mark.parametrize("M,N,K", [(128, 32, 32), (300, 256, 64), (1000, 4, 256), (256, 320, 96), (77, 64, 512),
                                   (4096, 128, 256), (65536, 256, 256), (40000, 100, 128), (38000, 4, 256),
                                   (50000, 64, 32)])
@pytest.mark.parametrize("mode", [S.PLAIN, S.BIAS, S.BIAS_GELU, S.BIAS_RELU])
def test_gemm_tn_against_torch_fp32(M, N, K, mode):
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K + mode)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    outf = torch.full((M, N), float("nan"), device="cuda")
    outh = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    act = mode in (S.BIAS_GELU, S.BIAS_RELU)
    rc = dem.lib().dem_mlp_gemm_tn(_p(A), _p(B), M, N, K, _p(bias) if mode != S.PLAIN else None, mode, _p(outf),
                                   _p(outh) if act else None, _s())
    assert rc == 0
    torch.cuda.synchronize()
    _status_ok()
    ref = A.float() @ B.float().T
    bound = 1e-5 * (A.float().abs() @ B.float().abs().T) + 1e-6
    if mode != S.PLAIN:
        ref = ref + bias
    assert torch.all((outf - ref).abs() <= bound), float((outf - ref).abs().max())
    if act:
        if mode == S.BIAS_GELU:
            fn = lambda x: torch.nn.functional.gelu(x, approximate="tanh")
        else:
            fn = torch.relu
        want = fn(ref)
        assert torch.all((outh.float() - want).abs() <= want.abs() * (2.0 ** -8 + 1e-3) + 1e-6 + fn(ref + bound).sub(
            fn(ref - bound)).abs())


def test_small_kernels():
    L = dem.lib()
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(300, 6, device="cuda", generator=g)
    idx = torch.randperm(300, device="cuda", generator=g)[:200].to(torch.int32)
    h = torch.zeros(200, 32, dtype=torch.bfloat16, device="cuda")
    assert L.dem_mlp_pack_bf16(_p(x), _p(idx), 200, 6, 32, _p(h), _s()) == 0
    want = torch.zeros(200, 32, device="cuda")
    want[:, :6] = x[idx.long()]
    assert torch.equal(h, want.to(torch.bfloat16))
    xg = torch.zeros(200, 6, device="cuda")
    assert L.dem_mlp_gather(_p(x), _p(idx), 200, 6, _p(xg), _s()) == 0
    assert torch.equal(xg, x[idx.long()])
    # transpose with zero padding of the columns beyond the rows
    a = torch.randn(200, 70, device="cuda", generator=g).to(torch.bfloat16)
    at = torch.full((70, 224), 7.0, device="cuda").to(torch.bfloat16)
    assert L.dem_mlp_transpose_bf16(_p(a), 200, 70, 224, _p(at), _s()) == 0
    assert torch.equal(at[:, :200], a.T) and torch.all(at[:, 200:] == 0)
    # column sums (fixed order) against a float64 sum
    m = torch.randn(5000, 300, device="cuda", generator=g)
    cs = torch.zeros(300, device="cuda")
    scratch = torch.zeros(S.COLSUM_SPLIT * 300, device="cuda")
    assert L.dem_mlp_colsum(_p(m), 5000, 300, _p(cs), _p(scratch), _s()) == 0
    ref = m.double().sum(0)
    assert torch.all((cs.double() - ref).abs() <= 1e-5 * m.double().abs().sum(0))
    # activation backward
    z = torch.randn(4000, device="cuda", generator=g) * 3
    dh = torch.randn(4000, device="cuda", generator=g)
    for act in (S.BIAS_GELU, S.BIAS_RELU):
        dz16 = torch.zeros(4000, dtype=torch.bfloat16, device="cuda")
        dz = torch.zeros(4000, device="cuda")
        assert L.dem_mlp_act_backward(_p(dh), _p(z), 4000, act, _p(dz16), _p(dz), _s()) == 0
        d = torch.from_numpy(O.act_grad(z.double().cpu().numpy(), "gelu" if act == S.BIAS_GELU else "relu"))
        ref = dh.double() * d.cuda()
        # hardware tanh (relative error ~2^-11) inside the GELU derivative
        tol = 1e-3 * dh.double().abs() * (1 + z.double().abs()) if act == S.BIAS_GELU else 1e-7 * ref.abs()
        assert torch.all((dz.double() - ref).abs() <= tol + 1e-6)
        assert torch.equal(dz16, dz.to(torch.bfloat16))
    # MSE gradient and loss
    y = torch.randn(1000, 4, device="cuda", generator=g)
    t = torch.randn(1000, 4, device="cuda", generator=g)
    dy16 = torch.zeros(1000, 4, dtype=torch.bfloat16, device="cuda")
    dy = torch.zeros(1000, 4, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.dem_mlp_mse_grad(_p(y), _p(t), 4000, _p(dy16), _p(dy), _p(loss), _s()) == 0
    assert torch.allclose(dy, 2 * (y - t) / 4000, rtol=1e-6, atol=0)
    assert float(loss) == pytest.approx(float(((y - t).double() ** 2).mean()), rel=1e-9)   # FP32 difference, FP64 squares
    # Adam with the device step counter, against the oracle
    w = torch.randn(500, device="cuda", generator=g)
    gr = torch.randn(500, device="cuda", generator=g)
    mo, ve = torch.zeros(500, device="cuda"), torch.zeros(500, device="cuda")
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    wh = torch.zeros(500, dtype=torch.bfloat16, device="cuda")
    wn, mn, vn = w.double().cpu().numpy(), np.zeros(500), np.zeros(500)
    for it in range(1, 4):
        assert L.dem_mlp_tick(_p(step), _s()) == 0
        assert L.dem_mlp_adam(_p(w), _p(gr), _p(mo), _p(ve), 500, 1e-2, 0.9, 0.999, 1e-8, 1e-3, _p(step), _p(wh),
                              _s()) == 0
        wn, mn, vn = O.adam(wn, gr.double().cpu().numpy(), mn, vn, it, lr=1e-2, l2=1e-3)
    torch.cuda.synchronize()
    assert int(step) == 3
    assert np.allclose(w.cpu().numpy(), wn, rtol=1e-5, atol=1e-6)
    assert torch.equal(wh, w.to(torch.bfloat16))
    # the one-launch Adam over a descriptor list equals the per-array launches
    arrs = []
    for n_, l2 in ((700, 1e-3), (33, 0.0)):
        w0 = torch.randn(n_, device="cuda", generator=g)
        g0 = torch.randn(n_, device="cuda", generator=g)
        arrs.append([(w0.clone(), g0, torch.zeros(n_, device="cuda"), torch.zeros(n_, device="cuda"),
                      torch.zeros(n_, dtype=torch.bfloat16, device="cuda"), l2) for _ in range(2)])
    st1 = torch.zeros(1, dtype=torch.int32, device="cuda")
    st2 = torch.zeros(1, dtype=torch.int32, device="cuda")
    rec = np.zeros(2, dtype=[("w", "<u8"), ("g", "<u8"), ("m", "<u8"), ("v", "<u8"), ("wh", "<u8"), ("n", "<u8"),
                             ("l2", "<f4"), ("pad", "<f4")])
    for k, pair in enumerate(arrs):
        w_, g_, m_, v_, h_, l2 = pair[1]
        rec[k] = (w_.data_ptr(), g_.data_ptr(), m_.data_ptr(), v_.data_ptr(), h_.data_ptr(), w_.numel(), l2, 0.0)
    lst = torch.from_numpy(rec.view(np.uint8).copy()).cuda()
    for it in range(3):
        assert L.dem_mlp_tick(_p(st1), _s()) == 0 and L.dem_mlp_tick(_p(st2), _s()) == 0
        for pair in arrs:
            w_, g_, m_, v_, h_, l2 = pair[0]
            assert L.dem_mlp_adam(_p(w_), _p(g_), _p(m_), _p(v_), w_.numel(), 1e-2, 0.9, 0.999, 1e-8, l2, _p(st1),
                                  _p(h_), _s()) == 0
        assert L.dem_mlp_adam_multi(_p(lst), 2, 700, 1e-2, 0.9, 0.999, 1e-8, _p(st2), _s()) == 0
    torch.cuda.synchronize()
    for pair in arrs:
        for a, b in zip(pair[0][:5], pair[1][:5]):
            assert torch.equal(a, b)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))


@pytest.mark.parametrize("activation", ["gelu", "relu"])
def test_network_gradients_against_the_oracle(activation):
    net = S.MLP((6, 64, 96, 4), activation=activation, seed=3)
    rng = np.random.default_rng(7)
    X = rng.uniform(-1, 1, (200, 6)).astype(np.float32)
    T = rng.normal(size=(200, 4)).astype(np.float32)
    loss, dW, db, dX = net.gradients(X, T, input_grad=True)
    W, b = net.weights()
    Wb = [O.bf16(w) for w in W]                     # the device multiplies the BF16 copies
    l_ref, dW_ref, db_ref, dX_ref = O.backward(Wb, b, X, T, activation, rnd=True, input_grad=True)
    l64, dW64, db64, _ = O.backward(W, b, X, T, activation, rnd=False)
    assert loss == pytest.approx(l_ref, rel=1e-4)
    assert loss == pytest.approx(l64, rel=2e-2)
    for l in range(len(W)):
        fo, fi = W[l].shape
        assert _rel(dW[l][:fo, :fi], dW_ref[l]) <= 2e-2, (l, _rel(dW[l][:fo, :fi], dW_ref[l]))
        assert _rel(db[l][:fo], db_ref[l]) <= 2e-2
        assert _rel(dW[l][:fo, :fi], dW64[l]) <= 5e-2
        # padding rows and columns get exactly zero gradient
        assert not np.any(dW[l][fo:, :]) and not np.any(dW[l][:, fi:]) and not np.any(db[l][fo:])
    assert _rel(dX, dX_ref) <= 2e-2


def test_training_fits_a_smooth_map_and_graph_replay_is_bit_identical():
    rng = np.random.default_rng(11)
    X = rng.uniform(-1, 1, (8192, 6)).astype(np.float32)
    Y = np.stack([np.sin(2 * X[:, 0]) + X[:, 1] ** 2, X[:, 2] * X[:, 3], np.exp(0.5 * X[:, 4]) - X[:, 5],
                  X[:, 0] * X[:, 5] + 0.3 * X[:, 2]], axis=1).astype(np.float32)
    a = S.MLP((6, 256, 256, 256, 4), seed=1)
    b = S.MLP((6, 256, 256, 256, 4), seed=1)
    la = a.fit(X, Y, epochs=4, batch=256, graph=False)
    lb = b.fit(X, Y, epochs=4, batch=256, graph=True)
    for wa, wb in zip(a.params, b.params):
        assert torch.equal(wa, wb)
    assert la == pytest.approx(lb, rel=1e-9)
    lc = b.fit(X, Y, epochs=40, batch=256, seed=1)
    assert lc[-1] < 0.02 * la[0], (la[0], lc[-1])
    Xt = rng.uniform(-1, 1, (4096, 6)).astype(np.float32)
    Yt = np.stack([np.sin(2 * Xt[:, 0]) + Xt[:, 1] ** 2, Xt[:, 2] * Xt[:, 3], np.exp(0.5 * Xt[:, 4]) - Xt[:, 5],
                   Xt[:, 0] * Xt[:, 5] + 0.3 * Xt[:, 2]], axis=1)
    P = b.predict(Xt)
    assert float(np.mean((P - Yt) ** 2)) < 0.02 * float(np.mean((Yt - Yt.mean(0)) ** 2)) + 1e-3
    # the network's predictions follow the oracle forward pass on its own BF16 weights
    W, bb = b.weights()
    y_ref, _, _ = O.forward([O.bf16(w) for w in W], bb, Xt[:512], "gelu", rnd=True)
    assert _rel(P[:512], y_ref) <= 1e-2
