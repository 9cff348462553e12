"""CPU checks of the surrogate MLP's oracle (oracle/mlp.py) and of the
dem_mlp_* argument checks.

The oracle's float64 path is pinned to scikit-learn's MLPRegressor (the
reference's surrogate, NN_MP.py:374-378): the same weights give the same
predictions, and the same backprop gradients up to the loss scaling
(sklearn differentiates sum((y - t)^2) / (2 n_samples), the oracle
mean((y - t)^2) over all n_samples * n_out entries, a factor 2 / n_out).
The GELU path, which sklearn does not have, is checked against central
differences.  The bf16 rounding helper is checked on exactly representable
cases.
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np
import pytest

from dem_api import dem
from oracle import mlp as O


def _net(sizes, seed):
    rng = np.random.default_rng(seed)
    W = [rng.normal(0, 1 / np.sqrt(a), (b, a)) for a, b in zip(sizes[:-1], sizes[1:])]
    b = [rng.normal(0, 0.1, n) for n in sizes[1:]]
    return W, b


def test_bf16_rounding_ties_to_even():
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -7)                 # bf16 spacing at 1.0
    # halfway cases go to the even neighbour: 1 + ulp/2 -> 1, 1 + 3 ulp/2 -> 1 + 2 ulp
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5], np.float32)
    want = np.array([1.0, 1.0, 1.0 + 2 * ulp, 1.0, -2.5], np.float32)
    assert np.array_equal(O.bf16(x), want)
    assert O.bf16(one + ulp) == one + ulp
    r = np.random.default_rng(0).normal(size=1000).astype(np.float32)
    assert np.all(np.abs(O.bf16(r) - r) <= np.abs(r) * 2.0 ** -8)     # half a bf16 ulp (8 significant bits)
    assert np.all(O.bf16(r).view(np.uint32) & 0xFFFF == 0)


def _sklearn(sizes, W, b, X, Y):
    from sklearn.neural_network import MLPRegressor
    m = MLPRegressor(hidden_layer_sizes=sizes[1:-1], activation="relu", alpha=0.0, max_iter=1)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        m.fit(X, Y)
    m.coefs_ = [w.T.copy() for w in W]
    m.intercepts_ = [x.copy() for x in b]
    return m


def test_oracle_forward_matches_sklearn_mlpregressor():
    sizes = (6, 40, 30, 4)
    W, b = _net(sizes, 1)
    rng = np.random.default_rng(2)
    X = rng.uniform(-1, 1, (64, 6))
    Y = rng.normal(size=(64, 4))
    m = _sklearn(sizes, W, b, X, Y)
    y, _, _ = O.forward(W, b, X, "relu", rnd=False)
    assert np.allclose(y, m.predict(X), rtol=1e-12, atol=1e-12)


def test_oracle_gradients_match_sklearn_backprop():
    sizes = (6, 40, 30, 4)
    W, b = _net(sizes, 3)
    rng = np.random.default_rng(4)
    X = rng.uniform(-1, 1, (50, 6))
    Y = rng.normal(size=(50, 4))
    m = _sklearn(sizes, W, b, X, Y)
    nl = len(W)
    acts = [X] + [None] * nl
    deltas = [None] * nl
    cg = [np.empty_like(c) for c in m.coefs_]
    ig = [np.empty_like(c) for c in m.intercepts_]
    _, cg, ig = m._backprop(X, Y, None, acts, deltas, cg, ig)
    loss, dW, db, _ = O.backward(W, b, X, Y, "relu", rnd=False)
    k = 2.0 / sizes[-1]
    for l in range(nl):
        assert np.allclose(dW[l], k * cg[l].T, rtol=1e-10, atol=1e-14)
        assert np.allclose(db[l], k * ig[l], rtol=1e-10, atol=1e-14)
    assert loss == pytest.approx(np.mean((m.predict(X) - Y) ** 2), rel=1e-12)


@pytest.mark.parametrize("kind", ["gelu", "relu"])
def test_oracle_gradients_against_central_differences(kind):
    sizes = (6, 12, 10, 3)
    W, b = _net(sizes, 5)
    rng = np.random.default_rng(6)
    X = rng.uniform(-1, 1, (20, 6))
    Y = rng.normal(size=(20, 3))
    _, dW, db, dX = O.backward(W, b, X, Y, kind, rnd=False, input_grad=True)
    h = 1e-6

    def f(W_, b_, X_):
        return float(np.mean((O.forward(W_, b_, X_, kind, rnd=False)[0] - Y) ** 2))

    for l in range(len(W)):
        for (i, j) in [(0, 0), (1, 2), (W[l].shape[0] - 1, W[l].shape[1] - 1)]:
            Wp = [w.copy() for w in W]; Wp[l][i, j] += h
            Wm = [w.copy() for w in W]; Wm[l][i, j] -= h
            assert dW[l][i, j] == pytest.approx((f(Wp, b, X) - f(Wm, b, X)) / (2 * h), rel=1e-5, abs=1e-9)
        bp = [x.copy() for x in b]; bp[l][1] += h
        bm = [x.copy() for x in b]; bm[l][1] -= h
        assert db[l][1] == pytest.approx((f(W, bp, X) - f(W, bm, X)) / (2 * h), rel=1e-5, abs=1e-9)
    Xp = X.copy(); Xp[3, 2] += h
    Xm = X.copy(); Xm[3, 2] -= h
    assert dX[3, 2] == pytest.approx((f(W, b, Xp) - f(W, b, Xm)) / (2 * h), rel=1e-5, abs=1e-9)


def test_oracle_adam_first_steps():
    w, g = np.array([1.0, -2.0]), np.array([0.5, -0.25])
    m = v = np.zeros(2)
    w1, m, v = O.adam(w, g, m, v, 1, lr=0.1)
    # first bias-corrected Adam step moves each weight by lr against the gradient's sign
    assert np.allclose(w1, w - 0.1 * np.sign(g), rtol=1e-6)


def test_mlp_entry_points_reject_bad_arguments_before_device_work():
    L = dem.lib()
    buf = (C.c_uint8 * 4096)()
    a = C.addressof(buf)
    a16 = (a + 15) // 16 * 16
    ARG = -1
    assert L.dem_mlp_gemm_tn(a16, a16, 128, 64, 30, None, 0, a16, None, None) == ARG     # K not a multiple of 32
    assert L.dem_mlp_gemm_tn(a16 + 2, a16, 128, 64, 32, None, 0, a16, None, None) == ARG  # A not 16-byte aligned
    assert L.dem_mlp_gemm_tn(a16, a16, 128, 64, 32, None, 7, a16, None, None) == ARG     # unknown epilogue
    assert L.dem_mlp_gemm_tn(a16, a16, 128, 64, 32, None, 2, None, a16, None) == ARG     # GELU without bias
    assert L.dem_mlp_gemm_tn(a16, a16, 0, 64, 32, None, 0, a16, None, None) == ARG
    assert L.dem_mlp_act_backward(a16, a16, 16, 1, a16, None, None) == ARG               # plain bias is no activation
    assert L.dem_mlp_colsum(a16, 4, 4, a16, None, None) == ARG                           # no scratch
    assert L.dem_mlp_adam(a16, a16, a16, a16, 4, 1e-3, 0.9, 0.999, 1e-8, 0.0, None, None, None) == ARG
    assert L.dem_mlp_pack_bf16(a16, None, 4, 8, 4, a16, None) == ARG                     # kpad < k
    assert L.dem_mlp_transpose_bf16(a16, 8, 4, 4, a16, None) == ARG                      # ldo < rows
