"""CPU checks of the learned screen's float64 restatement (oracle/screen_ref.py):
its gradient against central differences and torch autograd, its bfloat16
rounding against torch's, and its Gaussian-MI feature against the
reference's -linear estimator restated in oracle/gc_oracle.c."""

import math

import numpy as np
import pytest
import torch

from oracle import screen_ref as sr
from gmx_correlation_b200.synth import synth_traj


def _params(rng, scale=1.0):
    p = np.zeros(sr.STRIDE)
    for off, n, fan in [(sr.OFF_W1, sr.HIDDEN * sr.IN, sr.IN), (sr.OFF_B1, sr.HIDDEN, sr.IN),
                        (sr.OFF_W2, sr.HIDDEN ** 2, sr.HIDDEN), (sr.OFF_B2, sr.HIDDEN, sr.HIDDEN),
                        (sr.OFF_W3, sr.HIDDEN ** 2, sr.HIDDEN), (sr.OFF_B3, sr.HIDDEN, sr.HIDDEN),
                        (sr.OFF_W4, sr.HIDDEN, sr.HIDDEN), (sr.OFF_B4, 1, sr.HIDDEN)]:
        p[off:off + n] = rng.uniform(-scale, scale, n) / math.sqrt(fan)
    return p


def test_layout_matches_library_constants():
    assert sr.N_PARAMS == 38401 and sr.STRIDE == 38464


def test_backward_matches_central_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    X = rng.standard_normal((48, sr.IN))
    t = rng.uniform(0, 1, 48)
    y, cache = sr.forward(p, X)
    g, _ = sr.backward(p, cache, y, t)
    idx = np.concatenate([rng.choice(np.arange(sr.OFF_W1, sr.OFF_B1), 6), rng.choice(np.arange(sr.OFF_W2, sr.OFF_B2), 6),
                          rng.choice(np.arange(sr.OFF_W3, sr.OFF_B3), 6), np.arange(sr.OFF_W4, sr.OFF_W4 + 4),
                          [sr.OFF_B1 + 3, sr.OFF_B2 + 5, sr.OFF_B3 + 7, sr.OFF_B4]])
    num = sr.numeric_grad(p, X, t, idx)
    np.testing.assert_allclose(g[idx], num, rtol=1e-5, atol=1e-9)


def test_backward_matches_torch_autograd():
    rng = np.random.default_rng(1)
    p = _params(rng)
    X = rng.standard_normal((64, sr.IN))
    t = rng.uniform(0, 1, 64)
    y, cache = sr.forward(p, X)
    g, loss = sr.backward(p, cache, y, t)
    P = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    Xt, tt = torch.tensor(X), torch.tensor(t)

    def sl(a, b):
        return P[a:b]

    h = Xt
    for ow, ob, fin in [(sr.OFF_W1, sr.OFF_B1, sr.IN), (sr.OFF_W2, sr.OFF_B2, sr.HIDDEN),
                        (sr.OFF_W3, sr.OFF_B3, sr.HIDDEN)]:
        W = sl(ow, ob).reshape(sr.HIDDEN, fin)
        b = sl(ob, ob + sr.HIDDEN)
        h = torch.nn.functional.gelu(h @ W.T + b)
    yt = h @ sl(sr.OFF_W4, sr.OFF_B4) + P[sr.OFF_B4]
    lt = ((yt - tt) ** 2).mean()
    lt.backward()
    assert abs(lt.item() - loss) < 1e-12
    np.testing.assert_allclose(g[:sr.N_PARAMS], P.grad.numpy()[:sr.N_PARAMS], rtol=1e-9, atol=1e-14)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(2)
    v = np.concatenate([rng.standard_normal(4000) * 10 ** rng.uniform(-6, 6, 4000),
                        [1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.0 - 2 ** -8, 0.0]]).astype(np.float32)
    ours = sr.bf16(v)
    theirs = torch.tensor(v).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(ours, theirs)


def test_gaussian_feature_matches_linear_estimator(oracle):
    x = synth_traj(12, 400, 6, 0.05, 3)
    st = sr.atom_stats(x)
    a1 = np.array([1, 5, 11, 7])
    a2 = np.array([0, 2, 3, 6])
    F = sr.pair_features(x, 10, a1, a2, stats=st)
    gm = oracle.gauss_matrix(x)
    np.testing.assert_allclose(F[:, 0], gm[a1, a2], rtol=1e-9, atol=1e-12)
    assert F.shape == (4, sr.BASE + sr.HIST)
    # histogram cells are fractions of T summing to 1; eigenvalues sum to 6
    np.testing.assert_allclose(F[:, sr.BASE:].sum(1), 1.0, atol=1e-12)
    np.testing.assert_allclose(F[:, 1:7].sum(1), 6.0, atol=1e-9)
    assert np.all(F[:, 22] == 10 / 400)
