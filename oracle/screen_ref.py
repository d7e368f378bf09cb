"""TEST INFRASTRUCTURE ONLY -- CPU restatement of the learned KSG screen.

The screen has no counterpart in the reference; this module restates the
library's own definitions (include/gmx_corr_b200.h, "Learned KSG screen")
in float64 numpy so that tests can check the CUDA kernels against them:

  * ``atom_stats`` / ``pair_features``: the per-pair feature rows of
    gmx_correlation_b200/csrc/screen_features.cu;
  * ``forward`` / ``backward``: the ensemble network
    40 -> 128 -> 128 -> 128 -> 1 with exact-erf GELU and the mean squared
    error, in exact float64 arithmetic, or with every matrix-product operand
    rounded to bfloat16 (round to nearest even) as the tensor-core kernels
    do (``bf16=True``).

Only tests/ use it; the product never imports it.
"""

from __future__ import annotations

import math

import numpy as np

BASE, HIST, COMP, HIDDEN = 23, 64, 17, 128
IN = BASE + COMP

# Parameter layout of one member (floats), as gc_screen_param_stride documents.
OFF_W1 = 0
OFF_B1 = OFF_W1 + HIDDEN * IN
OFF_W2 = OFF_B1 + HIDDEN
OFF_B2 = OFF_W2 + HIDDEN * HIDDEN
OFF_W3 = OFF_B2 + HIDDEN
OFF_B3 = OFF_W3 + HIDDEN * HIDDEN
OFF_W4 = OFF_B3 + HIDDEN
OFF_B4 = OFF_W4 + HIDDEN
N_PARAMS = OFF_B4 + 1
STRIDE = (N_PARAMS + 63) // 64 * 64


# ---------------------------------------------------------------- features

def atom_stats(x):
    """Per-atom means, sds, kurtoses, covariance (all / T), PC1 rank bins."""
    n, T, _ = x.shape
    mean = x.sum(1) / T
    xc = x - mean[:, None, :]
    cov = np.einsum("atd,ate->ade", xc, xc) / T
    var = np.einsum("add->ad", cov)
    m4 = (xc ** 4).sum(1) / T
    kurt = np.where(var > 0, m4 / np.where(var > 0, var * var, 1.0) - 3.0, 0.0)
    bins = np.zeros((n, T), np.int64)
    for a in range(n):
        w, v = np.linalg.eigh(cov[a])
        ax = v[:, -1]
        big = np.argmax(np.abs(ax))
        if ax[big] < 0:
            ax = -ax
        proj = (xc[a] @ ax).astype(np.float32)
        order = np.lexsort((np.arange(T), proj))  # by value, then frame
        bins[a, order] = (8 * np.arange(T)) // T
    return dict(mean=mean, sd=np.sqrt(var), kurt=kurt, cov=cov, bins=bins, xc=xc)


def pair_features(x, k, a1, a2, pca=None, stats=None):
    """Feature rows (len(a1), 40) with pca=(mean[64], comp[17][64]), else
    (len(a1), 87) with the raw histogram cells."""
    st = stats if stats is not None else atom_stats(x)
    T = x.shape[1]
    rows = []
    for p, q in zip(np.atleast_1d(a1), np.atleast_1d(a2)):
        cr = st["xc"][p].T @ st["xc"][q] / T
        C = np.block([[st["cov"][p], cr], [cr.T, st["cov"][q]]])
        d1, d2, d6 = np.linalg.det(st["cov"][p]), np.linalg.det(st["cov"][q]), np.linalg.det(C)
        g = 0.5 * (math.log(d1) + math.log(d2) - math.log(d6)) if min(d1, d2, d6) > 0 else 0.0
        sd = np.concatenate([st["sd"][p], st["sd"][q]])
        R = C / np.outer(sd, sd)
        ev = np.sort(np.linalg.eigvalsh(R))[::-1]
        k1 = np.sort(st["kurt"][p])[::-1]
        k2 = np.sort(st["kurt"][q])[::-1]
        if k2[0] > k1[0]:
            k1, k2 = k2, k1
        cc = np.sort(np.abs(R[:3, 3:]).ravel())[::-1]
        h = np.bincount(st["bins"][p] * 8 + st["bins"][q], minlength=64).reshape(8, 8).astype(np.float64)
        i = np.arange(8) - 3.5
        if (h * np.outer(i, i)).sum() < 0:
            h = h[:, ::-1]
        cells = (0.5 * (h + h.T) / T).ravel()
        if pca is not None:
            tail = (cells - pca[0]) @ np.asarray(pca[1], np.float64).T
        else:
            tail = cells
        rows.append(np.concatenate([[g], ev, k1, k2, cc, [k / T], tail]))
    return np.array(rows)


# ----------------------------------------------------------------- network

def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float64)
    return dict(W1=p[OFF_W1:OFF_B1].reshape(HIDDEN, IN), b1=p[OFF_B1:OFF_W2],
                W2=p[OFF_W2:OFF_B2].reshape(HIDDEN, HIDDEN), b2=p[OFF_B2:OFF_W3],
                W3=p[OFF_W3:OFF_B3].reshape(HIDDEN, HIDDEN), b3=p[OFF_B3:OFF_W4],
                W4=p[OFF_W4:OFF_B4].reshape(1, HIDDEN), b4=p[OFF_B4:OFF_B4 + 1])


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def standardise(F, mean, sd):
    """(F - mean) / sd in float32, as the gather kernel computes it."""
    F = np.asarray(F, np.float32)
    return ((F - np.asarray(mean, np.float32)) / np.asarray(sd, np.float32)).astype(np.float64)


def forward(params, X, bf16_ops=False):
    """One member: X (M, 40) standardised -> (y (M,), cache)."""
    P = unpack(params)
    r = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))
    cache = {"X": X}
    h = X
    for l in (1, 2, 3):
        z = r(h) @ r(P[f"W{l}"]).T + P[f"b{l}"]
        cache[f"Z{l}"] = z
        h = gelu(z)
        cache[f"H{l}"] = h
    y = (r(h) @ r(P["W4"]).T)[:, 0] + P["b4"][0]
    return y, cache


def backward(params, cache, y, t, bf16_ops=False):
    """Gradient (STRIDE,) of mean((y - t)^2) and the loss."""
    P = unpack(params)
    r = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))
    M = len(t)
    d = y - np.asarray(t, np.float64)
    loss = float((d * d).mean())
    dY = (2.0 * d / M)[:, None]
    # bf16 emulation: dY and dZ are float32 on the device before rounding
    g = np.zeros(STRIDE)
    ins = {1: cache["X"], 2: cache["H1"], 3: cache["H2"], 4: cache["H3"]}
    dZ = dY
    offs = {1: (OFF_W1, OFF_B1), 2: (OFF_W2, OFF_B2), 3: (OFF_W3, OFF_B3), 4: (OFF_W4, OFF_B4)}
    for l in (4, 3, 2, 1):
        ow, ob = offs[l]
        W = P[f"W{l}"]
        gW = r(dZ).T @ r(ins[l])
        g[ow:ow + W.size] = gW.ravel()
        g[ob:ob + W.shape[0]] = dZ.sum(0)
        if l > 1:
            dH = r(dZ) @ r(W)
            dZ = dH * gelu_grad(cache[f"Z{l - 1}"])
    return g, loss


def member_grad(params, F, t, mean, sd, bf16_ops=False):
    X = standardise(F, mean, sd)
    y, cache = forward(params, X, bf16_ops)
    return backward(params, cache, y, t, bf16_ops)


def numeric_grad(params, X, t, idx, h=1e-6):
    """Central differences of the float64 loss at parameter indices idx."""
    out = np.zeros(len(idx))
    p = np.array(params, np.float64)
    for j, i in enumerate(idx):
        old = p[i]
        p[i] = old + h
        lp = float(((forward(p, X)[0] - t) ** 2).mean())
        p[i] = old - h
        lm = float(((forward(p, X)[0] - t) ** 2).mean())
        p[i] = old
        out[j] = (lp - lm) / (2 * h)
    return out
