"""The MILCA estimator family of the reference's lib/kraskov.cpp (:347-2155).

    out = milca("mi_xnyn", rows, k=10, dimx=3, dimy=3, psi=psi, scal=scal)
    out["mic"], out["mir"], out["rows"]

``rows``: (D, N) float64, one row per variable component (the reference's
``double **x``); ``psi``: digamma table psi[0..N] (default: the reference's
table, ``kraskov_prepare``'s); ``scal``: per-row scale of the 1-D box counts
(default (N-5) / (max + 1e-9) per row, so every box lies in 0..N-5).  The
returned ``rows`` are sorted as the reference leaves its caller's rows.  The
k = 1..K forms (mi2K, redK, mi_xnynK, mi_xnynKembed, mi_d) return ``mic`` and
``mir`` arrays of K values; mi2h adds ``hc`` and ``hr``.
"""

from __future__ import annotations

import ctypes

import numpy as np

_RANGE = {"mi2K", "redK", "mi_xnynK", "mi_xnynKembed", "mi_d"}
NAMES = ["mi2", "mi2c", "mi2r", "mi2r_", "mi2K", "mi2h", "red", "redc", "redr", "redK", "redr_embed", "mi_xnyn",
         "mic_xnyn", "mir_xnyn", "mi_xnynK", "mi_xnynKembed", "mi_d"]


def psi_table(n: int) -> np.ndarray:
    """The reference's digamma table psi[0..n] (psi[1] = -0.57721566490153, psi[i+1] = psi[i] + 1/i)."""
    p = np.zeros(n + 1)
    if n >= 1:
        p[1] = -0.57721566490153
    for i in range(1, n):
        p[i + 1] = p[i] + 1.0 / i
    return p


def default_scal(rows: np.ndarray) -> np.ndarray:
    n = rows.shape[1]
    return (n - 5) / (rows.max(axis=1) + 1e-9)


def milca(name: str, rows, k: int, *, dim=None, dimx=None, dimy=None, edim=1, tau=1, psi=None, scal=None, phi=None,
          minmax=None) -> dict:
    from . import _check, lib

    if name not in NAMES:
        raise ValueError(f"unknown MILCA function {name!r}")
    x = np.array(rows, dtype=np.float64, order="C", copy=True)
    D, N = x.shape
    dim = D if dim is None else dim
    psi = psi_table(N) if psi is None else np.ascontiguousarray(psi, dtype=np.float64)
    scal = default_scal(x) if scal is None else np.ascontiguousarray(scal, dtype=np.float64)
    L = lib()
    ptrs = (ctypes.POINTER(ctypes.c_double) * D)(*[x[d].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
                                                  for d in range(D)])
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    ps, sc = dp(psi), dp(scal)
    v = (ctypes.c_double * 4)()
    r = lambda i: ctypes.byref(v, 8 * i)  # noqa: E731
    fn = getattr(L, "gc_milca_" + name)
    fn.restype = ctypes.c_int
    out = {}
    kr = np.zeros(2 * k)
    if name in ("mi2", "mi2c", "mi2r", "mi2r_"):
        args = {"mi2": (r(0), r(1)), "mi2c": (r(0),), "mi2r": (r(1),), "mi2r_": (r(1),)}[name]
        _check(fn(ptrs, N, k, ps, sc, *args))
    elif name == "mi2h":
        _check(fn(ptrs, N, k, ps, sc, r(0), r(1), r(2), r(3)))
        out["hc"], out["hr"] = v[2], v[3]
    elif name in ("red", "redc", "redr"):
        args = {"red": (r(0), r(1)), "redc": (r(0),), "redr": (r(1),)}[name]
        _check(fn(ptrs, dim, N, k, ps, sc, *args))
    elif name == "redr_embed":
        _check(fn(ptrs, dim, edim, tau, N, k, ps, r(1)))
    elif name in ("mi_xnyn", "mic_xnyn", "mir_xnyn"):
        args = {"mi_xnyn": (r(0), r(1)), "mic_xnyn": (r(0),), "mir_xnyn": (r(1),)}[name]
        _check(fn(ptrs, dimx, dimy, N, k, ps, sc, *args))
    elif name == "mi2K":
        _check(fn(ptrs, N, k, ps, sc, dp(kr)))
    elif name == "redK":
        _check(fn(ptrs, dim, N, k, ps, sc, dp(kr)))
    elif name == "mi_xnynK":
        _check(fn(ptrs, dimx, dimy, N, k, ps, sc, dp(kr)))
    elif name == "mi_xnynKembed":
        _check(fn(ptrs, dim, N, k, ps, dp(kr)))
    elif name == "mi_d":
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        kf = np.zeros(2 * k, dtype=np.float32)
        _check(fn(ptrs, dim, N, k, kf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ps, dp(phi),
                  *[ctypes.c_double(float(m)) for m in minmax]))
        kr = kf
    if name in _RANGE:
        out["mic"], out["mir"] = kr[0::2].copy(), kr[1::2].copy()
    else:
        if name in ("mi2", "mi2c", "mi2h", "red", "redc", "mi_xnyn", "mic_xnyn"):
            out["mic"] = v[0]
        if name in ("mi2", "mi2r", "mi2r_", "mi2h", "red", "redr", "redr_embed", "mi_xnyn", "mir_xnyn"):
            out["mir"] = v[1]
    out["rows"] = x
    return out
