"""TEST INFRASTRUCTURE ONLY -- the CPU checkers.

ctypes wrappers over
  * oracle/_build/libgcoracle.so : the plain-C restatement (gc_oracle.c), and
  * oracle/_ref/libgcref.so      : the unmodified reference sources compiled
                                   here (ref_shim.cpp + lib/*.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this package, and only to check or time the reference's algorithm; the
product (gmx_correlation_b200) never imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libgcoracle.so"
REF_SO = HERE / "_ref" / "libgcref.so"
# The reference checkout: $GMXCORR_REFERENCE, else a `reference` directory
# beside this repository's root.  Only build() reads it; the compiled
# libraries under _ref/ are all the checkers need afterwards.
_ROOT = HERE.parent
REF_SRC = Path(os.environ["GMXCORR_REFERENCE"]) if os.environ.get("GMXCORR_REFERENCE") else (
    _ROOT.parent / "reference")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(ref: bool = True) -> None:
    """Compile the restatement, and the reference when its sources exist."""
    targets = ["oracle"] + (["ref", "refgpu"] if ref and (REF_SRC / "lib").is_dir() else [])
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REF_SRC}", *targets], check=True)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class Oracle:
    """The C restatement of the reference algorithms."""

    def __init__(self):
        if not ORACLE_SO.exists():
            build(ref=False)
        L = ctypes.CDLL(str(ORACLE_SO))
        L.gco_ksg_pair_detail.restype = ctypes.c_double
        L.gco_gcmi_pair.restype = ctypes.c_double
        L.gco_te_pair.restype = ctypes.c_double
        L.gco_erfinv.restype = ctypes.c_double
        L.gco_erfinv.argtypes = [ctypes.c_double]
        self.L = L

    def prepare(self, x):
        n, T = x.shape[0], x.shape[1]
        X = np.zeros((3 * n, T))
        psi = np.zeros(T + 1)
        self.L.gco_prepare(_d(x), n, T, _d(X), _d(psi))
        return X, psi

    def ksg_pair_detail(self, X, psi, k, a1, a2):
        T = X.shape[1]
        nx = np.zeros(T, np.int32)
        ny = np.zeros(T, np.int32)
        ex = np.zeros(T)
        ey = np.zeros(T)
        kth = np.zeros(T, np.int32)
        dk = np.zeros(T)
        mi = self.L.gco_ksg_pair_detail(_d(X), T, k, a1, a2, _d(psi), _i(nx), _i(ny), _d(ex), _d(ey),
                                        _i(kth), _d(dk))
        return dict(mi=mi, nx=nx, ny=ny, epsx=ex, epsy=ey, kth=kth, dk=dk)

    def ksg_matrix(self, x, k, nthreads=0):
        n, T = x.shape[0], x.shape[1]
        m = np.zeros(n * n)
        if self.L.gco_ksg_matrix(_d(x), n, T, k, nthreads, _d(m)) != 0:
            raise ValueError("invalid KSG input")
        return m.reshape(n, n)

    def gauss_matrix(self, x):
        n, T = x.shape[0], x.shape[1]
        m = np.zeros(n * n)
        self.L.gco_gauss_matrix(_d(x), n, T, _d(m))
        return m.reshape(n, n)

    def gcmi_matrix(self, x):
        n, T = x.shape[0], x.shape[1]
        m = np.zeros(n * n)
        if self.L.gco_gcmi_matrix(_d(x), n, T, _d(m)) != 0:
            raise ValueError("invalid GCMI input")
        return m.reshape(n, n)

    def te_matrix(self, x, k, lag, nthreads=0):
        n, T = x.shape[0], x.shape[1]
        m = np.zeros(n * n)
        self.L.gco_te_matrix(_d(x), n, T, k, lag, nthreads, _d(m))
        return m.reshape(n, n)

    def te_pair(self, x, k, lag, a1, a2):
        n, T = x.shape[0], x.shape[1]
        Nv = T - lag
        psi = np.zeros(Nv + 1)
        self.L.gco_te_psi(Nv, _d(psi))
        nxp = np.zeros(Nv, np.int32)
        nxf = np.zeros(Nv, np.int32)
        nyp = np.zeros(Nv, np.int32)
        eps = np.zeros(Nv)
        te = self.L.gco_te_pair(_d(x), T, k, lag, a1, a2, _d(psi), _i(nxp), _i(nxf), _i(nyp), _d(eps))
        return dict(te=te, nxp=nxp, nxfxp=nxf, nypxp=nyp, eps=eps)

    def pearsify(self, m, dim=3):
        m = np.ascontiguousarray(m, dtype=np.float64).copy()
        self.L.gco_pearsify(_d(m), m.shape[0], dim)
        return m

    def center(self, raw):
        raw = np.ascontiguousarray(raw, dtype=np.float64)
        n, T = raw.shape[0], raw.shape[1]
        x = np.zeros_like(raw)
        xav = np.zeros((n, 3))
        self.L.gco_center(_d(raw), n, T, _d(x), _d(xav))
        return x, xav


class Reference:
    """The reference's own CPU code (compiled from its unmodified sources)."""

    def __init__(self):
        if not REF_SO.exists():
            if not (REF_SRC / "lib").is_dir():
                raise FileNotFoundError(f"{REF_SO} not built and the reference sources are absent")
            build(ref=True)
        L = ctypes.CDLL(str(REF_SO))
        L.gcref_last_error.restype = ctypes.c_char_p
        self.L = L

    @staticmethod
    def available() -> bool:
        return REF_SO.exists() or (REF_SRC / "lib").is_dir()

    def _ok(self, rc):
        if rc != 0:
            raise RuntimeError(self.L.gcref_last_error().decode())

    def max_threads(self) -> int:
        return int(self.L.gcref_max_threads())

    def milca(self, name, rows, k, *, dim=None, dimx=0, dimy=0, edim=1, tau=1, psi, scal=None, phi=None,
              minmax=(0.0, 1.0, 0.0, 1.0)):
        """One of the reference's MILCA estimators (lib/kraskov.cpp:347-2155) on
        rows (D, N); returns (out[4], floats[2K] for mi_d, the rows as the
        reference leaves them).  out: mic, mir, hc, hr, or 2K values."""
        x = np.array(rows, dtype=np.float64, order="C", copy=True)
        D, N = x.shape
        dim = D if dim is None else dim
        out = np.zeros(max(4, 2 * k))
        outf = np.zeros(2 * k, dtype=np.float32)
        # a zero word before the table: where a 1-D box count is -1 the
        # reference reads psi[-1]
        psig = np.concatenate([[0.0], np.asarray(psi, dtype=np.float64)])
        scal = np.zeros(D) if scal is None else np.ascontiguousarray(scal, dtype=np.float64)
        phi = np.zeros(k + 1) if phi is None else np.ascontiguousarray(phi, dtype=np.float64)
        f = self.L.gcref_milca
        f.argtypes = [ctypes.c_char_p, ctypes.c_void_p] + [ctypes.c_int] * 8 + [ctypes.c_void_p] * 3 + \
            [ctypes.c_double] * 4 + [ctypes.c_void_p] * 2
        self._ok(f(name.encode(), x.ctypes.data, D, N, k, dim, dimx, dimy, edim, tau, psig.ctypes.data + 8,
                   scal.ctypes.data, phi.ctypes.data, *[float(m) for m in minmax], out.ctypes.data,
                   outf.ctypes.data))
        return out, outf, x

    def ksg_matrix(self, x, k, nthreads=0):
        n, T = x.shape[0], x.shape[1]
        m = np.zeros(n * n)
        self._ok(self.L.gcref_ksg_matrix(_d(x), n, T, k, nthreads, _d(m)))
        return m.reshape(n, n)

    def ksg_pairs(self, x, k, a1, a2, nthreads=0):
        n, T = x.shape[0], x.shape[1]
        a1 = np.ascontiguousarray(a1, np.int32)
        a2 = np.ascontiguousarray(a2, np.int32)
        out = np.zeros(len(a1))
        self._ok(self.L.gcref_ksg_pairs(_d(x), n, T, k, _i(a1), _i(a2), len(a1), nthreads, _d(out)))
        return out

    def ksg_pair_detail(self, x, k, a1, a2):
        n, T = x.shape[0], x.shape[1]
        nx = np.zeros(T, np.int32)
        ny = np.zeros(T, np.int32)
        ex = np.zeros(T)
        ey = np.zeros(T)
        kth = np.zeros(T, np.int32)
        dk = np.zeros(T)
        mi = ctypes.c_double()
        self._ok(self.L.gcref_ksg_pair_detail(_d(x), n, T, k, a1, a2, _i(nx), _i(ny), _d(ex), _d(ey),
                                              _i(kth), _d(dk), ctypes.byref(mi)))
        return dict(mi=mi.value, nx=nx, ny=ny, epsx=ex, epsy=ey, kth=kth, dk=dk)

    def prepare(self, x):
        n, T = x.shape[0], x.shape[1]
        X = np.zeros((3 * n, T))
        psi = np.zeros(T + 1)
        self._ok(self.L.gcref_prepare(_d(x), n, T, _d(X), _d(psi)))
        return X, psi

    def gauss_matrix(self, x):
        n, T = x.shape[0], x.shape[1]
        m = np.zeros(n * n)
        self._ok(self.L.gcref_gauss_matrix(_d(x), n, T, _d(m)))
        return m.reshape(n, n)

    def gcmi_matrix(self, x, nthreads=0):
        n, T = x.shape[0], x.shape[1]
        m = np.zeros(n * n)
        self._ok(self.L.gcref_gcmi_matrix(_d(x), n, T, nthreads, _d(m)))
        return m.reshape(n, n)

    def te_matrix(self, x, k, lag, nthreads=0):
        n, T = x.shape[0], x.shape[1]
        m = np.zeros(n * n)
        self._ok(self.L.gcref_te_matrix(_d(x), n, T, k, lag, nthreads, _d(m)))
        return m.reshape(n, n)

    def pearsify(self, m, dim=3):
        m = np.ascontiguousarray(m, dtype=np.float64).copy()
        self.L.gcref_pearsify(_d(m), m.shape[0], dim)
        return m

    def write_matrix(self, m, path):
        m = np.ascontiguousarray(m, dtype=np.float64)
        self._ok(self.L.gcref_write_matrix(_d(m), m.shape[0], str(path).encode()))

    def write_xpm(self, m, path, title, legend):
        m = np.ascontiguousarray(m, dtype=np.float64)
        self._ok(self.L.gcref_write_xpm(_d(m), m.shape[0], str(path).encode(), title.encode(),
                                        legend.encode()))
