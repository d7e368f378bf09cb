"""gmx_correlation_b200 -- all-pairs generalized correlation on NVIDIA B200.

Python host binding of the C ABI in include/gmx_corr_b200.h.  The function
names and argument meanings follow the reference's estimator interface
(scdantu/gmx_correlation lib/correlation_core.h, lib/gcmi.h,
lib/transfer_entropy.h):

    kraskov_corrmatrix(x, k)      KSG (Kraskov alg. 2) MI matrix
    gauss_corrmatrix(x)           Gaussian (-linear) MI matrix
    gcmi_corrmatrix(x)            Gaussian-copula MI matrix
    te_matrix(x, k, lag)          transfer entropy, te[a1, a2] = TE(a2 -> a1)
    pearsify(mat, dim)            r(MI) = sqrt(1 - exp(-2 MI / dim))
    write_matrix / write_xpm_matrix / read_matrix

``x`` is the mean-centred t_traj block, shape (natoms, nframes, 3) float64.
Every estimator computes on the GPU; if the CUDA library is missing or no
device is present the call raises -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

__all__ = [
    "GCError", "lib", "gpu_available", "kraskov_corrmatrix", "gauss_corrmatrix",
    "gcmi_corrmatrix", "te_matrix", "kraskov_prepare", "kraskov_wrap", "pearsify",
    "write_matrix", "write_xpm_matrix", "read_matrix", "KsgPlan", "PATH_AUTO",
    "PATH_EXACT_FP64", "LIB_PATH", "probe_fp32", "screen_features", "ScreenModel", "ksg_screened",
    "SCREEN_IN", "SCREEN_RAW", "SCREEN_BASE", "SCREEN_COMP", "release_cache", "ksg_batch",
    "ksg_batch_release", "te_batch", "gcmi_batch", "corr_batch", "batch_release", "TePlan",
    "read_trajectory", "write_trajectory", "trajectory_info", "read_index", "parse_atoms",
]

LIB_PATH = Path(__file__).resolve().parent / "libgmxcorr_b200.so"
PATH_AUTO = 0
PATH_EXACT_FP64 = 1
# Learned-screen feature layout (include/gmx_corr_b200.h): 23 scalar
# features, then 17 histogram components (40) or the 64 raw cells (87).
SCREEN_BASE = 23
SCREEN_COMP = 17
SCREEN_IN = SCREEN_BASE + SCREEN_COMP
SCREEN_RAW = SCREEN_BASE + 64

_STATUS = {
    1: "invalid argument", 2: "no CUDA device", 3: "CUDA error", 4: "zero-variance component",
    5: "non-finite coordinate", 6: "out of device memory", 7: "I/O error", 8: "internal error",
    9: "device wait timed out",
}


class GCError(RuntimeError):
    """A C-ABI call failed; ``status`` holds the gc_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{_STATUS.get(status, status)}] {message}")
        self.status = status


class _TrajView(ctypes.Structure):
    _fields_ = [("natoms", ctypes.c_int), ("nframes", ctypes.c_int),
                ("xyz", ctypes.POINTER(ctypes.c_double)),
                ("rows", ctypes.POINTER(ctypes.POINTER(ctypes.c_double)))]


class _Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("path", ctypes.c_int), ("pair_begin", ctypes.c_long),
                ("pair_end", ctypes.c_long), ("stream", ctypes.c_void_p),
                ("detail_nx", ctypes.POINTER(ctypes.c_int32)),
                ("detail_ny", ctypes.POINTER(ctypes.c_int32)),
                ("pair_list", ctypes.POINTER(ctypes.c_int64)), ("pair_list_len", ctypes.c_long),
                ("variant", ctypes.c_int)]


class _ScreenOpts(ctypes.Structure):
    _fields_ = [("audit_frac", ctypes.c_double), ("sigma_max", ctypes.c_double), ("margin", ctypes.c_double),
                ("seed", ctypes.c_uint64)]


class _ScreenReport(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_long), ("flagged", ctypes.c_long), ("audited", ctypes.c_long),
                ("exact", ctypes.c_long), ("audit_accepted", ctypes.c_long), ("threshold", ctypes.c_double),
                ("audit_max_dr", ctypes.c_double), ("audit_rms_dr", ctypes.c_double),
                ("final_max_dr", ctypes.c_double), ("ms_features", ctypes.c_float), ("ms_mlp", ctypes.c_float),
                ("ms_ksg", ctypes.c_float)]


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded libgmxcorr_b200.so (raises if it was never built)."""
    global _lib
    if _lib is None:
        path = Path(os.environ.get("GMXCORR_B200_LIB", LIB_PATH))
        if not path.exists():
            raise GCError(3, f"{path} is missing: build it with `python -m gmx_correlation_b200.build`")
        L = ctypes.CDLL(str(path))
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)
        L.gc_last_error.restype = ctypes.c_char_p
        L.gc_opts_init.argtypes = [ctypes.POINTER(_Opts)]
        L.gc_ksg_matrix.argtypes = [ctypes.POINTER(_TrajView), ctypes.c_int, ctypes.POINTER(_Opts), dp]
        L.gc_ksg_matrix_prepared.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(_Opts), dp]
        L.gc_gauss_matrix.argtypes = [ctypes.POINTER(_TrajView), ctypes.POINTER(_Opts), dp]
        L.gc_gcmi_matrix.argtypes = [ctypes.POINTER(_TrajView), ctypes.POINTER(_Opts), dp]
        L.gc_te_matrix.argtypes = [ctypes.POINTER(_TrajView), ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(_Opts), dp]
        L.gc_ksg_prepare.argtypes = [ctypes.POINTER(_TrajView), ctypes.POINTER(_Opts), dp, dp, dp]
        L.gc_ksg_pair.argtypes = [dp, ctypes.c_int, ctypes.c_int, dp, ctypes.POINTER(_Opts), dp]
        L.gc_pearsify.argtypes = [dp, ctypes.c_int, ctypes.c_int]
        L.gc_pearsify.restype = None
        L.gc_write_matrix.argtypes = [dp, ctypes.c_int, ctypes.c_char_p]
        L.gc_write_xpm.argtypes = [dp, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p]
        L.gc_ksg_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Opts),
                                         ctypes.POINTER(ctypes.c_void_p)]
        L.gc_ksg_plan_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.gc_ksg_plan_sync.argtypes = [ctypes.c_void_p]
        L.gc_ksg_plan_pairs.argtypes = [ctypes.c_void_p]
        L.gc_ksg_plan_pairs.restype = ctypes.c_long
        L.gc_ksg_plan_launches.argtypes = [ctypes.c_void_p]
        L.gc_ksg_plan_handoffs.argtypes = [ctypes.c_void_p]
        L.gc_ksg_plan_handoffs.restype = ctypes.c_long
        L.gc_ksg_plan_is_fast.argtypes = [ctypes.c_void_p]
        L.gc_ksg_plan_handoff_reason.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.gc_ksg_plan_handoff_reason.restype = ctypes.c_long
        L.gc_ksg_plan_walk_mean.argtypes = [ctypes.c_void_p]
        L.gc_ksg_plan_walk_mean.restype = ctypes.c_double
        L.gc_ksg_plan_kernel_ms.argtypes = [ctypes.c_void_p]
        L.gc_ksg_plan_kernel_ms.restype = ctypes.c_float
        L.gc_probe_fp32.argtypes = [ctypes.c_int, dp, dp]
        L.gc_ksg_pair_mi_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_void_p, ctypes.c_void_p]
        L.gc_te_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(_Opts), ctypes.POINTER(ctypes.c_void_p)]
        L.gc_te_plan_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.gc_te_plan_sync.argtypes = [ctypes.c_void_p]
        for name, res in (("gc_te_plan_pairs", ctypes.c_long), ("gc_te_plan_launches", ctypes.c_int),
                          ("gc_te_plan_is_walk", ctypes.c_int), ("gc_te_plan_handoffs", ctypes.c_long),
                          ("gc_te_plan_walk_mean", ctypes.c_double), ("gc_te_plan_kernel_ms", ctypes.c_float)):
            getattr(L, name).argtypes = [ctypes.c_void_p]
            getattr(L, name).restype = res
        L.gc_te_plan_counts.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ip, ip, ip]
        L.gc_te_plan_destroy.argtypes = [ctypes.c_void_p]
        L.gc_te_plan_destroy.restype = None
        L.gc_ksg_plan_destroy.argtypes = [ctypes.c_void_p]
        L.gc_ksg_plan_destroy.restype = None
        L.gc_release_cache.restype = None
        L.gc_ksg_batch.argtypes = [ctypes.POINTER(_TrajView), ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                   ctypes.POINTER(_Opts), ctypes.POINTER(dp)]
        L.gc_ksg_batch_release.restype = None
        L.gc_te_batch.argtypes = [ctypes.POINTER(_TrajView), ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(_Opts), ctypes.POINTER(dp)]
        L.gc_te_batch_release.restype = None
        L.gc_gcmi_batch.argtypes = [ctypes.POINTER(_TrajView), ctypes.c_int, ctypes.POINTER(_Opts),
                                    ctypes.POINTER(dp)]
        L.gc_gcmi_batch_release.restype = None
        fp = ctypes.POINTER(ctypes.c_float)
        L.gc_screen_features.argtypes = [ctypes.POINTER(_TrajView), ctypes.c_int, ctypes.POINTER(_Opts), fp, fp, fp]
        L.gc_screen_model_create.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_void_p)]
        L.gc_screen_model_destroy.argtypes = [ctypes.c_void_p]
        L.gc_screen_model_destroy.restype = None
        L.gc_screen_model_members.argtypes = [ctypes.c_void_p]
        L.gc_screen_param_stride.restype = ctypes.c_long
        L.gc_screen_model_get_params.argtypes = [ctypes.c_void_p, fp]
        L.gc_screen_model_set_params.argtypes = [ctypes.c_void_p, fp]
        L.gc_screen_model_set_input.argtypes = [ctypes.c_void_p, fp, fp, fp, fp]
        L.gc_screen_train.argtypes = [ctypes.c_void_p, fp, fp, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_uint64, fp]
        L.gc_screen_grad.argtypes = [ctypes.c_void_p, fp, fp, ctypes.c_long, fp, fp]
        L.gc_screen_predict.argtypes = [ctypes.c_void_p, fp, ctypes.c_long, fp]
        L.gc_screen_opts_init.argtypes = [ctypes.POINTER(_ScreenOpts)]
        L.gc_screen_opts_init.restype = None
        L.gc_ksg_screened.argtypes = [ctypes.POINTER(_TrajView), ctypes.c_int, ctypes.c_void_p,
                                      ctypes.POINTER(_ScreenOpts), ctypes.POINTER(_Opts), dp,
                                      ctypes.POINTER(_ScreenReport)]
        _ = ip
        _lib = L
    return _lib


def _check(status: int):
    if status != 0:
        raise GCError(status, lib().gc_last_error().decode(errors="replace"))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _coords(x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.ndim != 3 or x.shape[2] != 3:
        raise ValueError("coordinates must have shape (natoms, nframes, 3)")
    return x


def _view(x: np.ndarray) -> _TrajView:
    v = _TrajView()
    v.natoms, v.nframes = x.shape[0], x.shape[1]
    v.xyz = _dptr(x)
    v.rows = None
    return v


VARIANT_DEFAULT, VARIANT_HBM_GATHER = 0, 1


def _opts(device=-1, path=PATH_AUTO, pairs=None, stream=None, pair_list=None, variant=VARIANT_DEFAULT) -> _Opts:
    o = _Opts()
    lib().gc_opts_init(ctypes.byref(o))
    o.device, o.path, o.variant = device, path, variant
    if pairs is not None:
        o.pair_begin, o.pair_end = int(pairs[0]), int(pairs[1])
    if pair_list is not None:
        o._keep = np.ascontiguousarray(pair_list, dtype=np.int64)
        o.pair_list = o._keep.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        o.pair_list_len = len(o._keep)
    if stream is not None:
        o.stream = ctypes.c_void_p(stream)
    return o


def probe_fp32(device: int = -1):
    """(FADD+FMNMX lane-ops/s, FFMA flop/s) measured on the device."""
    mix, fma = ctypes.c_double(), ctypes.c_double()
    _check(lib().gc_probe_fp32(device, ctypes.byref(mix), ctypes.byref(fma)))
    return mix.value, fma.value


def gpu_available() -> bool:
    """True when a compute-capability 10.x (B200) device is visible."""
    return bool(lib().gc_gpu_available())


def kraskov_corrmatrix(x, k: int, *, path: int = PATH_AUTO, device: int = -1, pairs=None,
                       detail: bool = False, pair_list=None):
    """KSG MI matrix (natoms x natoms), diagonal 2000, as kraskov_corrmatrix.

    ``pairs=(begin, end)`` computes only that shard of the pair list
    p = a1*(a1-1)/2 + a2; ``pair_list`` computes exactly the listed pair
    indices.  With ``detail=True`` also returns the per-query counts
    (nx, ny), each of shape (npairs_computed, nframes).
    """
    x = _coords(x)
    n, T = x.shape[0], x.shape[1]
    out = np.zeros(n * n)
    o = _opts(device, path, pairs, pair_list=pair_list)
    nx = ny = None
    if detail:
        npairs = n * (n - 1) // 2
        b, e = (0, npairs) if pairs is None else (pairs[0], pairs[1] if pairs[1] > 0 else npairs)
        cnt = len(pair_list) if pair_list is not None else max(e - b, 0)
        nx = np.zeros((cnt, T), np.int32)
        ny = np.zeros_like(nx)
        o.detail_nx = nx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        o.detail_ny = ny.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    v = _view(x)
    _check(lib().gc_ksg_matrix(ctypes.byref(v), int(k), ctypes.byref(o), _dptr(out)))
    mat = out.reshape(n, n)
    return (mat, nx, ny) if detail else mat


def ksg_batch(trajs, ks, *, device: int = -1):
    """KSG MI matrices of several trajectories in one batched GPU run.

    ``trajs``: list of (natoms_i, nframes_i, 3) mean-centred arrays; ``ks``:
    one k per trajectory (or a single int).  Returns the list of matrices.
    """
    xs = [_coords(x) for x in trajs]
    if isinstance(ks, int):
        ks = [ks] * len(xs)
    if len(ks) != len(xs):
        raise ValueError("one k per trajectory")
    views = (_TrajView * len(xs))()
    for v, x in zip(views, xs):
        v.natoms, v.nframes = x.shape[0], x.shape[1]
        v.xyz = _dptr(x)
        v.rows = None
    outs = [np.zeros((x.shape[0], x.shape[0])) for x in xs]
    ptrs = (ctypes.POINTER(ctypes.c_double) * len(xs))(*[_dptr(m) for m in outs])
    karr = (ctypes.c_int * len(xs))(*[int(k) for k in ks])
    o = _opts(device)
    _check(lib().gc_ksg_batch(views, karr, len(xs), ctypes.byref(o), ptrs))
    return outs


def _views(xs):
    views = (_TrajView * len(xs))()
    for v, x in zip(views, xs):
        v.natoms, v.nframes = x.shape[0], x.shape[1]
        v.xyz = _dptr(x)
        v.rows = None
    return views


def te_batch(trajs, ks, lag: int = 1, *, device: int = -1):
    """TE matrices (te[a1, a2] = TE(a2 -> a1)) of several trajectories at one
    lag in one batched GPU run; ``ks`` one k per trajectory (or one int)."""
    xs = [_coords(x) for x in trajs]
    if isinstance(ks, int):
        ks = [ks] * len(xs)
    if len(ks) != len(xs):
        raise ValueError("one k per trajectory")
    outs = [np.zeros((x.shape[0], x.shape[0])) for x in xs]
    ptrs = (ctypes.POINTER(ctypes.c_double) * len(xs))(*[_dptr(m) for m in outs])
    karr = (ctypes.c_int * len(xs))(*[int(k) for k in ks])
    o = _opts(device)
    _check(lib().gc_te_batch(_views(xs), karr, len(xs), int(lag), ctypes.byref(o), ptrs))
    return outs


def gcmi_batch(trajs, *, device: int = -1):
    """GCMI matrices of several trajectories in one batched GPU run."""
    xs = [_coords(x) for x in trajs]
    outs = [np.zeros((x.shape[0], x.shape[0])) for x in xs]
    ptrs = (ctypes.POINTER(ctypes.c_double) * len(xs))(*[_dptr(m) for m in outs])
    o = _opts(device)
    _check(lib().gc_gcmi_batch(_views(xs), len(xs), ctypes.byref(o), ptrs))
    return outs


def corr_batch(trajs, ks, lags=(1, 5, 10), *, device: int = -1):
    """Every matrix of the batched workload: KSG MI, GCMI and TE at each lag.
    Returns {"ksg": [...], "gcmi": [...], "te": {lag: [...]}}."""
    out = {"ksg": ksg_batch(trajs, ks, device=device), "gcmi": gcmi_batch(trajs, device=device), "te": {}}
    for lag in lags:
        out["te"][int(lag)] = te_batch(trajs, ks, lag, device=device)
    return out


def batch_release() -> None:
    """Free the workspaces and graphs every batched entry point keeps."""
    lib().gc_ksg_batch_release()
    lib().gc_te_batch_release()
    lib().gc_gcmi_batch_release()


def ksg_batch_release() -> None:
    """Free the device workspace and graph the last ksg_batch kept."""
    lib().gc_ksg_batch_release()


def release_cache() -> None:
    """Free the device workspace kraskov_corrmatrix keeps between calls."""
    lib().gc_release_cache()


def gauss_corrmatrix(x, *, device: int = -1) -> np.ndarray:
    x = _coords(x)
    n = x.shape[0]
    out = np.zeros(n * n)
    v, o = _view(x), _opts(device)
    _check(lib().gc_gauss_matrix(ctypes.byref(v), ctypes.byref(o), _dptr(out)))
    return out.reshape(n, n)


def gcmi_corrmatrix(x, *, device: int = -1) -> np.ndarray:
    x = _coords(x)
    n = x.shape[0]
    out = np.zeros(n * n)
    v, o = _view(x), _opts(device)
    _check(lib().gc_gcmi_matrix(ctypes.byref(v), ctypes.byref(o), _dptr(out)))
    return out.reshape(n, n)


def te_matrix(x, k: int, lag: int = 1, *, path: int = PATH_AUTO, device: int = -1) -> np.ndarray:
    """te[a1, a2] = TE(a2 -> a1, lag); zero diagonal; zeros if nframes - lag <= k."""
    x = _coords(x)
    n = x.shape[0]
    out = np.zeros(n * n)
    v, o = _view(x), _opts(device, path)
    _check(lib().gc_te_matrix(ctypes.byref(v), int(k), int(lag), ctypes.byref(o), _dptr(out)))
    return out.reshape(n, n)


def kraskov_prepare(x, *, device: int = -1):
    """(X [3n, T], psi [T+1], scal [3n]) exactly as kraskov_prepare builds them."""
    x = _coords(x)
    n, T = x.shape[0], x.shape[1]
    X = np.zeros((3 * n, T))
    psi = np.zeros(T + 1)
    scal = np.zeros(3 * n)
    v, o = _view(x), _opts(device)
    _check(lib().gc_ksg_prepare(ctypes.byref(v), ctypes.byref(o), _dptr(X), _dptr(psi), _dptr(scal)))
    return X, psi, scal


def kraskov_corrmatrix_prepared(X, psi, k: int, *, path: int = PATH_AUTO, device: int = -1) -> np.ndarray:
    """KSG MI matrix from rows kraskov_prepare normalised (X [3n, T], psi
    [T+1]), as the reference's kraskov_corrmatrix_gpu(kr, natoms, mat, k)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    if X.ndim != 2 or X.shape[0] % 3 or psi.shape != (X.shape[1] + 1,):
        raise ValueError("X must be [3*natoms, nframes] and psi [nframes + 1]")
    n, T = X.shape[0] // 3, X.shape[1]
    out = np.zeros(n * n)
    o = _opts(device, path)
    _check(lib().gc_ksg_matrix_prepared(_dptr(X), _dptr(psi), n, T, int(k), ctypes.byref(o), _dptr(out)))
    return out.reshape(n, n)


def kraskov_wrap(X, psi, a1: int, a2: int, k: int, *, device: int = -1) -> float:
    """MI of one pair from prepared rows, as kraskov_wrap (a1's rows first)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    T = X.shape[1]
    rows = np.ascontiguousarray(np.concatenate([X[3 * a1:3 * a1 + 3], X[3 * a2:3 * a2 + 3]]))
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    mi = ctypes.c_double()
    o = _opts(device)
    _check(lib().gc_ksg_pair(_dptr(rows), T, int(k), _dptr(psi), ctypes.byref(o), ctypes.byref(mi)))
    return mi.value


def pearsify(mat: np.ndarray, dim: int = 3) -> np.ndarray:
    """In-place r(MI) conversion (returns ``mat``)."""
    if not (isinstance(mat, np.ndarray) and mat.dtype == np.float64 and mat.flags.c_contiguous):
        raise ValueError("pearsify needs a C-contiguous float64 array")
    lib().gc_pearsify(_dptr(mat), int(mat.shape[0]), int(dim))
    return mat


def write_matrix(mat: np.ndarray, path) -> None:
    m = np.ascontiguousarray(mat, dtype=np.float64)
    _check(lib().gc_write_matrix(_dptr(m), m.shape[0], str(path).encode()))


def write_xpm_matrix(mat: np.ndarray, path, title: str = "", legend: str = "") -> None:
    m = np.ascontiguousarray(mat, dtype=np.float64)
    _check(lib().gc_write_xpm(_dptr(m), m.shape[0], str(path).encode(), title.encode(), legend.encode()))


def read_matrix(path) -> np.ndarray:
    """Parse a correl.dat file (the consumer's reading of the format:
    optional `N x M [ ... ]` wrapper, values written column-major)."""
    raw = Path(path).read_text()
    inner = raw[raw.index("[") + 1: raw.rindex("]")] if "[" in raw else raw
    vals = [float(v) for v in inner.split() if v not in ("{", "}")]
    n = int(round(len(vals) ** 0.5))
    if n * n != len(vals):
        raise ValueError(f"{len(vals)} values do not form a square matrix")
    return np.array(vals).reshape(n, n).T


def ksg_pair_mi_noalloc(d_xyz: int, natoms: int, nframes: int, k: int, d_pair_mi: int,
                        stream: int = 0) -> None:
    """Pair MI into caller-owned device memory with no device allocation
    (natoms <= 64, nframes <= 1024); pointers are raw device addresses."""
    _check(lib().gc_ksg_pair_mi_noalloc(ctypes.c_void_p(d_xyz), int(natoms), int(nframes), int(k),
                                        ctypes.c_void_p(d_pair_mi), ctypes.c_void_p(stream or 0)))


class TePlan:
    """Device-resident transfer-entropy plan (one natoms x nframes, k, lag shape)."""

    def __init__(self, natoms: int, nframes: int, k: int, lag: int = 1, *, device: int = -1,
                 path: int = PATH_AUTO):
        self._h = ctypes.c_void_p()
        o = _opts(device, path)
        _check(lib().gc_te_plan_create(natoms, nframes, k, lag, ctypes.byref(o), ctypes.byref(self._h)))
        self.natoms, self.nframes, self.k, self.lag = natoms, nframes, k, lag

    def run(self, d_xyz: int, d_te: int, stream: int | None = None) -> None:
        """Enqueue one TE matrix (natoms x natoms doubles at d_te)."""
        _check(lib().gc_te_plan_run(self._h, ctypes.c_void_p(d_xyz), ctypes.c_void_p(d_te),
                                    ctypes.c_void_p(stream or 0)))

    def sync(self) -> None:
        _check(lib().gc_te_plan_sync(self._h))

    def counts(self, a1: int, a2: int):
        """(n_xp, n_xfxp, n_ypxp) per query of TE(a2 -> a1) from the last run."""
        nv = self.nframes - self.lag
        out = [np.zeros(nv, np.int32) for _ in range(3)]
        ip = ctypes.POINTER(ctypes.c_int32)
        _check(lib().gc_te_plan_counts(self._h, int(a1), int(a2), *[o.ctypes.data_as(ip) for o in out]))
        return tuple(out)

    pairs = property(lambda self: int(lib().gc_te_plan_pairs(self._h)))
    launches = property(lambda self: int(lib().gc_te_plan_launches(self._h)))
    is_walk = property(lambda self: bool(lib().gc_te_plan_is_walk(self._h)))
    handoffs = property(lambda self: int(lib().gc_te_plan_handoffs(self._h)))
    walk_mean = property(lambda self: float(lib().gc_te_plan_walk_mean(self._h)))
    kernel_ms = property(lambda self: float(lib().gc_te_plan_kernel_ms(self._h)))

    def close(self) -> None:
        if self._h:
            lib().gc_te_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KsgPlan:
    """Device-resident KSG plan: inputs already in HBM, nothing allocated per run."""

    def __init__(self, natoms: int, nframes: int, k: int, *, device: int = -1, pairs=None,
                 path: int = PATH_AUTO, pair_list=None, variant: int = VARIANT_DEFAULT):
        self._h = ctypes.c_void_p()
        o = _opts(device, path, pairs, pair_list=pair_list, variant=variant)
        _check(lib().gc_ksg_plan_create(natoms, nframes, k, ctypes.byref(o), ctypes.byref(self._h)))
        self.natoms, self.nframes, self.k = natoms, nframes, k

    @property
    def pairs(self) -> int:
        return int(lib().gc_ksg_plan_pairs(self._h))

    @property
    def launches(self) -> int:
        return int(lib().gc_ksg_plan_launches(self._h))

    def run(self, d_xyz: int, d_pair_mi: int, stream: int | None = None) -> None:
        """Enqueue one full KSG pass; pointers are raw device addresses."""
        _check(lib().gc_ksg_plan_run(self._h, ctypes.c_void_p(d_xyz), ctypes.c_void_p(d_pair_mi),
                                     ctypes.c_void_p(stream or 0)))

    def sync(self) -> None:
        _check(lib().gc_ksg_plan_sync(self._h))

    @property
    def handoffs(self) -> int:
        """Queries of the last run computed by the exact hand-over kernel."""
        return int(lib().gc_ksg_plan_handoffs(self._h))

    @property
    def handoff_reasons(self) -> dict:
        """Hand-overs of the last run by cause."""
        names = {2: "kth_outside_histogram", 3: "band_too_wide", 4: "ambiguous_set",
                 5: "maxima_scan_too_long", 6: "count_band_outside_walk"}
        return {v: int(lib().gc_ksg_plan_handoff_reason(self._h, k)) for k, v in names.items()}

    @property
    def walk_mean(self) -> float:
        """Mean sorted-row entries walked per query in the last run."""
        return float(lib().gc_ksg_plan_walk_mean(self._h))

    @property
    def is_fast(self) -> bool:
        return bool(lib().gc_ksg_plan_is_fast(self._h))

    @property
    def kernel_ms(self) -> float:
        """Device time of the neighbour kernel(s) of the last completed run."""
        return float(lib().gc_ksg_plan_kernel_ms(self._h))

    def close(self) -> None:
        if self._h:
            lib().gc_ksg_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _f32(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def screen_features(x, k: int, *, pca=None, pair_list=None, pairs=None, device: int = -1) -> np.ndarray:
    """Feature rows of the learned screen for the selected pairs.

    ``pca=(mean[64], comp[17][64])`` gives (npairs, 40) rows; without it the
    rows hold the 64 raw histogram cells, (npairs, 87).
    """
    x = _coords(x)
    n = x.shape[0]
    npairs = n * (n - 1) // 2
    if pair_list is not None:
        cnt = len(pair_list)
    elif pairs is not None:
        cnt = (pairs[1] if pairs[1] > 0 else npairs) - pairs[0]
    else:
        cnt = npairs
    width = SCREEN_IN if pca is not None else SCREEN_RAW
    out = np.zeros((max(cnt, 0), width), np.float32)
    o = _opts(device, PATH_AUTO, pairs, pair_list=pair_list)
    v = _view(x)
    if pca is not None:
        pm, pc = _f32(pca[0], (64,)), _f32(pca[1], (SCREEN_COMP, 64))
        _check(lib().gc_screen_features(ctypes.byref(v), int(k), ctypes.byref(o), _fptr(pm), _fptr(pc), _fptr(out)))
    else:
        _check(lib().gc_screen_features(ctypes.byref(v), int(k), ctypes.byref(o), None, None, _fptr(out)))
    return out


class ScreenModel:
    """Device-resident ensemble of the screen's BF16 networks."""

    def __init__(self, members: int = 4, seed: int = 0, device: int = -1):
        self._h = ctypes.c_void_p()
        _check(lib().gc_screen_model_create(int(members), int(seed), int(device), ctypes.byref(self._h)))
        self.members = members
        self.stride = int(lib().gc_screen_param_stride())
        self.sigma_max = 0.0
        self.margin = 0.0

    def get_params(self) -> np.ndarray:
        out = np.zeros((self.members, self.stride), np.float32)
        _check(lib().gc_screen_model_get_params(self._h, _fptr(out)))
        return out

    def set_params(self, params) -> None:
        p = _f32(params, (self.members, self.stride))
        _check(lib().gc_screen_model_set_params(self._h, _fptr(p)))

    def set_input(self, feat_mean, feat_sd, pca_mean, pca_comp) -> None:
        fm, fs = _f32(feat_mean, (SCREEN_IN,)), _f32(feat_sd, (SCREEN_IN,))
        pm, pc = _f32(pca_mean, (64,)), _f32(pca_comp, (SCREEN_COMP, 64))
        self._input = (fm, fs, pm, pc)
        _check(lib().gc_screen_model_set_input(self._h, _fptr(fm), _fptr(fs), _fptr(pm), _fptr(pc)))

    def train(self, feats, target, *, epochs: int = 20, batch: int = 1024, lr: float = 2e-3,
              seed: int = 0) -> np.ndarray:
        """Adam on the mean squared error; returns the per-epoch mean loss."""
        F = _f32(feats)
        t = _f32(target)
        if F.ndim != 2 or F.shape[1] != SCREEN_IN or t.shape != (F.shape[0],):
            raise ValueError("feats must be (n, 40) and target (n,)")
        loss = np.zeros(epochs, np.float32)
        _check(lib().gc_screen_train(self._h, _fptr(F), _fptr(t), F.shape[0], int(epochs), int(batch),
                                     float(lr), int(seed), _fptr(loss)))
        return loss

    def grad(self, feats, target):
        """(grad (members, stride), loss (members,)) of one full-batch pass."""
        F = _f32(feats)
        t = _f32(target)
        g = np.zeros((self.members, self.stride), np.float32)
        loss = np.zeros(self.members, np.float32)
        _check(lib().gc_screen_grad(self._h, _fptr(F), _fptr(t), F.shape[0], _fptr(g), _fptr(loss)))
        return g, loss

    def predict(self, feats) -> np.ndarray:
        """Prediction of every member, shape (members, n)."""
        F = _f32(feats)
        out = np.zeros((self.members, F.shape[0]), np.float32)
        _check(lib().gc_screen_predict(self._h, _fptr(F), F.shape[0], _fptr(out)))
        return out

    def close(self) -> None:
        if self._h:
            lib().gc_screen_model_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ksg_screened(x, k: int, model: ScreenModel, *, audit_frac: float = 0.05, sigma_max=None, margin=None,
                 seed: int = 12345, device: int = -1, path: int = PATH_AUTO, stream=None):
    """Screened KSG r(MI) matrix and its report (a dict).

    Exact KSG runs on the pairs whose ensemble spread exceeds ``sigma_max``
    or whose prediction lies within ``margin`` of the reported threshold,
    and on a random ``audit_frac`` sample; the rest keep the prediction.
    ``sigma_max`` / ``margin`` default to the model's calibrated values.
    """
    x = _coords(x)
    n = x.shape[0]
    so = _ScreenOpts()
    lib().gc_screen_opts_init(ctypes.byref(so))
    so.audit_frac = float(audit_frac)
    so.sigma_max = float(model.sigma_max if sigma_max is None else sigma_max)
    so.margin = float(model.margin if margin is None else margin)
    so.seed = int(seed)
    rep = _ScreenReport()
    out = np.zeros(n * n)
    o = _opts(device, path, stream=stream)
    v = _view(x)
    _check(lib().gc_ksg_screened(ctypes.byref(v), int(k), model._h, ctypes.byref(so), ctypes.byref(o),
                                 _dptr(out), ctypes.byref(rep)))
    report = {f: getattr(rep, f) for f, _ in _ScreenReport._fields_}
    return out.reshape(n, n), report


from .trajio import parse_atoms, read_index, read_trajectory, trajectory_info, write_trajectory  # noqa: E402
