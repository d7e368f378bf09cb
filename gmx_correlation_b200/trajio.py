"""Trajectory ingest: GROMACS XTC / TRR files, the -dump text file, index groups.

Replaces the reference module's frame collection (src/gmx_correlation.cpp:
158-182, a static atom selection and every skip-th analysed frame; :184-223,
the per-atom mean subtracted), which reads frames through GROMACS.  The
decoding runs in the native library (``gc_traj_read``); this module binds it
and reads GROMACS index files (``.ndx``) for the selection.

    x = read_trajectory("traj.xtc", atoms=read_index("index.ndx")["C-alpha"], center=True)
    mat = gmx_correlation_b200.kraskov_corrmatrix(x, 100)
"""

from __future__ import annotations

import ctypes
import re

import numpy as np

XTC, TRR, DUMP = 1, 2, 3
CENTER, KEEP_DOUBLE, BEGIN, END = 1, 2, 4, 8
_FORMATS = {"xtc": XTC, "trr": TRR}


class _Select(ctypes.Structure):
    _fields_ = [("atoms", ctypes.POINTER(ctypes.c_int)), ("natoms", ctypes.c_int), ("skip", ctypes.c_int),
                ("t_begin", ctypes.c_double), ("t_end", ctypes.c_double), ("flags", ctypes.c_int)]


_bound = False


def _lib():
    from . import lib

    global _bound
    L = lib()
    if not _bound:
        ip, dpp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.POINTER(ctypes.c_double))
        L.gc_traj_info.argtypes = [ctypes.c_char_p, ip, ip, ip]
        L.gc_traj_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Select), dpp, ip, ip]
        L.gc_traj_free.argtypes = [ctypes.POINTER(ctypes.c_double)]
        L.gc_traj_free.restype = None
        fp = ctypes.POINTER(ctypes.c_float)
        L.gc_traj_write.argtypes = [ctypes.c_char_p, ctypes.c_int, fp, ctypes.c_int, ctypes.c_int, fp,
                                    ctypes.POINTER(ctypes.c_double), ctypes.c_float, ctypes.c_int]
        _bound = True
    return L


def _check(status):
    from . import _check as check

    check(status)


def trajectory_info(path) -> dict:
    """Format ("xtc", "trr" or "dump"), atom count and frame count of a file."""
    L = _lib()
    fmt, n, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(L.gc_traj_info(str(path).encode(), ctypes.byref(fmt), ctypes.byref(n), ctypes.byref(t)))
    return {"format": {XTC: "xtc", TRR: "trr", DUMP: "dump"}[fmt.value], "natoms": n.value, "nframes": t.value}


def read_trajectory(path, atoms=None, *, skip: int = 1, begin: float | None = None, end: float | None = None,
                    center: bool = True, keep_double: bool = False) -> np.ndarray:
    """Positions (nm) of the selected atoms as a (natoms, nframes, 3) float64 array.

    ``atoms``: 0-based indices in output order (None: every atom); ``skip``:
    every skip-th frame of those with begin <= time <= end (ps), as the
    reference's -skip / -b / -e; ``center``: subtract each atom's mean over
    the kept frames, summed in frame order (the reference's finishAnalysis),
    so the result is what the reference hands to its estimators.
    """
    L = _lib()
    sel = _Select()
    arr = None
    if atoms is not None:
        arr = np.ascontiguousarray(np.asarray(atoms, dtype=np.int32).ravel())
        sel.atoms = arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        sel.natoms = int(arr.size)
        if arr.size == 0:
            raise ValueError("empty atom selection")
    sel.skip = int(skip)
    sel.flags = (CENTER if center else 0) | (KEEP_DOUBLE if keep_double else 0)
    if begin is not None:
        sel.t_begin, sel.flags = float(begin), sel.flags | BEGIN
    if end is not None:
        sel.t_end, sel.flags = float(end), sel.flags | END
    out = ctypes.POINTER(ctypes.c_double)()
    n, t = ctypes.c_int(), ctypes.c_int()
    _check(L.gc_traj_read(str(path).encode(), ctypes.byref(sel), ctypes.byref(out), ctypes.byref(n),
                          ctypes.byref(t)))
    try:
        x = np.ctypeslib.as_array(out, shape=(n.value, t.value, 3)).copy()
    finally:
        L.gc_traj_free(out)
    del arr
    return x


def write_trajectory(path, frames, *, fmt: str | None = None, box=None, times=None, precision: float = 1000.0,
                     double: bool = False) -> None:
    """Writes frames (nframes, natoms, 3) of positions (nm) as XTC or TRR.

    ``fmt``: "xtc" or "trr" (default: from the file suffix); ``box``: (nframes,
    3, 3) or None; ``times``: ps per frame or None (the frame index);
    ``precision``: XTC positions are stored as round(x * precision);
    ``double``: a double-precision TRR.
    """
    L = _lib()
    fmt = fmt or str(path).rsplit(".", 1)[-1].lower()
    if fmt not in _FORMATS:
        raise ValueError("format must be xtc or trr")
    x = np.ascontiguousarray(frames, dtype=np.float32)
    if x.ndim != 3 or x.shape[2] != 3:
        raise ValueError("frames must be (nframes, natoms, 3)")
    fp = ctypes.POINTER(ctypes.c_float)
    b = None if box is None else np.ascontiguousarray(box, dtype=np.float32).reshape(x.shape[0], 9)
    tm = None if times is None else np.ascontiguousarray(times, dtype=np.float64).reshape(x.shape[0])
    _check(L.gc_traj_write(str(path).encode(), _FORMATS[fmt], x.ctypes.data_as(fp), x.shape[1], x.shape[0],
                           None if b is None else b.ctypes.data_as(fp),
                           None if tm is None else tm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           float(precision), KEEP_DOUBLE if double else 0))


def read_index(path) -> dict:
    """Groups of a GROMACS index file as {name: 0-based atom indices}.

    The file holds ``[ name ]`` headers, each followed by 1-based atom numbers
    separated by white space over any number of lines.
    """
    groups, name = {}, None
    with open(path) as f:
        for line in f:
            s = line.split(";", 1)[0].strip()
            if not s:
                continue
            m = re.fullmatch(r"\[\s*(.*?)\s*\]", s)
            if m:
                name = m.group(1)
                groups.setdefault(name, [])
                continue
            if name is None:
                raise ValueError(f"{path}: atom numbers before the first [ group ] header")
            groups[name].extend(int(v) - 1 for v in s.split())
    return {k: np.asarray(v, dtype=np.int32) for k, v in groups.items()}


def parse_atoms(spec: str) -> np.ndarray:
    """0-based indices of an atom-number list such as "1-10 15 20-22" (1-based, inclusive)."""
    out = []
    for tok in spec.replace(",", " ").split():
        if "-" in tok:
            a, b = tok.split("-", 1)
            a, b = int(a), int(b)
            if a < 1 or b < a:
                raise ValueError(f"bad atom range {tok!r}")
            out.extend(range(a - 1, b))
        else:
            v = int(tok)
            if v < 1:
                raise ValueError(f"bad atom number {tok!r}")
            out.append(v - 1)
    if not out:
        raise ValueError("empty atom selection")
    return np.asarray(out, dtype=np.int32)
