"""Trajectory ingest (host only): XTC / TRR / dump reading, selection, frame
window and centring, index files, and the CLI's use of them.

The native reader (csrc/trajio.cpp) is checked against oracle/xtc.py, an
independent pure-Python restatement of the format, and against TRR and short
XTC frames built byte by byte here.  GROMACS is absent, so no file written by
GROMACS pins it (parity with GROMACS' own reader is unpinned).
"""
import math
import zlib
import struct
import subprocess

import numpy as np
import pytest

from oracle import xtc as ox
from tests.conftest import ROOT

trajio = pytest.importorskip("gmx_correlation_b200.trajio")
CLI = ROOT / "gmx_correlation_b200" / "gmx_correlation_b200"


def _atom_major(frames):
    return np.ascontiguousarray(np.asarray(frames).transpose(1, 0, 2)).astype(np.float64)


def _waterish(rng, n, spread=0.05, lo=-2.0, hi=8.0):
    m = (n + 2) // 3
    base = rng.uniform(lo, hi, (m, 1, 3))
    return (base + rng.normal(0, spread, (m, 3, 3))).reshape(-1, 3)[:n]


def _trr_frame(natoms, step, t, box, x, v=None, real=4):
    fmt = ">f" if real == 4 else ">d"
    out = struct.pack(">iii", 1993, 13, 12) + b"GMX_trn_file"
    xs = natoms * 3 * real
    vs = xs if v is not None else 0
    out += struct.pack(">11i", 0, 0, 9 * real, 0, 0, 0, 0, xs, vs, 0, natoms)
    out += struct.pack(">ii", step, 0) + struct.pack(fmt, t) + struct.pack(fmt, 0.0)
    out += b"".join(struct.pack(fmt, float(b)) for b in np.ravel(box))
    out += b"".join(struct.pack(fmt, float(c)) for c in np.ravel(x))
    if v is not None:
        out += b"".join(struct.pack(fmt, float(c)) for c in np.ravel(v))
    return out


def test_magic_table_is_the_cube_root_ladder():
    # every entry is floor(8 * 2^((i - 9) / 3)) except three long-standing
    # entries of the format's table
    quirks = {37: 5060, 57: 524287, 69: 8388607}
    for i in range(9, len(ox.MAGIC)):
        want = quirks.get(i, math.floor(8 * 2 ** ((i - 9) / 3) + 1e-9))
        assert ox.MAGIC[i] == want, i
    assert len(ox.MAGIC) == 73 and ox.MAGIC[-1] == 2 ** 24


def test_trr_float_handbuilt(tmp_path):
    rng = np.random.default_rng(0)
    x = rng.normal(0, 2, (3, 5, 3)).astype(np.float32)
    v = rng.normal(0, 1, (3, 5, 3)).astype(np.float32)
    p = tmp_path / "h.trr"
    p.write_bytes(b"".join(_trr_frame(5, i, 0.5 * i, np.eye(3) * 4, x[i], v[i]) for i in range(3)))
    assert trajio.trajectory_info(p) == {"format": "trr", "natoms": 5, "nframes": 3}
    got = trajio.read_trajectory(p, center=False)
    np.testing.assert_array_equal(got, _atom_major(x))
    np.testing.assert_array_equal(got, _atom_major([f[3] for f in ox.read_trr(p)]))


def test_trr_double_handbuilt(tmp_path):
    rng = np.random.default_rng(1)
    x = rng.normal(0, 2, (2, 4, 3))
    p = tmp_path / "d.trr"
    p.write_bytes(b"".join(_trr_frame(4, i, float(i), np.zeros((3, 3)), x[i], real=8) for i in range(2)))
    # a mixed-precision reader rounds to float; keep_double keeps the file's values
    np.testing.assert_array_equal(trajio.read_trajectory(p, center=False),
                                  _atom_major(x.astype(np.float32)))
    np.testing.assert_array_equal(trajio.read_trajectory(p, center=False, keep_double=True), _atom_major(x))
    q = tmp_path / "w.trr"
    trajio.write_trajectory(q, x, double=True)
    np.testing.assert_array_equal(trajio.read_trajectory(q, center=False, keep_double=True),
                                  _atom_major(x.astype(np.float32)))


def test_xtc_short_frame_handbuilt(tmp_path):
    # up to 9 atoms an XTC frame holds plain floats after the atom count
    x = np.arange(27, dtype=np.float32).reshape(9, 3) * np.float32(0.37)
    body = struct.pack(">iiif", 1995, 9, 7, 1.5) + struct.pack(">9f", *np.eye(3).ravel()) + struct.pack(">i", 9)
    body += struct.pack(">27f", *x.ravel())
    p = tmp_path / "s.xtc"
    p.write_bytes(body * 2)
    got = trajio.read_trajectory(p, center=False)
    np.testing.assert_array_equal(got, _atom_major([x, x]))


@pytest.mark.parametrize("case", ["water", "spread", "large_range", "prec100", "prec1e6", "tiny", "one_frame"])
def test_xtc_native_equals_oracle(tmp_path, case):
    rng = np.random.default_rng(zlib.crc32(case.encode()))
    prec, T = 1000.0, 3
    if case == "water":
        x = _waterish(rng, 600)
    elif case == "spread":
        x = rng.uniform(-30, 30, (257, 3))
    elif case == "large_range":  # integer ranges above 2^24: per-coordinate bit fields
        x = rng.uniform(-2e4, 2e4, (40, 3))
    elif case == "prec100":
        x, prec = _waterish(rng, 200, 0.2), 100.0
    elif case == "prec1e6":
        x, prec = _waterish(rng, 120, 0.02), 1e6
    elif case == "tiny":
        x = _waterish(rng, 10)
    else:
        x, T = _waterish(rng, 99), 1
    frames = np.stack([x + rng.normal(0, 0.003 * (t + 1), x.shape) for t in range(T)]).astype(np.float32)
    p = tmp_path / f"{case}.xtc"
    trajio.write_trajectory(p, frames, precision=prec, times=np.arange(T) * 0.25)
    ref = ox.read_xtc(p)
    assert [f[0] for f in ref] == list(range(T)) and [f[1] for f in ref] == [0.25 * t for t in range(T)]
    got = trajio.read_trajectory(p, center=False)
    np.testing.assert_array_equal(got, _atom_major([f[3] for f in ref]))
    # the stored integers are the writer's float rounding of x * precision
    f = frames * np.float32(prec)
    q = np.where(f >= 0, f + np.float32(0.5), f - np.float32(0.5)).astype(np.float32).astype(np.int64)
    np.testing.assert_array_equal(got, _atom_major((q.astype(np.float32) * np.float32(1.0 / prec))))


def test_xtc_small_index_sweep(tmp_path):
    # pairs of atoms at distances from 1e-4 to 5 nm walk the small-word index
    # over most of the range table, in both directions
    rng = np.random.default_rng(7)
    rows = []
    for d in np.geomspace(1e-4, 5.0, 60):
        c = rng.uniform(0, 50, 3)
        rows += [c, c + d * rng.uniform(-1, 1, 3), c + d * rng.uniform(-1, 1, 3)]
    x = np.array(rows)
    frames = np.stack([x, x[::-1].copy(), rng.permutation(x)]).astype(np.float32)
    for prec in (1000.0, 1e5):
        p = tmp_path / f"sweep{int(prec)}.xtc"
        trajio.write_trajectory(p, frames, precision=prec)
        np.testing.assert_array_equal(trajio.read_trajectory(p, center=False),
                                      _atom_major([f[3] for f in ox.read_xtc(p)]))
    # one frame per scale: triplets of atoms d apart, triplets far apart, so
    # the runs of every frame use the table entry the scale selects (d from
    # 10 to 2^23 stored units covers every entry)
    frames = []
    for d in np.geomspace(10, 2 ** 23, 64) / 1000.0:
        c = np.arange(30)[:, None] * (4.0 * d) + rng.uniform(0, d, (30, 3))
        trip = c[:, None, :] + rng.uniform(0, d / 3, (30, 3, 3))
        frames.append(trip.reshape(90, 3))
    frames = np.array(frames, np.float32)
    p = tmp_path / "scales.xtc"
    trajio.write_trajectory(p, frames, precision=1000.0)
    seen = set()
    ints = ox._Bits.ints

    def spy(self, nbits, sizes):
        if sizes[0] == sizes[1] == sizes[2] and nbits >= 9 and ox.MAGIC[nbits] == sizes[0]:
            seen.add(nbits)
        return ints(self, nbits, sizes)

    ox._Bits.ints = spy
    try:
        ref = ox.read_xtc(p)
    finally:
        ox._Bits.ints = ints
    np.testing.assert_array_equal(trajio.read_trajectory(p, center=False), _atom_major([f[3] for f in ref]))
    assert len(seen) >= 55, sorted(seen)


def test_trr_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    frames = rng.normal(0, 3, (4, 33, 3)).astype(np.float32)
    p = tmp_path / "r.trr"
    trajio.write_trajectory(p, frames, box=np.tile(np.eye(3) * 5, (4, 1, 1)))
    np.testing.assert_array_equal(trajio.read_trajectory(p, center=False), _atom_major(frames))


def test_selection_window_skip_and_centring(tmp_path):
    rng = np.random.default_rng(4)
    T = 23
    frames = np.stack([_waterish(rng, 60) for _ in range(T)]).astype(np.float32)
    times = np.arange(T) * 2.0
    p = tmp_path / "sel.xtc"
    trajio.write_trajectory(p, frames, times=times)
    full = _atom_major([f[3] for f in ox.read_xtc(p)])
    atoms = np.array([5, 0, 59, 17, 17])  # output order and repeats as given
    got = trajio.read_trajectory(p, atoms, skip=3, begin=5.0, end=38.0, center=True)
    keep = np.flatnonzero((times >= 5.0) & (times <= 38.0))[::3]  # frnr counts frames inside the window
    want = ox.center(full[atoms][:, keep])
    np.testing.assert_array_equal(got, want)
    # the centring is the reference's frame-order sum, not numpy's pairwise sum
    assert got.shape == (5, keep.size, 3)


def test_dump_input(tmp_path):
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, (4, 7, 3))
    p = tmp_path / "traj_dump.txt"
    with open(p, "w") as f:
        f.write("4 7\n")
        for t in range(7):
            for a in range(4):
                f.write("%.10g %.10g %.10g\n" % tuple(x[a, t]))
    assert trajio.trajectory_info(p)["format"] == "dump"
    want = np.array([[[float("%.10g" % v) for v in x[a, t]] for t in range(7)] for a in range(4)])
    np.testing.assert_array_equal(trajio.read_trajectory(p, center=False), want)


def test_errors(tmp_path, gc):
    rng = np.random.default_rng(6)
    frames = np.stack([_waterish(rng, 30) for _ in range(3)]).astype(np.float32)
    p = tmp_path / "e.xtc"
    trajio.write_trajectory(p, frames)
    data = p.read_bytes()
    cut = tmp_path / "cut.xtc"
    cut.write_bytes(data[:-7])
    with pytest.raises(gc.GCError, match="frame 2"):
        trajio.read_trajectory(cut)
    with pytest.raises(gc.GCError, match="outside"):
        trajio.read_trajectory(p, [30])
    other = tmp_path / "o.xtc"
    trajio.write_trajectory(other, frames[:, :20])
    mixed = tmp_path / "mixed.xtc"
    mixed.write_bytes(data + other.read_bytes())
    with pytest.raises(gc.GCError, match="atom count changes"):
        trajio.read_trajectory(mixed)
    with pytest.raises(gc.GCError, match="No trajectory frames"):
        trajio.read_trajectory(p, begin=100.0)
    with pytest.raises(gc.GCError, match="skip"):
        trajio.read_trajectory(p, skip=0)
    junk = tmp_path / "junk.bin"
    junk.write_bytes(b"\x00\x01garbage")
    with pytest.raises(gc.GCError, match="not an XTC, TRR or dump"):
        trajio.read_trajectory(junk)
    with pytest.raises(gc.GCError, match="cannot open"):
        trajio.read_trajectory(tmp_path / "missing.xtc")


def test_index_and_atom_lists(tmp_path):
    ndx = tmp_path / "index.ndx"
    ndx.write_text("[ System ]\n1 2 3 4\n5 6\n[ C-alpha ] ; comment\n 2  4\n\n6\n[ empty ]\n")
    g = trajio.read_index(ndx)
    assert list(g) == ["System", "C-alpha", "empty"]
    np.testing.assert_array_equal(g["C-alpha"], [1, 3, 5])
    np.testing.assert_array_equal(trajio.parse_atoms("1-3 7,9"), [0, 1, 2, 6, 8])
    with pytest.raises(ValueError):
        trajio.parse_atoms("3-1")


def _read_dump(path):
    with open(path) as f:
        n, T = map(int, f.readline().split())
        v = np.loadtxt(f, ndmin=2).reshape(T, n, 3)
    return np.ascontiguousarray(v.transpose(1, 0, 2))


def _cli(*args):
    # the coordinates are read and the dump written before any device work,
    # so this runs without a GPU (the estimator call afterwards may fail)
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True)


@pytest.mark.skipif(not CLI.exists(), reason="CLI not built")
def test_cli_reads_xtc_with_index_group(tmp_path):
    rng = np.random.default_rng(8)
    T = 40
    frames = np.stack([_waterish(rng, 50) for _ in range(T)]).astype(np.float32)
    p = tmp_path / "t.xtc"
    trajio.write_trajectory(p, frames, times=np.arange(T) * 10.0)
    ndx = tmp_path / "index.ndx"
    ndx.write_text("[ Protein ]\n" + " ".join(str(i) for i in range(1, 51)) + "\n[ CA ]\n3 9 12 40 41 50\n")
    dump = tmp_path / "dump.txt"
    _cli("-f", p, "-n", ndx, "-sel", "CA", "-b", 50, "-e", 300, "-skip", 2, "-k", 3, "-dump", dump,
         "-o", tmp_path / "c.dat")
    full = _atom_major([f[3] for f in ox.read_xtc(p)])
    times = np.arange(T) * 10.0
    keep = np.flatnonzero((times >= 50) & (times <= 300))[::2]
    want = ox.center(full[[2, 8, 11, 39, 40, 49]][:, keep])
    want_txt = "\n".join(" ".join("%.10g" % v for v in want[a, t]) for t in range(keep.size) for a in range(6))
    got_txt = dump.read_text().split("\n", 1)[1].strip()
    assert dump.read_text().split("\n", 1)[0] == f"6 {keep.size}"
    assert got_txt == want_txt
    # an atom-number list selects the same atoms
    dump2 = tmp_path / "dump2.txt"
    _cli("-f", p, "-sel", "3 9 12 40-41 50", "-b", 50, "-e", 300, "-skip", 2, "-k", 3, "-dump", dump2,
         "-o", tmp_path / "c.dat")
    assert dump2.read_text() == dump.read_text()


@pytest.mark.skipif(not CLI.exists(), reason="CLI not built")
def test_cli_selection_errors(tmp_path):
    frames = np.zeros((3, 12, 3), np.float32)
    p = tmp_path / "z.trr"
    trajio.write_trajectory(p, frames)
    ndx = tmp_path / "i.ndx"
    ndx.write_text("[ A ]\n1 2\n")
    r = _cli("-f", p, "-n", ndx, "-sel", "B")
    assert r.returncode != 0 and "no group 'B'" in r.stderr and "'A'" in r.stderr
    r = _cli("-f", p, "-sel", "1-20", "-k", 1)
    assert r.returncode != 0 and "outside" in r.stderr
    r = _cli("-f", p, "-sel", "x")
    assert r.returncode != 0 and "neither an index group" in r.stderr


def test_absurd_atom_counts_fail_without_allocating(tmp_path, gc):
    # a corrupt header announcing a billion atoms is rejected from the bytes
    # the file holds, before anything is allocated for them
    n = 1 << 30
    head = struct.pack(">iiif", 1995, n, 0, 0.0) + struct.pack(">9f", *np.eye(3).ravel()) + struct.pack(">i", n)
    body = struct.pack(">f6iii", 1000.0, 0, 0, 0, 1, 1, 1, 9, 8) + bytes(8)
    p = tmp_path / "huge.xtc"
    p.write_bytes(head + body)
    with pytest.raises(gc.GCError, match="more atoms or bytes"):
        trajio.read_trajectory(p)
    t = tmp_path / "huge.trr"
    t.write_bytes(struct.pack(">iii", 1993, 13, 12) + b"GMX_trn_file" +
                  struct.pack(">11i", 0, 0, 0, 0, 0, 0, 0, (1 << 26) * 12, 0, 0, 1 << 26) +
                  struct.pack(">iiff", 0, 0, 0.0, 0.0) + bytes(64))
    with pytest.raises(gc.GCError, match="truncated"):
        trajio.read_trajectory(t)
