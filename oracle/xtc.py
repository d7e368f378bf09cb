"""Test infrastructure: a pure-Python restatement of the XTC / TRR readers.

The oracle for the native trajectory ingest (gmx_correlation_b200/csrc/
trajio.cpp).  Only tests import it.  It decodes small files frame by frame
with plain Python integers, following the published xdrfile / GROMACS
"xdr3dfcoord" decoder structure (a byte-wise bit reader that keeps the count
of unread bits of the last byte, a byte-wise mixed-radix division) rather
than the native reader's 32-bit bit accumulator, so that the two only agree
when both follow the format.  GROMACS itself is absent here, so neither is
checked against files written by GROMACS: parity with GROMACS' reader is
unpinned; what is pinned is agreement of two independent restatements plus
hand-built TRR and short-XTC frames in the tests.

The reference reads frames through GROMACS (src/gmx_correlation.cpp:158-182)
and centres them in finishAnalysis (:184-223); ``center`` restates the latter.
"""

from __future__ import annotations

import struct

import numpy as np

# Ranges of the small-difference words (about 2^(i/3)); part of the format.
MAGIC = [0] * 9 + [
    8, 10, 12, 16, 20, 25, 32, 40, 50, 64, 80, 101, 128, 161, 203, 256, 322, 406, 512, 645, 812, 1024, 1290, 1625,
    2048, 2580, 3250, 4096, 5060, 6501, 8192, 10321, 13003, 16384, 20642, 26007, 32768, 41285, 52015, 65536,
    82570, 104031, 131072, 165140, 208063, 262144, 330280, 416127, 524287, 660561, 832255, 1048576, 1321122,
    1664510, 2097152, 2642245, 3329021, 4194304, 5284491, 6658042, 8388607, 10568983, 13316085, 16777216]
FIRSTIDX = 9


class _Bits:
    """The format's bit reader: a byte counter, the unread bit count of the
    last byte read and that byte history."""

    def __init__(self, data: bytes):
        self.data, self.cnt, self.lastbits, self.lastbyte = data, 0, 0, 0

    def bits(self, nbits: int) -> int:
        mask = (1 << nbits) - 1
        num = 0
        while nbits >= 8:
            self.lastbyte = ((self.lastbyte << 8) | self.data[self.cnt]) & 0xFFFFFFFF
            self.cnt += 1
            num |= (self.lastbyte >> self.lastbits) << (nbits - 8)
            nbits -= 8
        if nbits > 0:
            if self.lastbits < nbits:
                self.lastbits += 8
                self.lastbyte = ((self.lastbyte << 8) | self.data[self.cnt]) & 0xFFFFFFFF
                self.cnt += 1
            self.lastbits -= nbits
            num |= (self.lastbyte >> self.lastbits) & ((1 << nbits) - 1)
        return num & mask

    def ints(self, nbits: int, sizes) -> list:
        by = []
        while nbits > 8:
            by.append(self.bits(8))
            nbits -= 8
        if nbits > 0:
            by.append(self.bits(nbits))
        by += [0] * max(0, 4 - len(by))
        out = [0, 0, 0]
        for i in (2, 1):
            num = 0
            for j in range(len(by) - 1, -1, -1):
                num = (num << 8) | by[j]
                p = num // sizes[i]
                by[j] = p
                num -= p * sizes[i]
            out[i] = num
        out[0] = by[0] | (by[1] << 8) | (by[2] << 16) | (by[3] << 24)
        return out


def _sizeofint(size: int) -> int:
    n, num = 0, 1
    while size >= num and n < 32:
        n += 1
        num <<= 1
    return n


def _sizeofints(sizes) -> int:
    total = sizes[0] * sizes[1] * sizes[2]
    return max(1, total.bit_length()) if total > 1 else 1


class _Stream:
    def __init__(self, data: bytes):
        self.d, self.p = data, 0

    def left(self) -> int:
        return len(self.d) - self.p

    def i32(self) -> int:
        v = struct.unpack_from(">i", self.d, self.p)[0]
        self.p += 4
        return v

    def f32(self) -> float:
        v = struct.unpack_from(">f", self.d, self.p)[0]
        self.p += 4
        return v

    def f64(self) -> float:
        v = struct.unpack_from(">d", self.d, self.p)[0]
        self.p += 8
        return v

    def opaque(self, n: int) -> bytes:
        v = self.d[self.p:self.p + n]
        self.p += n + (4 - n % 4) % 4
        return v


def _xtc_coords(s: _Stream, natoms: int) -> np.ndarray:
    lsize = s.i32()
    assert lsize == natoms
    if natoms <= 9:
        return np.array([s.f32() for _ in range(3 * natoms)], dtype=np.float32).reshape(natoms, 3)
    precision = np.float32(s.f32())
    minint = [s.i32() for _ in range(3)]
    maxint = [s.i32() for _ in range(3)]
    sizeint = [maxint[d] - minint[d] + 1 for d in range(3)]
    if any(v > 0xFFFFFF for v in sizeint):
        bitsizeint, bitsize = [_sizeofint(v) for v in sizeint], 0
    else:
        bitsizeint, bitsize = None, _sizeofints(sizeint)
    smallidx = s.i32()
    smaller = MAGIC[max(FIRSTIDX, smallidx - 1)] // 2
    smallnum = MAGIC[smallidx] // 2
    sizesmall = [MAGIC[smallidx]] * 3
    nbytes = s.i32()
    b = _Bits(s.opaque(nbytes))
    inv = np.float32(1.0 / float(precision))
    out = []
    i, run = 0, 0
    while i < natoms:
        if bitsize == 0:
            cur = [b.bits(bitsizeint[d]) for d in range(3)]
        else:
            cur = b.ints(bitsize, sizeint)
        i += 1
        cur = [cur[d] + minint[d] for d in range(3)]
        prev = list(cur)
        is_smaller = 0
        if b.bits(1) == 1:
            run = b.bits(5)
            is_smaller = run % 3
            run -= is_smaller
            is_smaller -= 1
        if run > 0:
            for k in range(0, run, 3):
                c = b.ints(smallidx, sizesmall)
                i += 1
                c = [c[d] + prev[d] - smallnum for d in range(3)]
                if k == 0:
                    c, prev = prev, c
                    out.append(prev)
                else:
                    prev = list(c)
                out.append(c)
        else:
            out.append(cur)
        smallidx += is_smaller
        if is_smaller < 0:
            smallnum = smaller
            smaller = MAGIC[smallidx - 1] // 2 if smallidx > FIRSTIDX else 0
        elif is_smaller > 0:
            smaller = smallnum
            smallnum = MAGIC[smallidx] // 2
        sizesmall = [MAGIC[smallidx]] * 3
    q = np.array(out, dtype=np.int64).reshape(natoms, 3)
    return (q.astype(np.float32) * inv).astype(np.float32)


def read_xtc(path) -> list:
    """Frames of an XTC file as (step, time, box (3x3), positions (natoms, 3) float32)."""
    s = _Stream(open(path, "rb").read())
    frames = []
    while s.left() > 0:
        assert s.i32() == 1995
        natoms, step, t = s.i32(), s.i32(), s.f32()
        box = np.array([s.f32() for _ in range(9)], dtype=np.float32).reshape(3, 3)
        frames.append((step, t, box, _xtc_coords(s, natoms)))
    return frames


def read_trr(path) -> list:
    """Frames of a TRR file as (step, time, box, positions float32 or float64)."""
    s = _Stream(open(path, "rb").read())
    frames = []
    while s.left() > 0:
        assert s.i32() == 1993
        assert s.i32() == 13
        n = s.i32()
        assert s.opaque(n) == b"GMX_trn_file"
        ir, e, box, vir, pres, top, sym, xs, vs, fs, natoms = (s.i32() for _ in range(11))
        real = box // 9 if box else xs // (natoms * 3)
        step, _nre = s.i32(), s.i32()
        rd = s.f32 if real == 4 else s.f64
        t, _lam = rd(), rd()
        dt = np.float32 if real == 4 else np.float64
        b = np.array([rd() for _ in range(box // real)], dtype=dt).reshape(-1, 3) if box else None
        for size in (vir, pres):
            s.p += size
        x = np.array([rd() for _ in range(xs // real)], dtype=dt).reshape(natoms, 3)
        s.p += vs + fs
        frames.append((step, t, b, x))
    return frames


def center(x: np.ndarray) -> np.ndarray:
    """The reference's centring (src/gmx_correlation.cpp:195-223): per atom the
    mean over frames summed in frame order, subtracted.  x: (natoms, nframes, 3)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    for a in range(x.shape[0]):
        for d in range(3):
            col = x[a, :, d]
            av = 0.0
            for v in col:
                av += float(v)
            av /= col.size
            out[a, :, d] = col - av
    return out
