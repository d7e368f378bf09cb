// Trajectory ingest: GROMACS XTC and TRR files and the -dump text file.
//
// Replaces the GROMACS front end's frame collection (src/gmx_correlation.cpp:
// 158-182 analyzeFrame, :184-223 the centring in finishAnalysis), which reads
// frames through GROMACS' trajectory library.  GROMACS is not a dependency
// here, so the two binary formats are decoded natively:
//
//  * XDR: every int, float and double big-endian in 4 / 8 bytes; opaque data
//    padded to a multiple of 4 bytes (RFC 4506).
//  * TRR (magic 1993): a header of XDR ints (version string "GMX_trn_file",
//    the byte sizes of box, virial, pressure, topology, symmetry, x, v and f
//    blocks, natoms, step, nre), time and lambda, then the blocks the sizes
//    announce.  Float or double precision follows from a block's size per
//    value.
//  * XTC (magic 1995): natoms, step, time, box (9 floats), natoms again, then
//    the compressed coordinates: up to 9 atoms as plain floats, otherwise the
//    precision, the integer bounding box, a starting "small" index and a bit
//    stream.  Positions are rounded to integers (x * precision); each atom is
//    either a full integer triple packed into the fewest bits that hold the
//    bounding box (a mixed-radix number over the three ranges) or, inside a
//    run, a small difference to the previous atom packed the same way over
//    the range of the current small index.  The first two atoms of a run are
//    stored swapped (water O-H ordering).  A 1-bit flag per full atom says
//    whether a 5-bit run word follows (run length * 3 + the change of the
//    small index + 1); without it the previous run length repeats.  The small
//    index selects ranges from a fixed table of integers close to
//    2^(i/3) (kMagic below), part of the format.
//
// The XTC codec follows that published format (the xdrfile/GROMACS
// "xdr3dfcoord" scheme); its output is float positions as GROMACS' mixed-
// precision build delivers them (integer x float(1 / precision)).  Double-
// precision TRR positions are rounded to float by default for the same reason
// (the reference module reads positions as GROMACS `real`).
//
// All frame filtering (time window, every skip-th frame) and the centring
// happen here; the result is the t_traj layout x[atom][frame][dim].

#include "gc_internal.h"
#include "gmx_corr_b200.h"
#include "host_common.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using gc::host::fail;

namespace {

// ---------------------------------------------------------------------------
// XDR primitives
// ---------------------------------------------------------------------------

struct File
{
    FILE* f = nullptr;
    explicit File(FILE* p) : f(p) {}
    ~File()
    {
        if (f)
            std::fclose(f);
    }
    File(const File&) = delete;
    File& operator=(const File&) = delete;
};

// Reads big-endian words; every call returns false at end of file or on a
// short read.
struct XdrIn
{
    FILE* f;

    // bytes from the read position to the end of the file
    long left() const
    {
        const long here = std::ftell(f);
        if (here < 0 || std::fseek(f, 0, SEEK_END) != 0)
            return 0;
        const long end = std::ftell(f);
        std::fseek(f, here, SEEK_SET);
        return end > here ? end - here : 0;
    }

    bool raw(void* p, size_t n) { return std::fread(p, 1, n, f) == n; }
    bool u32(uint32_t& v)
    {
        unsigned char b[4];
        if (!raw(b, 4))
            return false;
        v = (uint32_t)b[0] << 24 | (uint32_t)b[1] << 16 | (uint32_t)b[2] << 8 | (uint32_t)b[3];
        return true;
    }
    bool i32(int32_t& v)
    {
        uint32_t u;
        if (!u32(u))
            return false;
        std::memcpy(&v, &u, 4);
        return true;
    }
    bool f32(float& v)
    {
        uint32_t u;
        if (!u32(u))
            return false;
        std::memcpy(&v, &u, 4);
        return true;
    }
    bool f64(double& v)
    {
        uint32_t hi, lo;
        if (!u32(hi) || !u32(lo))
            return false;
        const uint64_t u = (uint64_t)hi << 32 | lo;
        std::memcpy(&v, &u, 8);
        return true;
    }
    // n big-endian 4-byte floats / 8-byte doubles in one read
    bool f32s(float* v, size_t n)
    {
        if (!raw(v, n * 4))
            return false;
        uint32_t* u = reinterpret_cast<uint32_t*>(v);
        for (size_t i = 0; i < n; ++i)
            u[i] = __builtin_bswap32(u[i]);
        return true;
    }
    bool f64s(double* v, size_t n)
    {
        if (!raw(v, n * 8))
            return false;
        uint64_t* u = reinterpret_cast<uint64_t*>(v);
        for (size_t i = 0; i < n; ++i)
            u[i] = __builtin_bswap64(u[i]);
        return true;
    }
    // n bytes of opaque data and the padding to a multiple of 4
    bool opaque(unsigned char* p, size_t n)
    {
        if (!raw(p, n))
            return false;
        unsigned char pad[4];
        const size_t  r = (4 - n % 4) % 4;
        return r == 0 || raw(pad, r);
    }
    bool skip(long n) { return n == 0 || std::fseek(f, n, SEEK_CUR) == 0; }
};

struct XdrOut
{
    FILE* f;
    bool  ok = true;

    void raw(const void* p, size_t n) { ok = ok && std::fwrite(p, 1, n, f) == n; }
    void u32(uint32_t v)
    {
        const unsigned char b[4] = {(unsigned char)(v >> 24), (unsigned char)(v >> 16), (unsigned char)(v >> 8),
                                    (unsigned char)v};
        raw(b, 4);
    }
    void i32(int32_t v)
    {
        uint32_t u;
        std::memcpy(&u, &v, 4);
        u32(u);
    }
    void f32(float v)
    {
        uint32_t u;
        std::memcpy(&u, &v, 4);
        u32(u);
    }
    void f64(double v)
    {
        uint64_t u;
        std::memcpy(&u, &v, 8);
        u32((uint32_t)(u >> 32));
        u32((uint32_t)u);
    }
    void opaque(const unsigned char* p, size_t n)
    {
        raw(p, n);
        const unsigned char pad[4] = {0, 0, 0, 0};
        raw(pad, (4 - n % 4) % 4);
    }
};

// One frame as read: positions of every atom in the file, frame-major.
struct Frame
{
    int                 natoms = 0;
    long long           step   = 0;
    double              time   = 0.0;
    std::vector<float>  xf; // float positions (XTC, float TRR, or rounded double TRR)
    std::vector<double> xd; // double positions (double TRR with keep_double, dump)
};

// ---------------------------------------------------------------------------
// XTC coordinate codec
// ---------------------------------------------------------------------------

constexpr int32_t kXtcMagic = 1995;
constexpr int32_t kTrrMagic = 1993;

// Ranges of the small-difference words: index i holds about 2^(i/3), so three
// differences of index i fit in i bits.  Indices below 9 are unused.
constexpr int kMagic[] = {0,       0,       0,       0,       0,        0,        0,        0,       0,
                          8,       10,      12,      16,      20,       25,       32,       40,      50,
                          64,      80,      101,     128,     161,      203,      256,      322,     406,
                          512,     645,     812,     1024,    1290,     1625,     2048,     2580,    3250,
                          4096,    5060,    6501,    8192,    10321,    13003,    16384,    20642,   26007,
                          32768,   41285,   52015,   65536,   82570,    104031,   131072,   165140,  208063,
                          262144,  330280,  416127,  524287,  660561,   832255,   1048576,  1321122, 1664510,
                          2097152, 2642245, 3329021, 4194304, 5284491,  6658042,  8388607,  10568983,
                          13316085, 16777216};
constexpr int kFirstIdx = 9;
constexpr int kLastIdx  = (int)(sizeof(kMagic) / sizeof(kMagic[0]));

// Bits needed for values 0 .. size - 1 ... as the format counts them: the
// number of doublings of 1 until it exceeds size.
int bits_of(unsigned size)
{
    int      n = 0;
    uint64_t v = 1;
    while (size >= v && n < 32)
    {
        ++n;
        v <<= 1;
    }
    return n;
}

// Bits of the mixed-radix number over three ranges (product of the sizes,
// little-endian bytes).
int bits_of3(const unsigned sizes[3])
{
    unsigned char bytes[32] = {1};
    int           nbytes    = 1;
    for (int i = 0; i < 3; ++i)
    {
        uint64_t t = 0;
        int      b = 0;
        for (; b < nbytes; ++b)
        {
            t        = (uint64_t)bytes[b] * sizes[i] + t;
            bytes[b] = (unsigned char)(t & 0xff);
            t >>= 8;
        }
        while (t != 0)
        {
            bytes[b++] = (unsigned char)(t & 0xff);
            t >>= 8;
        }
        nbytes = b;
    }
    int      bits = 0;
    unsigned top  = bytes[nbytes - 1];
    for (unsigned v = 1; top >= v; v <<= 1)
        ++bits;
    return bits + (nbytes - 1) * 8;
}

// MSB-first bit stream over the compressed bytes.
struct BitIn
{
    const unsigned char* p;
    size_t               n, pos = 0; // bytes, next byte
    uint64_t             acc  = 0;   // bits not consumed yet are the low `have` bits
    int                  have = 0;
    bool                 over = false;

    // the next nbits (0 .. 32) bits as an unsigned integer
    uint32_t get(int nbits)
    {
        while (have < nbits)
        {
            if (pos >= n)
            {
                over = true;
                return 0;
            }
            acc = (acc << 8) | p[pos++];
            have += 8;
        }
        have -= nbits;
        return (uint32_t)((acc >> have) & ((1ull << nbits) - 1ull));
    }
    // Three integers of a mixed-radix number of nbits bits: its bytes come
    // least significant first (the last one holds the remaining bits), the
    // number is ((v0 * s1) + v1) * s2 + v2.
    void get3(int nbits, const unsigned sizes[3], int out[3])
    {
        if (nbits <= 64)
        {
            uint64_t num = 0;
            int      sh = 0, rem = nbits;
            for (; rem > 8; rem -= 8, sh += 8)
                num |= (uint64_t)get(8) << sh;
            if (rem > 0)
                num |= (uint64_t)get(rem) << sh;
            out[2] = (int)(num % sizes[2]);
            num /= sizes[2];
            out[1] = (int)(num % sizes[1]);
            out[0] = (int)(uint32_t)(num / sizes[1]);
            return;
        }
        unsigned __int128 num = 0;
        int               sh = 0, rem = nbits;
        for (; rem > 8; rem -= 8, sh += 8)
            num |= (unsigned __int128)get(8) << sh;
        if (rem > 0)
            num |= (unsigned __int128)get(rem) << sh;
        out[2] = (int)(uint64_t)(num % sizes[2]);
        num /= sizes[2];
        out[1] = (int)(uint64_t)(num % sizes[1]);
        out[0] = (int)(uint32_t)(uint64_t)(num / sizes[1]);
    }
};

struct BitOut
{
    std::vector<unsigned char> bytes;
    uint32_t                   acc  = 0;
    int                        have = 0;

    void put(int nbits, uint32_t v)
    {
        for (int b = nbits - 1; b >= 0; --b)
        {
            acc = (acc << 1) | ((v >> b) & 1u);
            if (++have == 8)
            {
                bytes.push_back((unsigned char)acc);
                acc  = 0;
                have = 0;
            }
        }
    }
    void put3(int nbits, const unsigned sizes[3], const unsigned v[3])
    {
        // ((v0 * s1) + v1) * s2 + v2 as little-endian bytes
        unsigned char b[32];
        int           nb = 0;
        uint32_t      t  = v[0];
        do
        {
            b[nb++] = (unsigned char)(t & 0xff);
            t >>= 8;
        } while (t != 0);
        for (int i = 1; i < 3; ++i)
        {
            uint64_t c = v[i];
            int      j = 0;
            for (; j < nb; ++j)
            {
                c    = (uint64_t)b[j] * sizes[i] + c;
                b[j] = (unsigned char)(c & 0xff);
                c >>= 8;
            }
            while (c != 0)
            {
                b[j++] = (unsigned char)(c & 0xff);
                c >>= 8;
            }
            nb = j;
        }
        if (nbits >= nb * 8)
        {
            for (int j = 0; j < nb; ++j)
                put(8, b[j]);
            put(nbits - nb * 8, 0);
        }
        else
        {
            for (int j = 0; j < nb - 1; ++j)
                put(8, b[j]);
            put(nbits - (nb - 1) * 8, b[nb - 1]);
        }
    }
    void flush()
    {
        if (have > 0)
        {
            bytes.push_back((unsigned char)(acc << (8 - have)));
            acc  = 0;
            have = 0;
        }
    }
};

std::string g_err;

bool bad(const std::string& m)
{
    g_err = m;
    return false;
}

// Decodes the coordinate block of an XTC frame (after the box) into x
// (3 * natoms floats).
bool xtc_coords(XdrIn& in, int natoms, std::vector<float>& x, std::vector<unsigned char>& buf)
{
    int32_t lsize;
    if (!in.i32(lsize))
        return bad("truncated XTC frame");
    if (lsize != natoms)
        return bad("XTC frame: atom counts of header and coordinates differ");
    if (natoms <= 9)
    {
        x.resize((size_t)natoms * 3);
        for (int i = 0; i < natoms * 3; ++i)
            if (!in.f32(x[(size_t)i]))
                return bad("truncated XTC frame");
        return true;
    }
    float   precision;
    int32_t minint[3], maxint[3], smallidx, nbytes;
    if (!in.f32(precision) || !in.i32(minint[0]) || !in.i32(minint[1]) || !in.i32(minint[2]) ||
        !in.i32(maxint[0]) || !in.i32(maxint[1]) || !in.i32(maxint[2]) || !in.i32(smallidx) || !in.i32(nbytes))
        return bad("truncated XTC frame");
    if (!(precision > 0.0f) || smallidx < kFirstIdx || smallidx >= kLastIdx || nbytes < 0)
        return bad("corrupt XTC frame header");
    // every atom takes at least one bit of the stream, which the file holds
    if ((long long)natoms > 8LL * nbytes + 8 || (long long)nbytes > in.left())
        return bad("corrupt XTC frame: more atoms or bytes than the file holds");
    x.resize((size_t)natoms * 3);
    unsigned sizeint[3];
    int      bitsizeint[3] = {0, 0, 0}, bitsize = 0;
    bool     large = false;
    for (int d = 0; d < 3; ++d)
    {
        const int64_t s = (int64_t)maxint[d] - minint[d] + 1;
        if (s <= 0 || s > 0xffffffffLL)
            return bad("corrupt XTC frame bounds");
        sizeint[d] = (unsigned)s;
        large      = large || s > 0xffffff;
    }
    if (large)
        for (int d = 0; d < 3; ++d)
            bitsizeint[d] = bits_of(sizeint[d]);
    else
        bitsize = bits_of3(sizeint);
    buf.resize((size_t)nbytes);
    if (!in.opaque(buf.data(), (size_t)nbytes))
        return bad("truncated XTC frame");
    const float inv = (float)(1.0 / (double)precision);
    BitIn       bits{buf.data(), buf.size()};
    int         smaller  = kMagic[std::max(kFirstIdx, smallidx - 1)] / 2;
    int         smallnum = kMagic[smallidx] / 2;
    unsigned    sizesmall[3];
    sizesmall[0] = sizesmall[1] = sizesmall[2] = (unsigned)kMagic[smallidx];
    int   run = 0, i = 0;
    float* out = x.data();
    auto   emit = [&](const int c[3]) {
        *out++ = (float)c[0] * inv;
        *out++ = (float)c[1] * inv;
        *out++ = (float)c[2] * inv;
    };
    while (i < natoms)
    {
        int cur[3], prev[3];
        if (large)
            for (int d = 0; d < 3; ++d)
                cur[d] = (int)bits.get(bitsizeint[d]);
        else
            bits.get3(bitsize, sizeint, cur);
        ++i;
        for (int d = 0; d < 3; ++d)
        {
            cur[d] += minint[d];
            prev[d] = cur[d];
        }
        int is_smaller = 0;
        if (bits.get(1) == 1)
        {
            run        = (int)bits.get(5);
            is_smaller = run % 3;
            run -= is_smaller;
            --is_smaller;
        }
        if (run > 0)
        {
            if (i + run / 3 > natoms)
                return bad("corrupt XTC frame: run beyond the atom count");
            for (int k = 0; k < run; k += 3)
            {
                int c[3];
                bits.get3(smallidx, sizesmall, c);
                ++i;
                for (int d = 0; d < 3; ++d)
                    c[d] += prev[d] - smallnum;
                if (k == 0)
                {
                    // the first two atoms of a run were stored swapped
                    for (int d = 0; d < 3; ++d)
                        std::swap(c[d], prev[d]);
                    emit(prev);
                }
                else
                    for (int d = 0; d < 3; ++d)
                        prev[d] = c[d];
                emit(c);
            }
        }
        else
            emit(cur);
        smallidx += is_smaller;
        if (smallidx < kFirstIdx || smallidx >= kLastIdx)
            return bad("corrupt XTC frame: small index out of range");
        if (is_smaller < 0)
        {
            smallnum = smaller;
            smaller  = smallidx > kFirstIdx ? kMagic[smallidx - 1] / 2 : 0;
        }
        else if (is_smaller > 0)
        {
            smaller  = smallnum;
            smallnum = kMagic[smallidx] / 2;
        }
        sizesmall[0] = sizesmall[1] = sizesmall[2] = (unsigned)kMagic[smallidx];
        if (bits.over)
            return bad("corrupt XTC frame: bit stream shorter than its atoms");
    }
    return true;
}

// Encodes x (3 * natoms floats) as an XTC coordinate block.
bool xtc_write_coords(XdrOut& o, int natoms, const float* x, float precision)
{
    o.i32(natoms);
    if (natoms <= 9)
    {
        for (int i = 0; i < natoms * 3; ++i)
            o.f32(x[i]);
        return o.ok;
    }
    if (!(precision > 0.0f))
        precision = 1000.0f;
    o.f32(precision);
    std::vector<int> q((size_t)natoms * 3);
    int              minint[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, maxint[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    long long        mindiff = LLONG_MAX;
    for (int i = 0; i < natoms; ++i)
    {
        for (int d = 0; d < 3; ++d)
        {
            float f = x[(size_t)i * 3 + d] * precision;
            f       = f >= 0.0f ? f + 0.5f : f - 0.5f;
            if (!(std::fabs(f) < 2147483645.0f))
                return bad("XTC: coordinate too large for the precision");
            const int v          = (int)f;
            q[(size_t)i * 3 + d] = v;
            minint[d]            = std::min(minint[d], v);
            maxint[d]            = std::max(maxint[d], v);
        }
        if (i > 0)
        {
            long long diff = 0;
            for (int d = 0; d < 3; ++d)
                diff += std::llabs((long long)q[(size_t)i * 3 + d] - q[(size_t)(i - 1) * 3 + d]);
            mindiff = std::min(mindiff, diff);
        }
    }
    for (int d = 0; d < 3; ++d)
        o.i32(minint[d]);
    for (int d = 0; d < 3; ++d)
        o.i32(maxint[d]);
    unsigned sizeint[3];
    int      bitsizeint[3] = {0, 0, 0}, bitsize = 0;
    bool     large = false;
    for (int d = 0; d < 3; ++d)
    {
        const long long s = (long long)maxint[d] - minint[d] + 1;
        if (s > 0xffffffffLL)
            return bad("XTC: coordinate range too large for the precision");
        sizeint[d] = (unsigned)s;
        large      = large || s > 0xffffff;
    }
    if (large)
        for (int d = 0; d < 3; ++d)
            bitsizeint[d] = bits_of(sizeint[d]);
    else
        bitsize = bits_of3(sizeint);
    int smallidx = kFirstIdx;
    while (smallidx < kLastIdx - 1 && kMagic[smallidx] < mindiff)
        ++smallidx;
    o.i32(smallidx);
    const int maxidx   = std::min(kLastIdx - 1, smallidx + 8);
    const int minidx   = maxidx - 8;
    int       smaller  = kMagic[std::max(kFirstIdx, smallidx - 1)] / 2;
    int       smallnum = kMagic[smallidx] / 2;
    unsigned  sizesmall[3];
    sizesmall[0] = sizesmall[1] = sizesmall[2] = (unsigned)kMagic[smallidx];
    int       larger = kMagic[maxidx] / 2;
    BitOut    bits;
    int       i = 0, prevrun = -1;
    int       prev[3] = {0, 0, 0};
    auto      near = [](const int* a, const int* b, int lim) {
        return std::abs(a[0] - b[0]) < lim && std::abs(a[1] - b[1]) < lim && std::abs(a[2] - b[2]) < lim;
    };
    while (i < natoms)
    {
        int* cur        = q.data() + (size_t)i * 3;
        int  is_smaller = 0;
        bool is_small   = false;
        if (smallidx < maxidx && i >= 1 && near(cur, prev, larger))
            is_smaller = 1;
        else if (smallidx > minidx)
            is_smaller = -1;
        if (i + 1 < natoms && near(cur, cur + 3, smallnum))
        {
            // store the first two atoms of a run swapped
            for (int d = 0; d < 3; ++d)
                std::swap(cur[d], cur[3 + d]);
            is_small = true;
        }
        unsigned t[3];
        for (int d = 0; d < 3; ++d)
            t[d] = (unsigned)(cur[d] - minint[d]);
        if (large)
            for (int d = 0; d < 3; ++d)
                bits.put(bitsizeint[d], t[d]);
        else
            bits.put3(bitsize, sizeint, t);
        for (int d = 0; d < 3; ++d)
            prev[d] = cur[d];
        cur += 3;
        ++i;
        unsigned runw[24];
        int      run = 0;
        if (!is_small && is_smaller == -1)
            is_smaller = 0;
        while (is_small && run < 24)
        {
            if (is_smaller == -1)
            {
                long long s2 = 0;
                for (int d = 0; d < 3; ++d)
                    s2 += (long long)(cur[d] - prev[d]) * (cur[d] - prev[d]);
                if (s2 >= (long long)smaller * smaller)
                    is_smaller = 0;
            }
            for (int d = 0; d < 3; ++d)
            {
                runw[run++] = (unsigned)(cur[d] - prev[d] + smallnum);
                prev[d]     = cur[d];
            }
            ++i;
            cur += 3;
            is_small = i < natoms && near(cur, prev, smallnum);
        }
        if (run != prevrun || is_smaller != 0)
        {
            prevrun = run;
            bits.put(1, 1);
            bits.put(5, (unsigned)(run + is_smaller + 1));
        }
        else
            bits.put(1, 0);
        for (int k = 0; k < run; k += 3)
            bits.put3(smallidx, sizesmall, runw + k);
        if (is_smaller != 0)
        {
            smallidx += is_smaller;
            if (is_smaller < 0)
            {
                smallnum = smaller;
                smaller  = kMagic[smallidx - 1] / 2;
            }
            else
            {
                smaller  = smallnum;
                smallnum = kMagic[smallidx] / 2;
            }
            sizesmall[0] = sizesmall[1] = sizesmall[2] = (unsigned)kMagic[smallidx];
        }
    }
    bits.flush();
    o.i32((int32_t)bits.bytes.size());
    o.opaque(bits.bytes.data(), bits.bytes.size());
    return o.ok;
}

// ---------------------------------------------------------------------------
// Frames
// ---------------------------------------------------------------------------

// Reads the next XTC frame; false with g_err empty at a clean end of file.
bool xtc_frame(XdrIn& in, Frame& fr, std::vector<unsigned char>& buf)
{
    int32_t magic;
    g_err.clear();
    if (!in.i32(magic))
        return false;
    int32_t natoms, step;
    float   t, box[9];
    if (magic != kXtcMagic)
        return bad("not an XTC frame (magic " + std::to_string(magic) + ")");
    if (!in.i32(natoms) || !in.i32(step) || !in.f32(t))
        return bad("truncated XTC frame");
    for (float& b : box)
        if (!in.f32(b))
            return bad("truncated XTC frame");
    if (natoms < 1)
        return bad("XTC frame without atoms");
    fr.natoms = natoms;
    fr.step   = step;
    fr.time   = t;
    fr.xd.clear();
    return xtc_coords(in, natoms, fr.xf, buf);
}

// Reads the next TRR frame (positions only; velocities and forces skipped).
bool trr_frame(XdrIn& in, Frame& fr, bool keep_double)
{
    int32_t magic;
    g_err.clear();
    if (!in.i32(magic))
        return false;
    if (magic != kTrrMagic)
        return bad("not a TRR frame (magic " + std::to_string(magic) + ")");
    int32_t slen, len;
    char    version[16];
    if (!in.i32(slen) || !in.i32(len) || len < 0 || len > 15 || !in.opaque((unsigned char*)version, (size_t)len))
        return bad("truncated TRR header");
    version[len] = 0;
    if (slen != 13 || std::strcmp(version, "GMX_trn_file") != 0)
        return bad("TRR header without the GMX_trn_file version string");
    int32_t sz[11]; // ir, e, box, vir, pres, top, sym, x, v, f, natoms
    for (int32_t& v : sz)
        if (!in.i32(v))
            return bad("truncated TRR header");
    const int32_t box = sz[2], vir = sz[3], pres = sz[4], xs = sz[7], vs = sz[8], fs = sz[9], natoms = sz[10];
    if (sz[0] != 0 || sz[1] != 0 || sz[5] != 0 || sz[6] != 0)
        return bad("TRR frame with input-record, energy, topology or symmetry blocks (unsupported)");
    if (natoms < 0 || box < 0 || vir < 0 || pres < 0 || xs < 0 || vs < 0 || fs < 0)
        return bad("corrupt TRR header");
    const long long per = (long long)natoms * 3;
    int             real = 0;
    if (box)
        real = box / 9;
    else if (xs && per)
        real = (int)(xs / per);
    else if (vs && per)
        real = (int)(vs / per);
    else if (fs && per)
        real = (int)(fs / per);
    if (real != 4 && real != 8)
        return bad("TRR frame: cannot tell float from double precision");
    int32_t step, nre;
    if (!in.i32(step) || !in.i32(nre))
        return bad("truncated TRR header");
    double t = 0.0, lambda = 0.0;
    float  tf, lf;
    if (real == 4 ? !(in.f32(tf) && in.f32(lf)) : !(in.f64(t) && in.f64(lambda)))
        return bad("truncated TRR header");
    if (real == 4)
        t = tf;
    (void)lf;
    if ((box && box != 9 * real) || (vir && vir != 9 * real) || (pres && pres != 9 * real) ||
        (xs && xs != per * real) || (vs && vs != per * real) || (fs && fs != per * real))
        return bad("corrupt TRR header: block sizes disagree with the atom count");
    if (!xs)
        return bad("TRR frame without positions");
    if ((long long)box + vir + pres + xs + vs + fs > in.left())
        return bad("truncated TRR frame");
    if (!in.skip((long)box + vir + pres))
        return bad("truncated TRR frame");
    fr.natoms = natoms;
    fr.step   = step;
    fr.time   = t;
    fr.xf.clear();
    fr.xd.clear();
    if (real == 4)
    {
        fr.xf.resize((size_t)per);
        if (!in.f32s(fr.xf.data(), (size_t)per))
            return bad("truncated TRR frame");
    }
    else
    {
        std::vector<double>& dst = fr.xd;
        dst.resize((size_t)per);
        if (!in.f64s(dst.data(), (size_t)per))
            return bad("truncated TRR frame");
        if (!keep_double)
        {
            fr.xf.assign(dst.begin(), dst.end()); // rounded to float, as a mixed-precision reader does
            dst.clear();
        }
    }
    if (!in.skip((long)vs + fs))
        return bad("truncated TRR frame");
    return true;
}

int sniff(FILE* f)
{
    unsigned char b[4];
    const size_t  n = std::fread(b, 1, 4, f);
    std::rewind(f);
    if (n == 4)
    {
        const int32_t m = (int32_t)((uint32_t)b[0] << 24 | (uint32_t)b[1] << 16 | (uint32_t)b[2] << 8 | b[3]);
        if (m == kXtcMagic)
            return GC_TRAJ_XTC;
        if (m == kTrrMagic)
            return GC_TRAJ_TRR;
    }
    return GC_TRAJ_DUMP;
}

// Iterates the frames of a file; fn(frame) returns false to stop.
template <class Fn>
gc_status each_frame(const char* path, bool keep_double, int* format, Fn fn)
{
    File file(std::fopen(path, "rb"));
    if (!file.f)
        return fail(GC_ERR_IO, std::string("cannot open trajectory ") + path);
    const int fmt = sniff(file.f);
    if (format)
        *format = fmt;
    XdrIn                      in{file.f};
    Frame                      fr;
    std::vector<unsigned char> buf;
    if (fmt == GC_TRAJ_DUMP)
    {
        int n = 0, T = 0;
        if (std::fscanf(file.f, "%d %d", &n, &T) != 2 || n < 1 || T < 1)
            return fail(GC_ERR_INVALID, std::string("not an XTC, TRR or dump trajectory: ") + path);
        fr.natoms = n;
        fr.xd.resize((size_t)n * 3);
        for (int t = 0; t < T; ++t)
        {
            for (size_t i = 0; i < fr.xd.size(); ++i)
                if (std::fscanf(file.f, "%lf", &fr.xd[i]) != 1)
                    return fail(GC_ERR_INVALID, std::string("truncated dump file ") + path);
            fr.step = t;
            fr.time = t;
            if (!fn(fr))
                break;
        }
        return GC_OK;
    }
    for (long long idx = 0;; ++idx)
    {
        const bool ok = fmt == GC_TRAJ_XTC ? xtc_frame(in, fr, buf) : trr_frame(in, fr, keep_double);
        if (!ok)
        {
            if (g_err.empty())
                return GC_OK;
            return fail(GC_ERR_INVALID, std::string(path) + ", frame " + std::to_string(idx) + ": " + g_err);
        }
        if (!fn(fr))
            return GC_OK;
    }
}

} // namespace

namespace {

// The entry points: no C++ exception crosses the C ABI (a file announcing an
// absurd atom count could otherwise end the process with std::bad_alloc).
template <class F>
gc_status guarded(const char* what, F&& f)
{
    try
    {
        return f();
    }
    catch (const std::bad_alloc&)
    {
        return fail(GC_ERR_OUT_OF_MEMORY, std::string(what) + ": host allocation failed (a corrupt atom count?)");
    }
    catch (const std::exception& e)
    {
        return fail(GC_ERR_INTERNAL, std::string(what) + ": " + e.what());
    }
}

} // namespace

extern "C" {

static gc_status traj_info_impl(const char* path, int* format, int* natoms, int* nframes)
{
    if (!path)
        return fail(GC_ERR_INVALID, "gc_traj_info: null path");
    int       n = -1, T = 0;
    gc_status st = GC_OK;
    GC_TRY(each_frame(path, false, format, [&](const Frame& fr) {
        if (n >= 0 && fr.natoms != n)
        {
            st = fail(GC_ERR_INVALID, "gc_traj_info: the atom count changes between frames");
            return false;
        }
        n = fr.natoms;
        ++T;
        return true;
    }));
    GC_TRY(st);
    if (natoms)
        *natoms = n < 0 ? 0 : n;
    if (nframes)
        *nframes = T;
    return GC_OK;
}

static gc_status traj_read_impl(const char* path, const gc_traj_select* sel, double** xyz, int* natoms,
                                int* nframes)
{
    if (!path || !xyz || !natoms || !nframes)
        return fail(GC_ERR_INVALID, "gc_traj_read: null argument");
    *xyz                = nullptr;
    gc_traj_select s{};
    s.skip              = 1;
    if (sel)
        s = *sel;
    if (s.skip < 1)
        return fail(GC_ERR_INVALID, "The -skip value must be at least 1.");
    if (s.natoms < 0 || (s.natoms > 0 && !s.atoms))
        return fail(GC_ERR_INVALID, "gc_traj_read: selection without atom indices");
    // kept frames, one block of the selected atoms' positions each (no
    // reallocation of one growing buffer)
    std::vector<std::unique_ptr<double[]>> frames;
    int                 nsel = -1, file_atoms = -1;
    long long           analysed = 0; // frames inside the time window, as the reference counts frnr
    gc_status           st       = GC_OK;
    GC_TRY(each_frame(path, (s.flags & GC_TRAJ_KEEP_DOUBLE) != 0, nullptr, [&](const Frame& fr) {
        if (file_atoms < 0)
        {
            file_atoms = fr.natoms;
            nsel       = s.natoms > 0 ? s.natoms : fr.natoms;
            for (int i = 0; i < s.natoms; ++i)
                if (s.atoms[i] < 0 || s.atoms[i] >= fr.natoms)
                {
                    st = fail(GC_ERR_INVALID, "gc_traj_read: selected atom " + std::to_string(s.atoms[i]) +
                                                  " outside the file's " + std::to_string(fr.natoms) + " atoms");
                    return false;
                }
        }
        else if (fr.natoms != file_atoms)
        {
            st = fail(GC_ERR_INVALID, "gc_traj_read: the atom count changes between frames");
            return false;
        }
        if ((s.flags & GC_TRAJ_BEGIN) && fr.time < s.t_begin)
            return true;
        if ((s.flags & GC_TRAJ_END) && fr.time > s.t_end)
            return true;
        if (analysed++ % s.skip != 0)
            return true;
        const bool dbl = !fr.xd.empty();
        frames.emplace_back(new double[(size_t)nsel * 3]);
        double* out = frames.back().get();
        for (int i = 0; i < nsel; ++i)
        {
            const size_t a = (size_t)(s.natoms > 0 ? s.atoms[i] : i) * 3;
            for (int d = 0; d < 3; ++d)
                out[(size_t)i * 3 + d] = dbl ? fr.xd[a + d] : (double)fr.xf[a + d];
        }
        return true;
    }));
    GC_TRY(st);
    const size_t T = nsel > 0 ? frames.size() : 0;
    if (T == 0)
        return fail(GC_ERR_INVALID, "No trajectory frames were selected for analysis.");
    if (T > (size_t)gc::kMaxFrames)
        return fail(GC_ERR_INVALID, "gc_traj_read: more frames than the library handles");
    double* out = static_cast<double*>(std::malloc(sizeof(double) * T * (size_t)nsel * 3));
    if (!out)
        return fail(GC_ERR_OUT_OF_MEMORY, "gc_traj_read: host allocation failed");
    // x[atom][frame][dim]; with GC_TRAJ_CENTER each atom's mean position
    // (summed in frame order, then divided) is subtracted, as the reference
    // module does before the estimators run
    // every atom's sum still runs over its frames in order; the passes go
    // frame by frame, the transpose in tiles of frames
    std::vector<double> av((size_t)nsel * 3, 0.0);
    if (s.flags & GC_TRAJ_CENTER)
    {
        for (size_t t = 0; t < T; ++t)
        {
            const double* f = frames[t].get();
            for (size_t e = 0; e < (size_t)nsel * 3; ++e)
                av[e] += f[e];
        }
        for (double& v : av)
            v /= (double)T;
    }
    constexpr size_t kTile = 32;
    for (size_t t0 = 0; t0 < T; t0 += kTile)
    {
        const size_t t1 = std::min(T, t0 + kTile);
        for (int a = 0; a < nsel; ++a)
            for (size_t t = t0; t < t1; ++t)
                for (int d = 0; d < 3; ++d)
                    out[((size_t)a * T + t) * 3 + d] = frames[t][(size_t)a * 3 + d] - av[(size_t)a * 3 + d];
    }
    *xyz     = out;
    *natoms  = nsel;
    *nframes = (int)T;
    return GC_OK;
}

void gc_traj_free(double* xyz) { std::free(xyz); }

static gc_status traj_write_impl(const char* path, int format, const float* xyz, int natoms, int nframes,
                                 const float* box,
                        const double* times, float precision, int flags)
{
    if (!path || !xyz || natoms < 1 || nframes < 0)
        return fail(GC_ERR_INVALID, "gc_traj_write: need a path, positions, natoms >= 1 and nframes >= 0");
    if (format != GC_TRAJ_XTC && format != GC_TRAJ_TRR)
        return fail(GC_ERR_INVALID, "gc_traj_write: format must be GC_TRAJ_XTC or GC_TRAJ_TRR");
    File file(std::fopen(path, "wb"));
    if (!file.f)
        return fail(GC_ERR_IO, std::string("cannot create ") + path);
    XdrOut       o{file.f};
    const size_t per = (size_t)natoms * 3;
    const bool   dbl = format == GC_TRAJ_TRR && (flags & GC_TRAJ_KEEP_DOUBLE);
    for (int t = 0; t < nframes; ++t)
    {
        const float* x    = xyz + per * t;
        const float  zero[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const float* b    = box ? box + 9 * (size_t)t : zero;
        const double tm   = times ? times[t] : (double)t;
        if (format == GC_TRAJ_XTC)
        {
            o.i32(kXtcMagic);
            o.i32(natoms);
            o.i32(t);
            o.f32((float)tm);
            for (int i = 0; i < 9; ++i)
                o.f32(b[i]);
            g_err.clear();
            if (!xtc_write_coords(o, natoms, x, precision))
                return fail(g_err.empty() ? GC_ERR_IO : GC_ERR_INVALID,
                            g_err.empty() ? std::string("write error on ") + path : g_err);
        }
        else
        {
            const int real = dbl ? 8 : 4;
            o.i32(kTrrMagic);
            o.i32(13);
            o.i32(12);
            o.raw("GMX_trn_file", 12);
            const int32_t sz[11] = {0, 0, 9 * real, 0, 0, 0, 0, (int32_t)(per * real), 0, 0, natoms};
            for (int32_t v : sz)
                o.i32(v);
            o.i32(t);
            o.i32(0);
            if (dbl)
            {
                o.f64(tm);
                o.f64(0.0);
                for (int i = 0; i < 9; ++i)
                    o.f64(b[i]);
                for (size_t i = 0; i < per; ++i)
                    o.f64(x[i]);
            }
            else
            {
                o.f32((float)tm);
                o.f32(0.0f);
                for (int i = 0; i < 9; ++i)
                    o.f32(b[i]);
                for (size_t i = 0; i < per; ++i)
                    o.f32(x[i]);
            }
        }
        if (!o.ok)
            return fail(GC_ERR_IO, std::string("write error on ") + path);
    }
    return GC_OK;
}

// The guarded entry points follow.

gc_status gc_traj_info(const char* path, int* format, int* natoms, int* nframes)
{
    return guarded("gc_traj_info", [&] { return traj_info_impl(path, format, natoms, nframes); });
}

gc_status gc_traj_read(const char* path, const gc_traj_select* sel, double** xyz, int* natoms, int* nframes)
{
    return guarded("gc_traj_read", [&] { return traj_read_impl(path, sel, xyz, natoms, nframes); });
}

gc_status gc_traj_write(const char* path, int format, const float* xyz, int natoms, int nframes, const float* box,
                        const double* times, float precision, int flags)
{
    return guarded("gc_traj_write",
                   [&] { return traj_write_impl(path, format, xyz, natoms, nframes, box, times, precision, flags); });
}

} // extern "C"
