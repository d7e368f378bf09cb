// Index and grid geometry shared by host (api.cpp) and device code.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define GC_HD __host__ __device__
#else
#define GC_HD
#endif

namespace gc {

// Unordered pair index p = a1*(a1-1)/2 + a2 with a2 < a1 (the order of
// kraskov_corrmatrix's loop and MPI pair id, lib/correlation_core.cpp:404-408).
GC_HD inline void pair_from_index(long p, int* a1, int* a2)
{
    // a1 = floor((1 + sqrt(1 + 8p)) / 2), corrected for rounding.
    long x = (long)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
    while (x * (x - 1) / 2 > p)
        --x;
    while ((x + 1) * x / 2 <= p)
        ++x;
    *a1 = (int)x;
    *a2 = (int)(p - x * (x - 1) / 2);
}

// Box count of mir_xnyn (lib/kraskov.cpp:1260-1263): the smallest power of
// two with 0.5*BOX*BOX*K >= N.
GC_HD inline int ksg_box_count(int N, int K)
{
    int box = 1;
    while (0.5 * box * box * K < N)
        box *= 2;
    return box;
}

// Position, in the reference neighbour search's traversal, of the grid cell
// whose offset from the query cell is (dxm, dym) modulo bs: square shells
// jj = 0 .. bs/2-1 (the rows iy-jj and iy+jj for ascending ix, then the
// columns ix-jj and ix+jj), then the half layer jj = bs/2
// (neiK, lib/kraskov.cpp:273-341).
GC_HD inline long long scan_pos(int dxm, int dym, int bs)
{
    const int h  = bs / 2;
    const int rx = dxm >= h ? dxm - bs : dxm;
    const int ry = dym >= h ? dym - bs : dym;
    const int ax = rx < 0 ? -rx : rx, ay = ry < 0 ? -ry : ry;
    const int jj = ax > ay ? ax : ay;
    if (jj < h)
    {
        if (jj == 0)
            return 0;
        const long long base = (long long)(2 * jj - 1) * (2 * jj - 1);
        if (ay == jj)
            return base + (long long)(rx + jj) * 2 + (ry == jj ? 1 : 0);
        return base + 2 * (2 * jj + 1) + (rx == jj ? (2 * jj - 1) : 0) + (ry + jj - 1);
    }
    const long long base = (long long)(2 * h - 1) * (2 * h - 1);
    if (ry == -h)
        return base + (rx + h);
    return base + 2 * h + (ry + h - 1);
}

// Highest byte offset a tie-break rank key (scan position * T + frame) can
// use, for the radix selection over ranks (host only).
inline int rank_top_shift(int box, int T)
{
    const unsigned long long maxrank = (unsigned long long)box * box * (unsigned long long)T;
    const int                bits    = 64 - __builtin_clzll(maxrank);
    return ((bits - 1) / 8) * 8;
}

} // namespace gc
