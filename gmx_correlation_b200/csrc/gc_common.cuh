// Shared device helpers for the gmx_correlation_b200 kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gc_geom.h"

namespace gc {

constexpr unsigned kFull = 0xffffffffu;

// Grid geometry of the joint KSG search for one pair: cells on component 0
// of atom a1 and component 0 of atom a2 (make_box2ind(x, 6, N, 0, dimx, ...),
// lib/kraskov.cpp:1294), cell index (int)(x*inveps) & (bs-1) (:69-71), query
// cell (int)(x/epsgrid) & (bs-1) (:271).
struct ScanGrid
{
    int    bs, ib, inveps;
    double epsgrid;
    __host__ __device__ explicit ScanGrid(int box)
        : bs(box), ib(box - 1), inveps(box / 4), epsgrid(4.0 / box)
    {
    }
    __device__ __forceinline__ int qcell(double c) const { return ((int)(c / epsgrid)) & ib; }
    __device__ __forceinline__ int cell(double c) const { return ((int)(c * (double)inveps)) & ib; }
    // Tie-break rank: scan position of the candidate's cell, then frame.
    __device__ __forceinline__ unsigned long long rank(int ix, int iy, double c1, double c2, int j, int T) const
    {
        const long long pos = scan_pos((cell(c1) - ix) & ib, (cell(c2) - iy) & ib, bs);
        return (unsigned long long)pos * (unsigned long long)T + (unsigned long long)j;
    }
};

__device__ __forceinline__ unsigned long long dbits(double v)
{
    return (unsigned long long)__double_as_longlong(v);
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        const unsigned long long w = __shfl_xor_sync(kFull, v, o);
        v                          = w > v ? w : v;
    }
    return v;
}

// Exact k-th smallest (1-based) 64-bit key among the warp's elements, by
// byte-wise radix selection with a 256-bin shared-memory histogram.  The
// callable `key(j, &k)` returns false for elements to skip; elements are
// j = 0 .. n-1, strided over the lanes.  Keys are re-generated each pass
// (no element storage).  top_shift is the bit offset of the most
// significant byte that can be non-zero (56 for IEEE doubles).  Returns the
// key; *below gets the number of elements with a strictly smaller key.
// Once the chosen byte bucket holds a single element, that element is the
// answer and one more pass reads it (distinct distances usually end the
// selection after the third of eight bytes).  Every lane returns the same
// values.
template <class KeyFn>
__device__ unsigned long long warp_select_u64(KeyFn&& key, int n, int k, int top_shift,
                                              unsigned* hist, int lane, int* below)
{
    unsigned long long prefix = 0ull, mask = 0ull;
    int                krem   = k;
#pragma unroll 1
    for (int shift = top_shift; shift >= 0; shift -= 8)
    {
#pragma unroll
        for (int b = 0; b < 8; ++b)
            hist[lane * 8 + b] = 0u;
        __syncwarp();
#pragma unroll 1
        for (int j = lane; j < n; j += 32)
        {
            unsigned long long kv;
            if (key(j, kv) && (kv & mask) == prefix)
                atomicAdd(&hist[(unsigned)(kv >> shift) & 255u], 1u);
        }
        __syncwarp();
        unsigned c[8], s = 0;
#pragma unroll
        for (int b = 0; b < 8; ++b)
        {
            c[b] = hist[lane * 8 + b];
            s += c[b];
        }
        unsigned incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const unsigned y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o)
                incl += y;
        }
        const unsigned excl  = incl - s;
        const bool     here  = excl < (unsigned)krem && (unsigned)krem <= incl;
        const unsigned owner = __ballot_sync(kFull, here);
        int            digit = 0;
        unsigned       bel = 0, cnt = 0;
        if (here)
        {
            unsigned acc = excl;
#pragma unroll
            for (int b = 0; b < 8; ++b)
            {
                if (acc + c[b] >= (unsigned)krem)
                {
                    digit = lane * 8 + b;
                    bel   = acc;
                    cnt   = c[b];
                    break;
                }
                acc += c[b];
            }
        }
        const int src = owner ? __ffs(owner) - 1 : 0;
        digit         = __shfl_sync(kFull, digit, src);
        bel           = __shfl_sync(kFull, bel, src);
        cnt           = __shfl_sync(kFull, cnt, src);
        krem -= (int)bel;
        prefix |= (unsigned long long)digit << shift;
        mask |= 0xFFull << shift;
        if (cnt == 1u && shift > 0)
        {
            // a single candidate carries this prefix: it is the k-th key (so
            // it is untied, and krem == 1); one more pass reads it whole
            unsigned long long found = 0ull;
            for (int j = lane; j < n; j += 32)
            {
                unsigned long long kv;
                if (key(j, kv) && (kv & mask) == prefix)
                    found = kv;
            }
            const unsigned hi = __reduce_or_sync(kFull, (unsigned)(found >> 32));
            const unsigned lo = __reduce_or_sync(kFull, (unsigned)found);
            __syncwarp();
            *below = k - krem;
            return ((unsigned long long)hi << 32) | lo;
        }
        __syncwarp();
    }
    *below = k - krem;
    return prefix;
}

} // namespace gc
